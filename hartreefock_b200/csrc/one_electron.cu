// One-electron integrals on the device: overlap S, kinetic energy T and
// nuclear attraction V for every contracted shell pair, the matrices of
// QuantumMatrix.cpp:34-155 / IntegralsRepository.cpp:34-321 (GaussianOverlap,
// GaussianKinetic, GaussianNuclear), as hfg_one_electron (include/hfgpu.h).
//
// One warp per shell pair (La >= Lb), one kernel per pair class.  The lanes
// split the primitive pairs for S and T, and the (primitive pair, nucleus)
// products for V; the warp then sums its lanes with shuffles.
//   S, T: Obara-Saika in one dimension, s(i+1,j) = PA s(i,j) +
//         (i s(i-1,j) + j s(i,j-1))/2p and the same for j with PB, from
//         s(0,0) = sqrt(pi/p); t(i,j) = b(2j+1) s(i,j) - 2b^2 s(i,j+2)
//         - j(j-1)/2 s(i,j-2); S = sx sy sz, T = tx sy sz + sx ty sz + sx sy tz.
//   V:    the vertical recursion of the (La Lb|00) electron-repulsion class
//         with W - P replaced by C - P and rho/zeta by 1 (the nuclear
//         attraction recursion has that form), F_m scaled by -Z 2pi/p K, summed
//         over nuclei and primitive pairs, then the class's horizontal
//         recursion to (a|V|b).
// The Boys function is the engine's tabulated one (Taylor on the staged
// grid, downward recursion).  All FP64; normalisation as the ERIs
// (GaussianOrbital.cpp:25-30: radial (2a/pi)^(3/4) (4a)^(L/2) per primitive,
// 1/sqrt((2l-1)!!(2m-1)!!(2n-1)!!) per Cartesian component).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/hfgpu.h"
#include "eri_kernels.cuh"

namespace hfg {
hfg_status fail_external(hfg_status st, const std::string &msg);
const std::vector<double> &boys_table_for_external();
}  // namespace hfg

namespace hfg {
namespace {

struct OneShell {
  double c[3];
  int L, nprim, prim_off, ao;
};

// Cartesian exponent of component c of shell L along axis d, canonical order
// (QuantumNumbers.h:60-80): s; x y z; xx xy xz yy yz zz
__device__ __forceinline__ int cart_exp(int L, int c, int d) {
  if (L == 0) return 0;
  if (L == 1) return c == d ? 1 : 0;
  // d shells: (2,0,0) (1,1,0) (1,0,1) (0,2,0) (0,1,1) (0,0,2)
  constexpr int e[6][3] = {{2, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 2, 0}, {0, 1, 1}, {0, 0, 2}};
  return e[c][d];
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

constexpr int kOneWarps = 4;

template <int LA, int LB>
__global__ void __launch_bounds__(32 * kOneWarps) one_electron_kernel(const OneShell *__restrict__ shells,
                                                                       const int2 *__restrict__ pairs, int npairs,
                                                                       const double *__restrict__ expo,
                                                                       const double *__restrict__ coef,
                                                                       const double *__restrict__ nuc, int natoms,
                                                                       const double *__restrict__ boys, int n,
                                                                       double *S, double *T, double *V) {
  constexpr int NA = ncart(LA), NB = ncart(LB), LT = LA + LB;
  using Cls = EriClass<LA, LB, 0, 0, false>;
  constexpr int NE = Cls::kAcc;
  __shared__ double tab[kBoysGrid * kBoysRow];
  stage_boys<LT>(tab, boys);
  const int lane = threadIdx.x & 31;
  for (int w = blockIdx.x * kOneWarps + (threadIdx.x >> 5); w < npairs; w += gridDim.x * kOneWarps) {
    const OneShell A = shells[pairs[w].x], B = shells[pairs[w].y];
    const double AB0 = A.c[0] - B.c[0], AB1 = A.c[1] - B.c[1], AB2 = A.c[2] - B.c[2];
    const double ab2 = AB0 * AB0 + AB1 * AB1 + AB2 * AB2;
    double accS[NA * NB], accT[NA * NB], accE[NE];
#pragma unroll
    for (int x = 0; x < NA * NB; ++x) accS[x] = accT[x] = 0.0;
#pragma unroll
    for (int x = 0; x < NE; ++x) accE[x] = 0.0;
    const int npp = A.nprim * B.nprim;
    // S and T: lanes over primitive pairs
    for (int q = lane; q < npp; q += 32) {
      const int i = q / B.nprim, j = q - i * B.nprim;
      const double a = expo[A.prim_off + i], b = expo[B.prim_off + j], p = a + b, ip = 1.0 / p;
      const double K = exp(-a * b * ip * ab2);
      const double cc = coef[A.prim_off + i] * pow(2.0 * a / M_PI, 0.75) * pow(4.0 * a, 0.5 * LA) *
                        coef[B.prim_off + j] * pow(2.0 * b / M_PI, 0.75) * pow(4.0 * b, 0.5 * LB) * K;
      double s[3][LA + 1][LB + 3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double P = (a * A.c[d] + b * B.c[d]) * ip;
        const double PA = P - A.c[d], PB = P - B.c[d];
        s[d][0][0] = sqrt(M_PI * ip);
#pragma unroll
        for (int x = 0; x < LA; ++x) s[d][x + 1][0] = PA * s[d][x][0] + (x > 0 ? x * s[d][x - 1][0] : 0.0) * 0.5 * ip;
#pragma unroll
        for (int y = 0; y < LB + 2; ++y)
#pragma unroll
          for (int x = 0; x <= LA; ++x)
            s[d][x][y + 1] = PB * s[d][x][y] +
                             ((x > 0 ? x * s[d][x - 1][y] : 0.0) + (y > 0 ? y * s[d][x][y - 1] : 0.0)) * 0.5 * ip;
      }
#pragma unroll
      for (int ca = 0; ca < NA; ++ca)
#pragma unroll
        for (int cb = 0; cb < NB; ++cb) {
          double sd[3], td[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const int x = cart_exp(LA, ca, d), y = cart_exp(LB, cb, d);
            sd[d] = s[d][x][y];
            td[d] = b * (2 * y + 1) * s[d][x][y] - 2.0 * b * b * s[d][x][y + 2] -
                    (y >= 2 ? 0.5 * y * (y - 1) * s[d][x][y - 2] : 0.0);
          }
          accS[ca * NB + cb] += cc * sd[0] * sd[1] * sd[2];
          accT[ca * NB + cb] += cc * (td[0] * sd[1] * sd[2] + sd[0] * td[1] * sd[2] + sd[0] * sd[1] * td[2]);
        }
    }
    // V: lanes over (primitive pair, nucleus)
    for (int q = lane; q < npp * natoms; q += 32) {
      const int pq = q / natoms, c = q - pq * natoms;
      const int i = pq / B.nprim, j = pq - i * B.nprim;
      const double a = expo[A.prim_off + i], b = expo[B.prim_off + j], p = a + b, ip = 1.0 / p;
      const double K = exp(-a * b * ip * ab2);
      const double cc = coef[A.prim_off + i] * pow(2.0 * a / M_PI, 0.75) * pow(4.0 * a, 0.5 * LA) *
                        coef[B.prim_off + j] * pow(2.0 * b / M_PI, 0.75) * pow(4.0 * b, 0.5 * LB) * K;
      double P[3], PA[3], PC[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        P[d] = (a * A.c[d] + b * B.c[d]) * ip;
        PA[d] = P[d] - A.c[d];
        PC[d] = P[d] - nuc[4 * c + d];
      }
      const double Tb = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
      double F[LT + 1];
      boys_eval<LT, double>(F, Tb, -nuc[4 * c + 3] * 2.0 * M_PI * ip * cc, tab);
      Cls::template prim<double>(accE, F, PA[0], PA[1], PA[2], -PC[0], -PC[1], -PC[2], 0.5 * ip, 1.0, 0.0, 0.0, 0.0,
                                 0.0, 0.0);
    }
#pragma unroll
    for (int x = 0; x < NA * NB; ++x) {
      accS[x] = warp_sum(accS[x]);
      accT[x] = warp_sum(accT[x]);
    }
#pragma unroll
    for (int x = 0; x < NE; ++x) accE[x] = warp_sum(accE[x]);
    if (lane == 0) {
      double outV[NA * NB];
      Cls::template hrr<double>(outV, accE, AB0, AB1, AB2, 0.0, 0.0, 0.0);
#pragma unroll
      for (int ca = 0; ca < NA; ++ca)
#pragma unroll
        for (int cb = 0; cb < NB; ++cb) {
          const double nn = comp_norm<LA>(ca) * comp_norm<LB>(cb);
          const long long r = A.ao + ca, s = B.ao + cb;
          const int x = ca * NB + cb;
          S[r * n + s] = S[s * n + r] = nn * accS[x];
          T[r * n + s] = T[s * n + r] = nn * accT[x];
          V[r * n + s] = V[s * n + r] = nn * outV[x];
        }
    }
  }
}

// Dipole moment integrals about the origin (MomentMatrix::Calculate,
// QuantumMatrix.cpp:61-98, through GaussianMoment::CalculateMoment,
// GaussianMoment.cpp:44-90): per axis d, m(i,j) = s(i+1,j) + A_d s(i,j), so
// that M_d = m_d(a_d, b_d) s(a_e, b_e) s(a_f, b_f) over the other two axes.
// One warp per shell pair, lanes over primitive pairs, warp sums.
template <int LA, int LB>
__global__ void __launch_bounds__(32 * kOneWarps) moment_kernel(const OneShell *__restrict__ shells,
                                                                 const int2 *__restrict__ pairs, int npairs,
                                                                 const double *__restrict__ expo,
                                                                 const double *__restrict__ coef, int n, double *Mx,
                                                                 double *My, double *Mz) {
  constexpr int NA = ncart(LA), NB = ncart(LB);
  const int lane = threadIdx.x & 31;
  for (int w = blockIdx.x * kOneWarps + (threadIdx.x >> 5); w < npairs; w += gridDim.x * kOneWarps) {
    const OneShell A = shells[pairs[w].x], B = shells[pairs[w].y];
    const double AB0 = A.c[0] - B.c[0], AB1 = A.c[1] - B.c[1], AB2 = A.c[2] - B.c[2];
    const double ab2 = AB0 * AB0 + AB1 * AB1 + AB2 * AB2;
    double acc[3][NA * NB];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int x = 0; x < NA * NB; ++x) acc[d][x] = 0.0;
    const int npp = A.nprim * B.nprim;
    for (int q = lane; q < npp; q += 32) {
      const int i = q / B.nprim, j = q - i * B.nprim;
      const double a = expo[A.prim_off + i], b = expo[B.prim_off + j], p = a + b, ip = 1.0 / p;
      const double K = exp(-a * b * ip * ab2);
      const double cc = coef[A.prim_off + i] * pow(2.0 * a / M_PI, 0.75) * pow(4.0 * a, 0.5 * LA) *
                        coef[B.prim_off + j] * pow(2.0 * b / M_PI, 0.75) * pow(4.0 * b, 0.5 * LB) * K;
      double s[3][LA + 2][LB + 1], m[3][LA + 1][LB + 1];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double P = (a * A.c[d] + b * B.c[d]) * ip;
        const double PA = P - A.c[d], PB = P - B.c[d];
        s[d][0][0] = sqrt(M_PI * ip);
#pragma unroll
        for (int x = 0; x < LA + 1; ++x) s[d][x + 1][0] = PA * s[d][x][0] + (x > 0 ? x * s[d][x - 1][0] : 0.0) * 0.5 * ip;
#pragma unroll
        for (int y = 0; y < LB; ++y)
#pragma unroll
          for (int x = 0; x <= LA + 1; ++x)
            s[d][x][y + 1] = PB * s[d][x][y] +
                             ((x > 0 ? x * s[d][x - 1][y] : 0.0) + (y > 0 ? y * s[d][x][y - 1] : 0.0)) * 0.5 * ip;
#pragma unroll
        for (int x = 0; x <= LA; ++x)
#pragma unroll
          for (int y = 0; y <= LB; ++y) m[d][x][y] = s[d][x + 1][y] + A.c[d] * s[d][x][y];
      }
#pragma unroll
      for (int ca = 0; ca < NA; ++ca)
#pragma unroll
        for (int cb = 0; cb < NB; ++cb) {
          const int x0 = cart_exp(LA, ca, 0), y0 = cart_exp(LB, cb, 0);
          const int x1 = cart_exp(LA, ca, 1), y1 = cart_exp(LB, cb, 1);
          const int x2 = cart_exp(LA, ca, 2), y2 = cart_exp(LB, cb, 2);
          const double s0 = s[0][x0][y0], s1 = s[1][x1][y1], s2 = s[2][x2][y2];
          acc[0][ca * NB + cb] += cc * m[0][x0][y0] * s1 * s2;
          acc[1][ca * NB + cb] += cc * s0 * m[1][x1][y1] * s2;
          acc[2][ca * NB + cb] += cc * s0 * s1 * m[2][x2][y2];
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int x = 0; x < NA * NB; ++x) acc[d][x] = warp_sum(acc[d][x]);
    if (lane == 0) {
      double *M[3] = {Mx, My, Mz};
#pragma unroll
      for (int ca = 0; ca < NA; ++ca)
#pragma unroll
        for (int cb = 0; cb < NB; ++cb) {
          const double nn = comp_norm<LA>(ca) * comp_norm<LB>(cb);
          const long long r = A.ao + ca, c = B.ao + cb;
#pragma unroll
          for (int d = 0; d < 3; ++d) M[d][r * n + c] = M[d][c * n + r] = nn * acc[d][ca * NB + cb];
        }
    }
  }
}

template <int LA, int LB>
void launch_one(const OneShell *shells, const int2 *pairs, int npairs, const double *expo, const double *coef,
                const double *nuc, int natoms, const double *boys, int n, double *S, double *T, double *V,
                int num_sms, cudaStream_t st) {
  if (npairs == 0) return;
  const int blocks = std::min((npairs + kOneWarps - 1) / kOneWarps, num_sms * 4);
  one_electron_kernel<LA, LB><<<blocks, 32 * kOneWarps, 0, st>>>(shells, pairs, npairs, expo, coef, nuc, natoms, boys,
                                                                  n, S, T, V);
}

template <class T>
struct DeviceArray {
  T *p = nullptr;
  ~DeviceArray() {
    if (p) cudaFree(p);
  }
  cudaError_t upload(const std::vector<T> &v) {
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(1, v.size()) * sizeof(T));
    if (e != cudaSuccess || v.empty()) return e;
    e = cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    // the staged copy's DMA runs on the legacy stream; the kernels below run
    // on a stream of their own
    return e == cudaSuccess ? cudaStreamSynchronize(cudaStreamLegacy) : e;
  }
};

}  // namespace
}  // namespace hfg

namespace hfg {
namespace {
// S, T, V (nuclei given) and / or the dipole moment matrices (Mx given)
hfg_status one_electron_all(const hfg_shells *sh, const double *nuc_xyz, const int32_t *nuc_Z, int32_t natoms,
                            int32_t device, double *S, double *T, double *V, double *Mx, double *My, double *Mz);
}  // namespace
}  // namespace hfg

extern "C" hfg_status hfg_one_electron(const hfg_shells *sh, const double *nuc_xyz, const int32_t *nuc_Z,
                                       int32_t natoms, int32_t device, double *S, double *T, double *V) {
  using namespace hfg;
  if (!sh || sh->nshells < 1 || sh->nbf < 1 || !nuc_xyz || !nuc_Z || natoms < 1 || !S || !T || !V)
    return fail_external(HFG_INVALID_ARG, "hfg_one_electron: arguments");
  return one_electron_all(sh, nuc_xyz, nuc_Z, natoms, device, S, T, V, nullptr, nullptr, nullptr);
}

extern "C" hfg_status hfg_moments(const hfg_shells *sh, int32_t device, double *Mx, double *My, double *Mz) {
  using namespace hfg;
  if (!sh || sh->nshells < 1 || sh->nbf < 1 || !Mx || !My || !Mz)
    return fail_external(HFG_INVALID_ARG, "hfg_moments: arguments");
  return one_electron_all(sh, nullptr, nullptr, 0, device, nullptr, nullptr, nullptr, Mx, My, Mz);
}

namespace hfg {
namespace {
hfg_status one_electron_all(const hfg_shells *sh, const double *nuc_xyz, const int32_t *nuc_Z, int32_t natoms,
                            int32_t device, double *S, double *T, double *V, double *Mx, double *My, double *Mz) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail_external(HFG_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail_external(HFG_INVALID_ARG, "device out of range");
  const int ns = sh->nshells, n = sh->nbf;
  int nexp = 0;
  std::vector<OneShell> shells(ns);
  for (int s = 0; s < ns; ++s) {
    const int L = sh->L[s];
    if (L < 0 || L > 2) return fail_external(HFG_UNSUPPORTED_L, "hfg_one_electron: shell above d");
    shells[s] = OneShell{{sh->center[3 * s], sh->center[3 * s + 1], sh->center[3 * s + 2]},
                         L, sh->nprim[s], sh->prim_offset[s], sh->ao_offset[s]};
    nexp = std::max(nexp, sh->prim_offset[s] + sh->nprim[s]);
    if (sh->ao_offset[s] < 0 || sh->ao_offset[s] + ncart(L) > n)
      return fail_external(HFG_INVALID_ARG, "hfg_one_electron: AO offsets outside nbf");
  }
  // pairs (a, b) with L_a >= L_b, one list per pair class (00 10 11 20 21 22)
  std::vector<int2> lists[3][3];
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b <= a; ++b) {
      int x = a, y = b;
      if (shells[x].L < shells[y].L) std::swap(x, y);
      lists[shells[x].L][shells[y].L].push_back(make_int2(x, y));
    }
  std::vector<int2> all;
  int off[3][3] = {}, cnt[3][3] = {};
  for (int la = 0; la < 3; ++la)
    for (int lb = 0; lb <= la; ++lb) {
      off[la][lb] = (int)all.size();
      cnt[la][lb] = (int)lists[la][lb].size();
      all.insert(all.end(), lists[la][lb].begin(), lists[la][lb].end());
    }
  std::vector<double> nuc(4 * (size_t)std::max(natoms, 1));
  for (int c = 0; c < natoms; ++c) {
    for (int d = 0; d < 3; ++d) nuc[4 * c + d] = nuc_xyz[3 * c + d];
    nuc[4 * c + 3] = (double)nuc_Z[c];
  }
  cudaError_t e = cudaSetDevice(device);
  int num_sms = 148;
  // a stream of this call's own: nothing here waits on, or is waited on by,
  // the legacy default stream that other host threads share
  struct OwnStream {
    cudaStream_t s = nullptr;
    ~OwnStream() {
      if (s) cudaStreamDestroy(s);
    }
  } os;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&os.s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device);
  DeviceArray<OneShell> d_sh;
  DeviceArray<int2> d_pairs;
  DeviceArray<double> d_exp, d_coef, d_nuc, d_boys, d_out;
  if (e == cudaSuccess) e = d_sh.upload(shells);
  if (e == cudaSuccess) e = d_pairs.upload(all);
  if (e == cudaSuccess) e = d_exp.upload(std::vector<double>(sh->exponent, sh->exponent + nexp));
  if (e == cudaSuccess) e = d_coef.upload(std::vector<double>(sh->coefficient, sh->coefficient + nexp));
  if (e == cudaSuccess) e = d_nuc.upload(nuc);
  if (e == cudaSuccess) e = d_boys.upload(boys_table_for_external());
  const size_t nn = (size_t)n * n;
  if (e == cudaSuccess) e = cudaMalloc(&d_out.p, 6 * nn * sizeof(double));
  if (e == cudaSuccess) e = cudaMemsetAsync(d_out.p, 0, 6 * nn * sizeof(double), os.s);
  if (e != cudaSuccess) return fail_external(HFG_OOM_BUDGET, std::string("hfg_one_electron: ") + cudaGetErrorString(e));
  double *dS = d_out.p, *dT = dS + nn, *dV = dT + nn, *dMx = dV + nn, *dMy = dMx + nn, *dMz = dMy + nn;
  if (S) {
#define HFG_ONE(LA, LB)                                                                                              \
  launch_one<LA, LB>(d_sh.p, d_pairs.p + off[LA][LB], cnt[LA][LB], d_exp.p, d_coef.p, d_nuc.p, natoms, d_boys.p, n, \
                     dS, dT, dV, num_sms, os.s)
    HFG_ONE(0, 0);
    HFG_ONE(1, 0);
    HFG_ONE(1, 1);
    HFG_ONE(2, 0);
    HFG_ONE(2, 1);
    HFG_ONE(2, 2);
#undef HFG_ONE
  }
  if (Mx) {
#define HFG_MOM(LA, LB)                                                                                           \
  if (cnt[LA][LB])                                                                                                \
    moment_kernel<LA, LB><<<std::min((cnt[LA][LB] + kOneWarps - 1) / kOneWarps, num_sms * 4), 32 * kOneWarps, 0, \
                            os.s>>>(d_sh.p, d_pairs.p + off[LA][LB], cnt[LA][LB], d_exp.p, d_coef.p, n, dMx, dMy, dMz)
    HFG_MOM(0, 0);
    HFG_MOM(1, 0);
    HFG_MOM(1, 1);
    HFG_MOM(2, 0);
    HFG_MOM(2, 1);
    HFG_MOM(2, 2);
#undef HFG_MOM
  }
  e = cudaGetLastError();
  if (S) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(S, dS, nn * sizeof(double), cudaMemcpyDeviceToHost, os.s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(T, dT, nn * sizeof(double), cudaMemcpyDeviceToHost, os.s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(V, dV, nn * sizeof(double), cudaMemcpyDeviceToHost, os.s);
  }
  if (Mx) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(Mx, dMx, nn * sizeof(double), cudaMemcpyDeviceToHost, os.s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(My, dMy, nn * sizeof(double), cudaMemcpyDeviceToHost, os.s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(Mz, dMz, nn * sizeof(double), cudaMemcpyDeviceToHost, os.s);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(os.s);
  if (e != cudaSuccess) return fail_external(HFG_DEVICE_ERROR, std::string("hfg_one_electron: ") + cudaGetErrorString(e));
  return HFG_OK;
}
}  // namespace
}  // namespace hfg
