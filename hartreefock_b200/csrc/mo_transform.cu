// AO -> MO transform of the two-electron integrals and the MP2 energies,
// for the post-HF consumers of the integral tables:
// MolecularOrbitalsIntegralsRepository::getElectronElectron
// (IntegralsRepository.h:190-291), RestrictedHartreeFock::CalculateMp2Energy
// (RestrictedHartreeFock.cpp:251-288) and
// UnrestrictedHartreeFock::CalculateMp2Energy (UnrestrictedHartreeFock.cpp:295-375).
//
// The reference transforms one MO integral at a time (four nested
// quarter-contractions, cached per index tuple).  Here the whole (ia|jb)
// block is two DGEMMs over the unpacked AO table (the 8-fold packed table
// of the context's stored mode, expanded on the device):
//   K[(l s),(j b)] = C[l][i0+j] C[s][a0+b]            (pair coefficients)
//   Y = M K,  M[(m n),(l s)] = (mn|ls)                (N^2 x N^2 times N^2 x ov)
//   X = K^T Y = (ia|jb)                              (ov x ov)
// FP64 throughout; cuBLAS for the two plain GEMMs.  Memory: N^4 + N^4/8
// doubles for the tables, 2 N^2 ov for K and Y.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/hfgpu.h"

namespace hfg {
hfg_status fail_external(hfg_status st, const std::string &msg);
}

namespace {

__device__ __forceinline__ long long tri(long long a, long long b) {
  return a < b ? b * (b + 1) / 2 + a : a * (a + 1) / 2 + b;
}

// full[(m n),(l s)] = packed[T(T(m,n), T(l,s))] (IntegralsRepository.h:151-162)
__global__ void unpack_eri(const double *__restrict__ packed, double *__restrict__ full, int n) {
  const long long nn = (long long)n * n, total = nn * nn;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
    const long long r = x / nn, c = x - r * nn;
    const int m = (int)(r / n), nu = (int)(r - (long long)m * n), l = (int)(c / n), s = (int)(c - (long long)l * n);
    full[x] = packed[tri(tri(m, nu), tri(l, s))];
  }
}

// K[(l s),(j b)] = Cj[l][j0+j] Cb[s][b0+b], Cj and Cb row-major n x n
__global__ void pair_coefficients(const double *__restrict__ Cj, int j0, int nj, const double *__restrict__ Cb, int b0,
                                  int nb, int n, double *__restrict__ K) {
  const long long ov = (long long)nj * nb, total = (long long)n * n * ov;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
    const long long r = x / ov, c = x - r * ov;
    const int l = (int)(r / n), s = (int)(r - (long long)l * n), j = (int)(c / nb), b = (int)(c - (long long)j * nb);
    K[x] = Cj[(long long)l * n + j0 + j] * Cb[(long long)s * n + b0 + b];
  }
}

// sum over i, j occupied and a, b virtual of (ia|jb)[2(ia|jb) - (ib|ja)] /
// (e_i + e_j - e_a - e_b), X[(i a),(j b)] = (ia|jb)
__global__ void mp2_energy(const double *__restrict__ X, const double *__restrict__ eps, int no, int nv,
                           double *out) {
  const long long ov = (long long)no * nv, total = ov * ov;
  double acc = 0;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
    const long long r = x / ov, c = x - r * ov;
    const int i = (int)(r / nv), a = (int)(r - (long long)i * nv), j = (int)(c / nv), b = (int)(c - (long long)j * nv);
    const double iajb = X[x], ibja = X[((long long)i * nv + b) * ov + (long long)j * nv + a];
    acc += iajb * (2.0 * iajb - ibja) / (eps[i] + eps[j] - eps[no + a] - eps[no + b]);
  }
  __shared__ double part[256];
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(out, part[0]);
}

// sum over the block of X^2 / (e_i + e_j - e_a - e_b), X[(i a),(j b)] with
// row stride `ldx` (columns j*nb + b); the four index ranges read their
// orbital energies from ei, ea, ej, eb
__global__ void mp2_sum_sq(const double *__restrict__ X, long long ldx, int ni, int na, int nj, int nb,
                           const double *__restrict__ ei, const double *__restrict__ ea, const double *__restrict__ ej,
                           const double *__restrict__ eb, double *out) {
  const long long rows = (long long)ni * na, cols = (long long)nj * nb, total = rows * cols;
  double acc = 0;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
    const long long r = x / cols, c = x - r * cols;
    const int i = (int)(r / na), a = (int)(r - (long long)i * na), j = (int)(c / nb), b = (int)(c - (long long)j * nb);
    const double v = X[r * ldx + c];
    acc += v * v / (ei[i] + ej[j] - ea[a] - eb[b]);
  }
  __shared__ double part[256];
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(out, part[0]);
}

int grid_for(long long total) { return (int)std::min<long long>(148LL * 32, (total + 255) / 256 + 1); }

struct Buffers {
  std::vector<void *> ptrs;
  ~Buffers() {
    for (void *p : ptrs) cudaFree(p);
  }
  cudaError_t get(double **p, size_t count) {
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(double));
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
};

struct Blas {
  cublasHandle_t h = nullptr;
  ~Blas() {
    if (h) cublasDestroy(h);
  }
};

// The unpacked AO table M[(m n),(l s)] of the context (stored-mode build),
// sized for `ov_max` columns of pair coefficients in the blocks that follow.
struct MoTables {
  int n = 0;
  double *M = nullptr, *K1 = nullptr, *K2 = nullptr, *Y = nullptr;
  long long cap = 0;  // columns of K1, K2, Y
  Blas blas;
};

hfg_status prepare(hfg_ctx *ctx, long long ov_max, cudaStream_t s, Buffers &buf, MoTables &t, const char *who) {
  const int n = hfg_ctx_nbf(ctx);
  if (n <= 0) return hfg::fail_external(HFG_INVALID_ARG, std::string(who) + ": context without a single molecule");
  const long long nn = (long long)n * n;
  const int64_t count = hfg_packed_size(n);
  size_t freeb = 0, totalb = 0;
  cudaMemGetInfo(&freeb, &totalb);
  const double need = 8.0 * ((double)count + (double)nn * nn + 3.0 * nn * ov_max);
  if (need > 0.9 * (double)freeb)
    return hfg::fail_external(HFG_OOM_BUDGET, std::string(who) + ": the unpacked AO table does not fit (" +
                                                  std::to_string(need / 1e9) + " GB needed)");
  double *packed = nullptr;
  cudaError_t e = buf.get(&packed, (size_t)count);
  if (e == cudaSuccess) e = buf.get(&t.M, (size_t)(nn * nn));
  if (e == cudaSuccess) e = buf.get(&t.K1, (size_t)(nn * ov_max));
  if (e == cudaSuccess) e = buf.get(&t.K2, (size_t)(nn * ov_max));
  if (e == cudaSuccess) e = buf.get(&t.Y, (size_t)(nn * ov_max));
  if (e != cudaSuccess) return hfg::fail_external(HFG_OOM_BUDGET, std::string(who) + ": " + cudaGetErrorString(e));
  hfg_status st = hfg_eri_packed_device(ctx, packed, count, s);
  if (st != HFG_OK) return st;
  // stream 0 means the context's own stream for the packed build: finish it
  // before the kernels below read the table
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return hfg::fail_external(HFG_DEVICE_ERROR, std::string(who) + ": " + cudaGetErrorString(e));
  unpack_eri<<<grid_for(nn * nn), 256, 0, s>>>(packed, t.M, n);
  if (cublasCreate(&t.blas.h) != CUBLAS_STATUS_SUCCESS || cublasSetStream(t.blas.h, s) != CUBLAS_STATUS_SUCCESS)
    return hfg::fail_external(HFG_DEVICE_ERROR, std::string(who) + ": cuBLAS handle");
  t.n = n;
  t.cap = ov_max;
  return HFG_OK;
}

// One orbital index range of a transformed block: columns [first, first+count)
// of the coefficient matrix C (row-major n x n, AO rows, MO columns).
struct Range {
  const double *C;
  int first, count;
};

// X[(i a),(j b)] = (i a | j b), each of the four indices over its own range
// and coefficient matrix.
hfg_status block(MoTables &t, Range i, Range a, Range j, Range b, double *dX, cudaStream_t s, const char *who) {
  const int n = t.n;
  const long long nn = (long long)n * n, ov1 = (long long)i.count * a.count, ov2 = (long long)j.count * b.count;
  if (ov1 > t.cap || ov2 > t.cap) return hfg::fail_external(HFG_INVALID_ARG, std::string(who) + ": block size");
  pair_coefficients<<<grid_for(nn * ov1), 256, 0, s>>>(i.C, i.first, i.count, a.C, a.first, a.count, n, t.K1);
  pair_coefficients<<<grid_for(nn * ov2), 256, 0, s>>>(j.C, j.first, j.count, b.C, b.first, b.count, n, t.K2);
  const double one = 1.0, zero = 0.0;
  // row-major Y = M K2  <=>  column-major Y^T = K2^T M^T
  if (cublasDgemm(t.blas.h, CUBLAS_OP_N, CUBLAS_OP_N, (int)ov2, (int)nn, (int)nn, &one, t.K2, (int)ov2, t.M, (int)nn,
                  &zero, t.Y, (int)ov2) != CUBLAS_STATUS_SUCCESS)
    return hfg::fail_external(HFG_DEVICE_ERROR, std::string(who) + ": DGEMM M K");
  // row-major X = K1^T Y  <=>  column-major X^T = Y^T K1
  if (cublasDgemm(t.blas.h, CUBLAS_OP_N, CUBLAS_OP_T, (int)ov2, (int)ov1, (int)nn, &one, t.Y, (int)ov2, t.K1, (int)ov1,
                  &zero, dX, (int)ov2) != CUBLAS_STATUS_SUCCESS)
    return hfg::fail_external(HFG_DEVICE_ERROR, std::string(who) + ": DGEMM K^T Y");
  return HFG_OK;
}

hfg_status finish(cudaStream_t s, const char *who) {
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return hfg::fail_external(HFG_DEVICE_ERROR, std::string(who) + ": " + cudaGetErrorString(e));
  return HFG_OK;
}

hfg_status transform(hfg_ctx *ctx, const double *dC, int i0, int ni, int a0, int na, double *dX, cudaStream_t s,
                     Buffers &buf) {
  const int n = hfg_ctx_nbf(ctx);
  if (n <= 0) return hfg::fail_external(HFG_INVALID_ARG, "hfg_mo_eri_ovov: context without a single molecule");
  if (!dC || !dX || ni < 1 || na < 1 || i0 < 0 || a0 < 0 || i0 + ni > n || a0 + na > n)
    return hfg::fail_external(HFG_INVALID_ARG, "hfg_mo_eri_ovov: orbital ranges");
  MoTables t;
  hfg_status st = prepare(ctx, (long long)ni * na, s, buf, t, "hfg_mo_eri_ovov");
  if (st != HFG_OK) return st;
  st = block(t, {dC, i0, ni}, {dC, a0, na}, {dC, i0, ni}, {dC, a0, na}, dX, s, "hfg_mo_eri_ovov");
  if (st != HFG_OK) return st;
  return finish(s, "hfg_mo_eri_ovov");
}

}  // namespace

extern "C" hfg_status hfg_mo_eri_ovov(hfg_ctx *ctx, const double *dC, int32_t i0, int32_t ni, int32_t a0, int32_t na,
                                      double *dX, void *stream) {
  if (!ctx) return hfg::fail_external(HFG_INVALID_ARG, "hfg_mo_eri_ovov: null context");
  Buffers buf;
  return transform(ctx, dC, i0, ni, a0, na, dX, static_cast<cudaStream_t>(stream), buf);
}

extern "C" hfg_status hfg_mp2_rhf(hfg_ctx *ctx, const double *C, const double *eps, int32_t nocc, double *e_mp2) {
  if (!ctx || !C || !eps || !e_mp2) return hfg::fail_external(HFG_INVALID_ARG, "hfg_mp2_rhf: arguments");
  const int n = hfg_ctx_nbf(ctx);
  if (n <= 0 || nocc < 1 || nocc >= n) return hfg::fail_external(HFG_INVALID_ARG, "hfg_mp2_rhf: occupied count");
  const int nv = n - nocc;
  Buffers buf;
  double *dC = nullptr, *dE = nullptr, *dX = nullptr, *dOut = nullptr;
  cudaError_t e = buf.get(&dC, (size_t)n * n);
  if (e == cudaSuccess) e = buf.get(&dE, (size_t)n);
  if (e == cudaSuccess) e = buf.get(&dX, (size_t)nocc * nv * nocc * nv);
  if (e == cudaSuccess) e = buf.get(&dOut, 1);
  if (e == cudaSuccess) e = cudaMemcpy(dC, C, sizeof(double) * n * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dE, eps, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);  // staged copies landed
  if (e == cudaSuccess) e = cudaMemset(dOut, 0, sizeof(double));
  if (e != cudaSuccess) return hfg::fail_external(HFG_OOM_BUDGET, std::string("hfg_mp2_rhf: ") + cudaGetErrorString(e));
  hfg_status st = transform(ctx, dC, 0, nocc, nocc, nv, dX, nullptr, buf);
  if (st != HFG_OK) return st;
  const long long ov = (long long)nocc * nv;
  mp2_energy<<<grid_for(ov * ov), 256>>>(dX, dE, nocc, nv, dOut);
  e = cudaMemcpy(e_mp2, dOut, sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return hfg::fail_external(HFG_DEVICE_ERROR, std::string("hfg_mp2_rhf: ") + cudaGetErrorString(e));
  return HFG_OK;
}

// UnrestrictedHartreeFock::CalculateMp2Energy (UnrestrictedHartreeFock.cpp:295-375):
// 0.25 (S+ + S-), S = sum over occupied i, j and virtual a, b of one spin of
// (ia|jb)^2 / (e_i + e_j - e_a - e_b).  The reference evaluates both sums
// through one MolecularOrbitalsIntegralsRepository whose four caches are
// keyed by orbital indices only (IntegralsRepository.h:190-291), so the
// second sum reuses values the first one cached with the other spin's
// coefficients.  The first sum leaves, with n+ occupied+ orbitals,
//   level 1 (m n | l b~)     for b virtual+            (b transformed)
//   level 2 (m n | j~ b~)    for j occupied+, b virtual+
//   level 3 (m a~ | j~ b~)   for a virtual+ too
//   level 4 (i~ a~ | j~ b~)  for i occupied+ too
// (~ = with C+).  In the second sum each quartet takes the deepest cached
// level, so index b is transformed with C+ when b is virtual+, j with C+
// when also j is occupied+, a when also a is virtual+, i when also i is
// occupied+, and every other index with C-; the orbital energies are the
// second spin's throughout.  The blocks below partition the second sum's
// (i, a, j, b) ranges by that rule, for n+ >= n- (the reference's default
// occupation of Molecule::Init gives n+ = n- or n- = n+ + 1 -- the beta
// spin holds the odd electron) and for n+ < n- alike.
namespace {

struct Mp2Block {
  Range i, a, j, b;
};

}  // namespace

extern "C" hfg_status hfg_mp2_uhf(hfg_ctx *ctx, const double *Cp, const double *ep, int32_t np, const double *Cm,
                                  const double *em, int32_t nm, double *e_mp2) {
  const char *who = "hfg_mp2_uhf";
  if (!ctx || !Cp || !ep || !Cm || !em || !e_mp2) return hfg::fail_external(HFG_INVALID_ARG, "hfg_mp2_uhf: arguments");
  const int n = hfg_ctx_nbf(ctx);
  if (n <= 0 || np < 0 || nm < 0 || np > n || nm > n)
    return hfg::fail_external(HFG_INVALID_ARG, "hfg_mp2_uhf: occupied counts (need 0 <= n+, n- <= nbf)");
  const int vp = n - np, vm = n - nm, lo = std::min(np, nm), hi = std::max(np, nm);
  Buffers buf;
  double *dCp = nullptr, *dCm = nullptr, *dEp = nullptr, *dEm = nullptr, *dX = nullptr, *dOut = nullptr;
  const long long ovmax = std::max<long long>(1, std::max<long long>((long long)np * vp, (long long)nm * vm));
  cudaError_t e = buf.get(&dCp, (size_t)n * n);
  if (e == cudaSuccess) e = buf.get(&dCm, (size_t)n * n);
  if (e == cudaSuccess) e = buf.get(&dEp, (size_t)n);
  if (e == cudaSuccess) e = buf.get(&dEm, (size_t)n);
  if (e == cudaSuccess) e = buf.get(&dX, (size_t)(ovmax * ovmax));
  if (e == cudaSuccess) e = buf.get(&dOut, 1);
  if (e == cudaSuccess) e = cudaMemcpy(dCp, Cp, sizeof(double) * n * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dCm, Cm, sizeof(double) * n * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dEp, ep, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dEm, em, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);  // staged copies landed
  if (e == cudaSuccess) e = cudaMemset(dOut, 0, sizeof(double));
  if (e != cudaSuccess) return hfg::fail_external(HFG_OOM_BUDGET, std::string(who) + ": " + cudaGetErrorString(e));
  cudaStream_t s = nullptr;
  MoTables t;
  hfg_status st = prepare(ctx, ovmax, s, buf, t, who);
  if (st != HFG_OK) return st;
  // first sum: all C+, i, j < n+, a, b >= n+
  std::vector<std::pair<Mp2Block, const double *>> blocks;
  blocks.push_back({{{dCp, 0, np}, {dCp, np, vp}, {dCp, 0, np}, {dCp, np, vp}}, dEp});
  // second sum, i, j < n-, a, b >= n-, partitioned by the cache rule above
  const Range iAll{dCm, 0, nm}, aAll{dCm, nm, vm};
  // b virtual+ (b >= max): j occupied+ (j < min) ...
  //   ... a virtual+: i occupied+ from C+, i in [n+, n-) from C-
  blocks.push_back({{{dCp, 0, lo}, {dCp, hi, n - hi}, {dCp, 0, lo}, {dCp, hi, n - hi}}, dEm});
  if (nm > np) blocks.push_back({{{dCm, np, nm - np}, {dCp, hi, n - hi}, {dCp, 0, lo}, {dCp, hi, n - hi}}, dEm});
  //   ... a in [n-, n+) occupied+ only: a and i from C-
  if (np > nm) blocks.push_back({{iAll, {dCm, nm, np - nm}, {dCp, 0, lo}, {dCp, hi, n - hi}}, dEm});
  // b virtual+, j in [n+, n-): j, a and i from C-
  if (nm > np) blocks.push_back({{iAll, aAll, {dCm, np, nm - np}, {dCp, hi, n - hi}}, dEm});
  // b in [n-, n+) occupied+ only: all C-
  if (np > nm) blocks.push_back({{iAll, aAll, {dCm, 0, nm}, {dCm, nm, np - nm}}, dEm});
  for (const auto &[q, eps] : blocks) {
    if (q.i.count <= 0 || q.a.count <= 0 || q.j.count <= 0 || q.b.count <= 0) continue;
    if ((st = block(t, q.i, q.a, q.j, q.b, dX, s, who)) != HFG_OK) return st;
    const long long rows = (long long)q.i.count * q.a.count, cols = (long long)q.j.count * q.b.count;
    // orbital energies of the sum's spin at the block's absolute orbital indices
    mp2_sum_sq<<<grid_for(rows * cols), 256, 0, s>>>(dX, cols, q.i.count, q.a.count, q.j.count, q.b.count,
                                                      eps + q.i.first, eps + q.a.first, eps + q.j.first,
                                                      eps + q.b.first, dOut);
  }
  if ((st = finish(s, who)) != HFG_OK) return st;
  double sum = 0;
  e = cudaMemcpy(&sum, dOut, sizeof(double), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return hfg::fail_external(HFG_DEVICE_ERROR, std::string(who) + ": " + cudaGetErrorString(e));
  *e_mp2 = 0.25 * sum;
  return HFG_OK;
}

namespace {

// T[p][q][r][s] over 2n spin orbitals (spatial orbital p / 2, spin p % 2) from
// X[(hp hq),(hr hs)] = (hp hq | hr hs):
// T = (hp hr | hq hs) [p, r and q, s same spin] - (hp hs | hq hr) [p, s and q, r same spin]
__global__ void spin_orbital_tensor(const double *__restrict__ X, int n, double *__restrict__ T) {
  const long long m = 2LL * n, total = m * m * m * m, nn = (long long)n * n;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(x % m), r = (int)((x / m) % m), q = (int)((x / (m * m)) % m), p = (int)(x / (m * m * m));
    const int hp = p >> 1, hq = q >> 1, hr = r >> 1, hs = s >> 1;
    double v = 0.0;
    if ((p & 1) == (r & 1) && (q & 1) == (s & 1)) v += X[((long long)hp * n + hr) * nn + (long long)hq * n + hs];
    if ((p & 1) == (s & 1) && (q & 1) == (r & 1)) v -= X[((long long)hp * n + hs) * nn + (long long)hq * n + hr];
    T[x] = v;
  }
}

}  // namespace

// The whole MO integral tensor (pq|rs), X[(p q),(r s)], p..s over every
// orbital of dC (device, row-major nbf x nbf).
extern "C" hfg_status hfg_mo_eri_full(hfg_ctx *ctx, const double *dC, double *dX, void *stream) {
  const char *who = "hfg_mo_eri_full";
  if (!ctx || !dC || !dX) return hfg::fail_external(HFG_INVALID_ARG, "hfg_mo_eri_full: arguments");
  const int n = hfg_ctx_nbf(ctx);
  if (n <= 0) return hfg::fail_external(HFG_INVALID_ARG, "hfg_mo_eri_full: context without a single molecule");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Buffers buf;
  MoTables t;
  hfg_status st = prepare(ctx, (long long)n * n, s, buf, t, who);
  if (st != HFG_OK) return st;
  if ((st = block(t, {dC, 0, n}, {dC, 0, n}, {dC, 0, n}, {dC, 0, n}, dX, s, who)) != HFG_OK) return st;
  return finish(s, who);
}

// SpinOrbitalsElectronElectronIntegralsRepository::Compute
// (SpinOrbitalsElectronElectronIntegralsRepository.cpp:30-52) for host C
// (row-major nbf x nbf): out receives the (2 nbf)^4 tensor, row-major
// [p][q][r][s].
extern "C" hfg_status hfg_spin_orbital_eri(hfg_ctx *ctx, const double *C, double *out, int64_t count) {
  const char *who = "hfg_spin_orbital_eri";
  if (!ctx || !C || !out) return hfg::fail_external(HFG_INVALID_ARG, "hfg_spin_orbital_eri: arguments");
  const int n = hfg_ctx_nbf(ctx);
  if (n <= 0) return hfg::fail_external(HFG_INVALID_ARG, "hfg_spin_orbital_eri: context without a single molecule");
  const long long m = 2LL * n, total = m * m * m * m, nn = (long long)n * n;
  if (count < total) return hfg::fail_external(HFG_INVALID_ARG, "hfg_spin_orbital_eri: output holds fewer than (2 nbf)^4");
  Buffers buf;
  double *dC = nullptr, *dX = nullptr, *dT = nullptr;
  cudaError_t e = buf.get(&dC, (size_t)nn);
  if (e == cudaSuccess) e = buf.get(&dX, (size_t)(nn * nn));
  if (e == cudaSuccess) e = buf.get(&dT, (size_t)total);
  if (e == cudaSuccess) e = cudaMemcpy(dC, C, sizeof(double) * nn, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
  if (e != cudaSuccess) return hfg::fail_external(HFG_OOM_BUDGET, std::string(who) + ": " + cudaGetErrorString(e));
  hfg_status st = hfg_mo_eri_full(ctx, dC, dX, nullptr);
  if (st != HFG_OK) return st;
  spin_orbital_tensor<<<grid_for(total), 256>>>(dX, n, dT);
  e = cudaMemcpy(out, dT, sizeof(double) * total, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return hfg::fail_external(HFG_DEVICE_ERROR, std::string(who) + ": " + cudaGetErrorString(e));
  return HFG_OK;
}
