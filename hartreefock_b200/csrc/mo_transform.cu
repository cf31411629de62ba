// AO -> MO transform of the two-electron integrals and the RHF MP2 energy,
// for the post-HF consumers of the integral tables:
// MolecularOrbitalsIntegralsRepository::getElectronElectron
// (IntegralsRepository.h:190-291) and RestrictedHartreeFock::CalculateMp2Energy
// (RestrictedHartreeFock.cpp:251-288).
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

// K[(l s),(j b)] = C[l][i0+j] C[s][a0+b], C row-major n x n (AO rows, MO columns)
__global__ void pair_coefficients(const double *__restrict__ C, int n, int i0, int ni, int a0, int na,
                                  double *__restrict__ K) {
  const long long ov = (long long)ni * na, total = (long long)n * n * ov;
  for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < total; x += (long long)gridDim.x * blockDim.x) {
    const long long r = x / ov, c = x - r * ov;
    const int l = (int)(r / n), s = (int)(r - (long long)l * n), j = (int)(c / na), b = (int)(c - (long long)j * na);
    K[x] = C[(long long)l * n + i0 + j] * C[(long long)s * n + a0 + b];
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

hfg_status transform(hfg_ctx *ctx, const double *dC, int i0, int ni, int a0, int na, double *dX, cudaStream_t s,
                     Buffers &buf) {
  const int n = hfg_ctx_nbf(ctx);
  if (n <= 0) return hfg::fail_external(HFG_INVALID_ARG, "hfg_mo_eri_ovov: context without a single molecule");
  if (!dC || !dX || ni < 1 || na < 1 || i0 < 0 || a0 < 0 || i0 + ni > n || a0 + na > n)
    return hfg::fail_external(HFG_INVALID_ARG, "hfg_mo_eri_ovov: orbital ranges");
  const long long nn = (long long)n * n, ov = (long long)ni * na;
  const int64_t count = hfg_packed_size(n);
  size_t freeb = 0, totalb = 0;
  cudaMemGetInfo(&freeb, &totalb);
  const double need = 8.0 * ((double)count + (double)nn * nn + 2.0 * nn * ov);
  if (need > 0.9 * (double)freeb)
    return hfg::fail_external(HFG_OOM_BUDGET, "hfg_mo_eri_ovov: the unpacked AO table does not fit (" +
                                                  std::to_string(need / 1e9) + " GB needed)");
  double *packed = nullptr, *M = nullptr, *K = nullptr, *Y = nullptr;
  cudaError_t e = buf.get(&packed, (size_t)count);
  if (e == cudaSuccess) e = buf.get(&M, (size_t)(nn * nn));
  if (e == cudaSuccess) e = buf.get(&K, (size_t)(nn * ov));
  if (e == cudaSuccess) e = buf.get(&Y, (size_t)(nn * ov));
  if (e != cudaSuccess) return hfg::fail_external(HFG_OOM_BUDGET, std::string("hfg_mo_eri_ovov: ") + cudaGetErrorString(e));
  hfg_status st = hfg_eri_packed_device(ctx, packed, count, s);
  if (st != HFG_OK) return st;
  // stream 0 means the context's own stream for the packed build: finish it
  // before the kernels below read the table
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return hfg::fail_external(HFG_DEVICE_ERROR, std::string("hfg_mo_eri_ovov: ") + cudaGetErrorString(e));
  unpack_eri<<<grid_for(nn * nn), 256, 0, s>>>(packed, M, n);
  pair_coefficients<<<grid_for(nn * ov), 256, 0, s>>>(dC, n, i0, ni, a0, na, K);
  Blas b;
  if (cublasCreate(&b.h) != CUBLAS_STATUS_SUCCESS || cublasSetStream(b.h, s) != CUBLAS_STATUS_SUCCESS)
    return hfg::fail_external(HFG_DEVICE_ERROR, "hfg_mo_eri_ovov: cuBLAS handle");
  const double one = 1.0, zero = 0.0;
  // row-major Y = M K  <=>  column-major Y^T = K^T M^T
  if (cublasDgemm(b.h, CUBLAS_OP_N, CUBLAS_OP_N, (int)ov, (int)nn, (int)nn, &one, K, (int)ov, M, (int)nn, &zero, Y,
                  (int)ov) != CUBLAS_STATUS_SUCCESS)
    return hfg::fail_external(HFG_DEVICE_ERROR, "hfg_mo_eri_ovov: DGEMM M K");
  // row-major X = K^T Y  <=>  column-major X^T = Y^T K
  if (cublasDgemm(b.h, CUBLAS_OP_N, CUBLAS_OP_T, (int)ov, (int)ov, (int)nn, &one, Y, (int)ov, K, (int)ov, &zero, dX,
                  (int)ov) != CUBLAS_STATUS_SUCCESS)
    return hfg::fail_external(HFG_DEVICE_ERROR, "hfg_mo_eri_ovov: DGEMM K^T Y");
  e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return hfg::fail_external(HFG_DEVICE_ERROR, std::string("hfg_mo_eri_ovov: ") + cudaGetErrorString(e));
  return HFG_OK;
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
