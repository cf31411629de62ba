// Device-resident SCF iteration for the host API (include/hfgpu_host.hpp):
// the steps of RestrictedHartreeFock::Step (RestrictedHartreeFock.cpp:61-166)
// and UnrestrictedHartreeFock::Step (UnrestrictedHartreeFock.cpp:87-191)
// with every matrix in HBM.  F = h + G comes straight from the engine's
// direct build on the same stream, DIIS (DIIS.h:34-96) keeps its Fock and
// error matrices on the device (Pulay B matrix from one Gram product, the
// small (m+1)x(m+1) solve on the host), the orthogonalised Fock matrix is
// diagonalised by cuSOLVER (dsyevd) and the density is one product of the
// occupied coefficients.  Per step only scalars (energy terms, norms, the
// B matrix, eigenvalues) cross to the host.  All arithmetic is FP64.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/hfgpu.h"
#include "scf_device.h"

namespace hfgpu {
namespace detail {

namespace {

void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}
void ck(cublasStatus_t e, const char *what) {
  if (e != CUBLAS_STATUS_SUCCESS) throw std::runtime_error(std::string(what) + ": cuBLAS status " + std::to_string((int)e));
}
void ck(cusolverStatus_t e, const char *what) {
  if (e != CUSOLVER_STATUS_SUCCESS)
    throw std::runtime_error(std::string(what) + ": cuSOLVER status " + std::to_string((int)e));
}

// F = h + G (G may be null: F = h), then F = (F + F^T)/2 when `sym`
__global__ void fock_from_g(const double *h, const double *G, double *F, int n, int sym) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n * n; x += gridDim.x * blockDim.x) {
    const int i = x / n, j = x - i * n;
    const double a = h[x] + (G ? G[x] : 0.0);
    if (sym) {
      const double b = h[j * n + i] + (G ? G[j * n + i] : 0.0);
      F[x] = 0.5 * (a + b);
    } else {
      F[x] = a;
    }
  }
}

// C_w = C with the columns of unoccupied levels zeroed (occ[k] = 0/1)
__global__ void mask_columns(const double *C, const int *occ, double *Cw, int n) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n * n; x += gridDim.x * blockDim.x) {
    const int k = x % n;
    Cw[x] = occ[k] ? C[x] : 0.0;
  }
}

int grid_of(size_t nn) { return (int)std::max<size_t>(1, std::min<size_t>(2048, (nn + 255) / 256)); }

}  // namespace

DeviceScf::DeviceScf(int n, int device) : n_(n), device_(device) {
  ck(cudaSetDevice(device), "cudaSetDevice");
  ck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cublasCreate(&blas_), "cublasCreate");
  ck(cublasSetStream(blas_, stream_), "cublasSetStream");
  ck(cusolverDnCreate(&solver_), "cusolverDnCreate");
  ck(cusolverDnSetStream(solver_, stream_), "cusolverDnSetStream");
  const size_t nn = (size_t)n * n;
  for (double **p : {&h_, &S_, &V_, &T1_, &T2_, &Ft_, &W_, &err_})
    ck(cudaMalloc((void **)p, nn * sizeof(double)), "cudaMalloc");
  for (int s = 0; s < 2; ++s)
    for (double **p : {&P_[s], &Pn_[s], &F_[s], &G_[s], &C_[s]}) ck(cudaMalloc((void **)p, nn * sizeof(double)), "cudaMalloc");
  ck(cudaMalloc((void **)&w_, 2 * (size_t)n * sizeof(double)), "cudaMalloc");
  ck(cudaMalloc((void **)&info_, sizeof(int)), "cudaMalloc");
  ck(cudaMalloc((void **)&occ_dev_, (size_t)n * sizeof(int)), "cudaMalloc");
  ck(cudaMalloc((void **)&scalars_, 64 * sizeof(double)), "cudaMalloc");
  ck(cudaMalloc((void **)&coef_, 16 * sizeof(double)), "cudaMalloc");
  ck(cudaMallocHost((void **)&host_scalars_, 64 * sizeof(double)), "cudaMallocHost");
  ck(cudaMallocHost((void **)&host_info_, sizeof(int)), "cudaMallocHost");
  ck(cudaMallocHost((void **)&host_w_, 2 * (size_t)n * sizeof(double)), "cudaMallocHost");
  ck(cusolverDnDsyevd_bufferSize(solver_, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, Ft_, n, w_, &lwork_),
     "dsyevd_bufferSize");
  ck(cudaMalloc((void **)&work_, (size_t)std::max(lwork_, 1) * sizeof(double)), "cudaMalloc");
  for (int s = 0; s < 2; ++s) {
    ck(cudaMalloc((void **)&diis_F_[s], kDiisKeep * nn * sizeof(double)), "cudaMalloc");
    ck(cudaMalloc((void **)&diis_E_[s], kDiisKeep * nn * sizeof(double)), "cudaMalloc");
  }
  for (auto &e : ev_) ck(cudaEventCreate(&e), "cudaEventCreate");
}

DeviceScf::~DeviceScf() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  for (double *p : {h_, S_, V_, T1_, T2_, Ft_, W_, err_, w_, scalars_, coef_, work_}) cudaFree(p);
  for (int s = 0; s < 2; ++s) {
    for (double *p : {P_[s], Pn_[s], F_[s], G_[s], C_[s], diis_F_[s], diis_E_[s]}) cudaFree(p);
  }
  cudaFree(info_);
  cudaFree(occ_dev_);
  cudaFreeHost(host_scalars_);
  cudaFreeHost(host_w_);
  cudaFreeHost(host_info_);
  for (auto &e : ev_)
    if (e) cudaEventDestroy(e);
  if (solver_) cusolverDnDestroy(solver_);
  if (blas_) cublasDestroy(blas_);
  if (stream_) cudaStreamDestroy(stream_);
}

void DeviceScf::upload(double *dst, const double *src) {
  ck(cudaMemcpyAsync(dst, src, (size_t)n_ * n_ * sizeof(double), cudaMemcpyHostToDevice, stream_), "upload");
}
void DeviceScf::download(double *dst, const double *src) {
  ck(cudaMemcpyAsync(dst, src, (size_t)n_ * n_ * sizeof(double), cudaMemcpyDeviceToHost, stream_), "download");
}

void DeviceScf::SetMatrices(const double *h, const double *S, const double *V) {
  upload(h_, h);
  upload(S_, S);
  upload(V_, V);
  ck(cudaStreamSynchronize(stream_), "SetMatrices");
}

void DeviceScf::SetDensity(int spin, const double *P) {
  upload(P_[spin], P);
  ck(cudaStreamSynchronize(stream_), "SetDensity");
}

void DeviceScf::ResetDiis() { diis_count_[0] = diis_count_[1] = diis_head_[0] = diis_head_[1] = 0; }

// row-major C(MxN) = alpha op(A) op(B) + beta C: the column-major product
// C^T = op(B)^T op(A)^T, so the operands swap and keep their op flags
void DeviceScf::gemm(bool ta, bool tb, int M, int N, int K, double alpha, const double *A, int lda, const double *B,
                     int ldb, double beta, double *C, int ldc) {
  ck(cublasDgemm(blas_, tb ? CUBLAS_OP_T : CUBLAS_OP_N, ta ? CUBLAS_OP_T : CUBLAS_OP_N, N, M, K, &alpha, B, ldb, A,
                 lda, &beta, C, ldc),
     "cublasDgemm");
}

void DeviceScf::FockFromG(int spin, const double *G, bool symmetrize) {
  fock_from_g<<<grid_of((size_t)n_ * n_), 256, 0, stream_>>>(h_, G, F_[spin], n_, symmetrize ? 1 : 0);
  ck(cudaGetLastError(), "fock_from_g");
}

void DeviceScf::SetFock(int spin, const double *F) { upload(F_[spin], F); }

// DIIS.h:9-96 on the device: ring of the last kDiisKeep (F, error) pairs;
// error = S P F - F P S = Z - Z^T with Z = S P F (S, P, F symmetric).
// Returns true once kDiisFirst pairs are held and extrapolates F in place;
// *err_est = sqrt of the two newest errors' squared norms.
bool DeviceScf::DiisStep(int spin, double *err_est) {
  const int n = n_;
  const size_t nn = (size_t)n * n;
  gemm(false, false, n, n, n, 1.0, S_, n, P_[spin], n, 0.0, T1_, n);
  gemm(false, false, n, n, n, 1.0, T1_, n, F_[spin], n, 0.0, T2_, n);
  const int slot = diis_head_[spin];
  double *E = diis_E_[spin] + (size_t)slot * nn;
  const double one = 1.0, mone = -1.0;
  ck(cublasDgeam(blas_, CUBLAS_OP_N, CUBLAS_OP_T, n, n, &one, T2_, n, &mone, T2_, n, E, n), "cublasDgeam");
  ck(cudaMemcpyAsync(diis_F_[spin] + (size_t)slot * nn, F_[spin], nn * sizeof(double), cudaMemcpyDeviceToDevice,
                     stream_),
     "diis copy");
  diis_head_[spin] = (slot + 1) % kDiisKeep;
  diis_count_[spin] = std::min(diis_count_[spin] + 1, kDiisKeep);
  const int m = diis_count_[spin];
  if (m < kDiisFirst) {
    *err_est = 0;
    return false;
  }
  // Gram matrix of the error ring (slot order): row-major m x m = E E^T
  gemm(false, true, m, m, (int)nn, 1.0, diis_E_[spin], (int)nn, diis_E_[spin], (int)nn, 0.0, scalars_, m);
  ck(cudaMemcpyAsync(host_scalars_, scalars_, (size_t)m * m * sizeof(double), cudaMemcpyDeviceToHost, stream_),
     "gram");
  ck(cudaStreamSynchronize(stream_), "gram sync");
  // logical order oldest .. newest, as the reference's list
  std::vector<int> order(m);
  const int oldest = (diis_head_[spin] - m + kDiisKeep) % kDiisKeep;
  for (int i = 0; i < m; ++i) order[i] = (oldest + i) % kDiisKeep;
  const int np1 = m + 1;
  std::vector<double> B((size_t)np1 * np1, 0.0), rhs(np1, 0.0);
  double last = 0;
  for (int i = 0; i < m; ++i) {
    for (int j = 0; j < m; ++j) B[(size_t)i * np1 + j] = host_scalars_[order[i] * m + order[j]];
    if (i == m - 1 || i == m - 2) last += B[(size_t)i * np1 + i];
    B[(size_t)m * np1 + i] = B[(size_t)i * np1 + m] = 1;
  }
  *err_est = std::sqrt(last);
  rhs[m] = 1;
  const std::vector<double> c = pulay_solve(B, np1, rhs);
  double cs[kDiisKeep] = {0};
  for (int i = 0; i < m; ++i) cs[order[i]] = c[i];
  ck(cudaMemcpyAsync(coef_, cs, sizeof cs, cudaMemcpyHostToDevice, stream_), "coef");
  // F = sum_slot c_slot F_slot: (1 x m) (m x nn) row-major
  gemm(false, false, 1, (int)nn, m, 1.0, coef_, m, diis_F_[spin], (int)nn, 0.0, F_[spin], (int)nn);
  ck(cudaStreamSynchronize(stream_), "diis sync");  // cs lives on this frame
  return true;
}

// Ft = V F V, eigen-decomposition, C = V Cp, Pn = factor * C_occ C_occ^T.
void DeviceScf::Diagonalize(int spin, const std::vector<bool> &occupied, double factor, double *eigenvalues) {
  const int n = n_;
  gemm(false, false, n, n, n, 1.0, V_, n, F_[spin], n, 0.0, T1_, n);
  gemm(false, false, n, n, n, 1.0, T1_, n, V_, n, 0.0, Ft_, n);
  ck(cudaEventRecord(ev_[2], stream_), "event");
  // symmetric input: row-major == column-major; on return column k of the
  // column-major array is eigenvector k, i.e. row k of the row-major view
  ck(cusolverDnDsyevd(solver_, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, Ft_, n, w_ + spin * n, work_,
                      lwork_, info_),
     "dsyevd");
  ck(cudaEventRecord(ev_[3], stream_), "event");
  // C = V Cp = V X^T with X the row-major eigenvector rows
  gemm(false, true, n, n, n, 1.0, V_, n, Ft_, n, 0.0, C_[spin], n);
  int nocc = 0;
  bool prefix = true;
  for (size_t k = 0; k < occupied.size(); ++k) {
    if (occupied[k]) {
      if ((int)k != nocc) prefix = false;
      ++nocc;
    }
  }
  if (prefix) {
    if (nocc > 0)
      gemm(false, true, n, n, nocc, factor, C_[spin], n, C_[spin], n, 0.0, Pn_[spin], n);
    else
      ck(cudaMemsetAsync(Pn_[spin], 0, (size_t)n * n * sizeof(double), stream_), "memset");
  } else {
    std::vector<int> occ(n, 0);
    for (size_t k = 0; k < occupied.size() && (int)k < n; ++k) occ[k] = occupied[k] ? 1 : 0;
    ck(cudaMemcpyAsync(occ_dev_, occ.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, stream_), "occ");
    mask_columns<<<grid_of((size_t)n * n), 256, 0, stream_>>>(C_[spin], occ_dev_, W_, n);
    gemm(false, true, n, n, n, factor, W_, n, W_, n, 0.0, Pn_[spin], n);
    ck(cudaStreamSynchronize(stream_), "occ sync");
  }
  ck(cudaMemcpyAsync(host_w_ + spin * n, w_ + spin * n, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, stream_),
     "w");
  ck(cudaMemcpyAsync(host_info_, info_, sizeof(int), cudaMemcpyDeviceToHost, stream_), "info");
  ck(cudaStreamSynchronize(stream_), "diag sync");
  const int info = *host_info_;
  if (info != 0) throw std::runtime_error("dsyevd did not converge (info " + std::to_string(info) + ")");
  float ms = 0;
  if (cudaEventElapsedTime(&ms, ev_[2], ev_[3]) == cudaSuccess) eigen_seconds_ += ms * 1e-3;
  std::copy(host_w_ + spin * n, host_w_ + (spin + 1) * n, eigenvalues);
}

// sum_ij Pn_ij h_ij (symmetric h), and ||Pn - P||_F^2
void DeviceScf::EnergyAndChange(int spin, double *trace_ph, double *change2) {
  const int n = n_;
  const int nn = n * n;
  ck(cublasSetPointerMode(blas_, CUBLAS_POINTER_MODE_DEVICE), "pointer mode");
  ck(cublasDdot(blas_, nn, Pn_[spin], 1, h_, 1, scalars_), "ddot");
  const double one = 1.0, mone = -1.0;
  ck(cublasSetPointerMode(blas_, CUBLAS_POINTER_MODE_HOST), "pointer mode");
  ck(cublasDgeam(blas_, CUBLAS_OP_N, CUBLAS_OP_N, n, n, &one, Pn_[spin], n, &mone, P_[spin], n, W_, n), "geam");
  ck(cublasSetPointerMode(blas_, CUBLAS_POINTER_MODE_DEVICE), "pointer mode");
  ck(cublasDdot(blas_, nn, W_, 1, W_, 1, scalars_ + 1), "ddot");
  ck(cublasSetPointerMode(blas_, CUBLAS_POINTER_MODE_HOST), "pointer mode");
  ck(cudaMemcpyAsync(host_scalars_, scalars_, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream_), "scalars");
  ck(cudaStreamSynchronize(stream_), "scalars sync");
  *trace_ph = host_scalars_[0];
  *change2 = host_scalars_[1];
}

// P = Pn (DIIS step) or alpha Pn + (1 - alpha) P (mixing)
void DeviceScf::UpdateDensity(int spin, bool take_new, double alpha) {
  const int n = n_;
  const double a = take_new ? 1.0 : alpha, b = take_new ? 0.0 : 1.0 - alpha;
  ck(cublasDgeam(blas_, CUBLAS_OP_N, CUBLAS_OP_N, n, n, &a, Pn_[spin], n, &b, P_[spin], n, P_[spin], n), "geam");
}

void DeviceScf::Sync() { ck(cudaStreamSynchronize(stream_), "sync"); }

void DeviceScf::CopyOut(int spin, double *P, double *C) {
  if (P) download(P, P_[spin]);
  if (C) download(C, C_[spin]);
  Sync();
}

}  // namespace detail
}  // namespace hfgpu

// ---------------------------------------------------------------------------
// hfg_eigh_batched (include/hfgpu.h): eigen-decomposition of a stack of small
// symmetric matrices in one cuSOLVER batched Jacobi call, for the batched
// SCF's F' = V F V step.  Handle and workspace are kept per host thread and
// grown on demand.
namespace {
struct BatchedEigh {
  cusolverDnHandle_t handle = nullptr;
  cusolverDnParams_t params = nullptr;
  int device = -1;
  void *dwork = nullptr;
  size_t dbytes = 0;
  std::vector<char> hwork;
  int *info = nullptr;
  int64_t info_cap = 0;
  void release() {
    if (dwork) cudaFree(dwork);
    if (info) cudaFree(info);
    if (params) cusolverDnDestroyParams(params);
    if (handle) cusolverDnDestroy(handle);
    dwork = nullptr;
    info = nullptr;
    params = nullptr;
    handle = nullptr;
    dbytes = 0;
    info_cap = 0;
    device = -1;
  }
  ~BatchedEigh() { release(); }
};
thread_local BatchedEigh g_eigh;
}  // namespace

namespace hfg {
hfg_status fail_external(hfg_status st, const std::string &msg);
}

extern "C" hfg_status hfg_eigh_batched(const double *dA, double *dV, double *dW, int32_t n, int32_t batch,
                                       int32_t method, void *stream) {
  using hfgpu::detail::ck;
  if (!dA || !dV || !dW || n < 1 || batch < 1 || method < 0 || method > 1)
    return hfg::fail_external(HFG_INVALID_ARG, "hfg_eigh_batched: arguments");
  try {
    BatchedEigh &e = g_eigh;
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    if (e.handle && e.device != dev) {
      cusolverDnDestroyParams(e.params);
      cusolverDnDestroy(e.handle);
      if (e.dwork) cudaFree(e.dwork);
      if (e.info) cudaFree(e.info);
      e.handle = nullptr;
      e.params = nullptr;
      e.dwork = nullptr;
      e.info = nullptr;
      e.dbytes = 0;
      e.info_cap = 0;
    }
    if (!e.handle) {
      ck(cusolverDnCreate(&e.handle), "cusolverDnCreate");
      ck(cusolverDnCreateParams(&e.params), "cusolverDnCreateParams");
      e.device = dev;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ck(cusolverDnSetStream(e.handle, s), "cusolverDnSetStream");
    const size_t bytes = (size_t)n * n * batch * sizeof(double);
    if (dV != dA) ck(cudaMemcpyAsync(dV, dA, bytes, cudaMemcpyDeviceToDevice, s), "copy A");
    if (method == 1) {
      // one divide-and-conquer solve per matrix, the single-molecule SCF's solver
      int lwork = 0;
      ck(cusolverDnDsyevd_bufferSize(e.handle, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, dV, n, dW, &lwork),
         "cusolverDnDsyevd_bufferSize");
      const size_t need = (size_t)lwork * sizeof(double);
      if (need > e.dbytes) {
        ck(cudaStreamSynchronize(s), "sync");
        if (e.dwork) cudaFree(e.dwork);
        e.dwork = nullptr;
        ck(cudaMalloc(&e.dwork, need), "cudaMalloc eigh workspace");
        e.dbytes = need;
      }
      if (batch > e.info_cap) {
        ck(cudaStreamSynchronize(s), "sync");
        if (e.info) cudaFree(e.info);
        e.info = nullptr;
        ck(cudaMalloc(&e.info, sizeof(int) * batch), "cudaMalloc eigh info");
        e.info_cap = batch;
      }
      const size_t nn = (size_t)n * n;
      for (int b = 0; b < batch; ++b)
        ck(cusolverDnDsyevd(e.handle, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, dV + b * nn, n,
                            dW + (size_t)b * n, static_cast<double *>(e.dwork), lwork, e.info + b),
           "cusolverDnDsyevd");
      return HFG_OK;
    }
    size_t dneed = 0, hneed = 0;
    ck(cusolverDnXsyevBatched_bufferSize(e.handle, e.params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n,
                                         CUDA_R_64F, dV, n, CUDA_R_64F, dW, CUDA_R_64F, &dneed, &hneed, batch),
       "cusolverDnXsyevBatched_bufferSize");
    if (dneed > e.dbytes) {
      ck(cudaStreamSynchronize(s), "sync");
      if (e.dwork) cudaFree(e.dwork);
      e.dwork = nullptr;
      ck(cudaMalloc(&e.dwork, dneed), "cudaMalloc eigh workspace");
      e.dbytes = dneed;
    }
    if (hneed > e.hwork.size()) e.hwork.resize(hneed);
    if (batch > e.info_cap) {
      ck(cudaStreamSynchronize(s), "sync");
      if (e.info) cudaFree(e.info);
      e.info = nullptr;
      ck(cudaMalloc(&e.info, sizeof(int) * batch), "cudaMalloc eigh info");
      e.info_cap = batch;
    }
    ck(cusolverDnXsyevBatched(e.handle, e.params, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, CUDA_R_64F, dV,
                              n, CUDA_R_64F, dW, CUDA_R_64F, e.dwork, e.dbytes,
                              e.hwork.empty() ? nullptr : e.hwork.data(), hneed, e.info, batch),
       "cusolverDnXsyevBatched");
    return HFG_OK;
  } catch (const std::exception &ex) {
    return hfg::fail_external(HFG_DEVICE_ERROR, ex.what());
  }
}

// ---------------------------------------------------------------------------
// hfg_pulay_solve_device (include/hfgpu.h): the DIIS system B c = (0 .. 0 1)
// of every molecule of a batch, on the device, by the same column-pivoted
// Householder QR with rank cut-off as the host SCF's solve
// (hfgpu::detail::pulay_solve, the role of Eigen's colPivHouseholderQr at
// DIIS.h:72).  One thread per system; systems up to kPulayMax unknowns.
namespace {
constexpr int kPulayMax = 8;
__global__ void pulay_kernel(const double *__restrict__ B, int n, int batch, double *__restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= batch) return;
  double A[kPulayMax * kPulayMax], b[kPulayMax], v[kPulayMax], z[kPulayMax];
  int perm[kPulayMax];
  for (int i = 0; i < n * n; ++i) A[i] = B[(size_t)t * n * n + i];
  for (int i = 0; i < n; ++i) {
    b[i] = i == n - 1 ? 1.0 : 0.0;
    perm[i] = i;
  }
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = -1;
    for (int j = k; j < n; ++j) {
      double s = 0;
      for (int i = k; i < n; ++i) s += A[i * n + j] * A[i * n + j];
      if (s > best) {
        best = s;
        p = j;
      }
    }
    if (p != k) {
      for (int i = 0; i < n; ++i) {
        const double x = A[i * n + k];
        A[i * n + k] = A[i * n + p];
        A[i * n + p] = x;
      }
      const int q = perm[k];
      perm[k] = perm[p];
      perm[p] = q;
    }
    double al = 0;
    for (int i = k; i < n; ++i) al += A[i * n + k] * A[i * n + k];
    al = sqrt(al);
    if (al == 0) continue;
    if (A[k * n + k] > 0) al = -al;
    v[0] = A[k * n + k] - al;
    for (int i = k + 1; i < n; ++i) v[i - k] = A[i * n + k];
    double vn = 0;
    for (int i = 0; i < n - k; ++i) vn += v[i] * v[i];
    const double beta = vn > 0 ? 2.0 / vn : 0.0;
    for (int j = k; j < n; ++j) {
      double s = 0;
      for (int i = k; i < n; ++i) s += v[i - k] * A[i * n + j];
      s *= beta;
      for (int i = k; i < n; ++i) A[i * n + j] -= s * v[i - k];
    }
    double s = 0;
    for (int i = k; i < n; ++i) s += v[i - k] * b[i];
    s *= beta;
    for (int i = k; i < n; ++i) b[i] -= s * v[i - k];
  }
  const double tol = fabs(A[0]) * 1e-15 * n;
  int rank = 0;
  while (rank < n && fabs(A[rank * n + rank]) > tol) ++rank;
  for (int i = 0; i < n; ++i) z[i] = 0.0;
  for (int i = rank - 1; i >= 0; --i) {
    double s = b[i];
    for (int j = i + 1; j < rank; ++j) s -= A[i * n + j] * z[j];
    z[i] = s / A[i * n + i];
  }
  for (int j = 0; j < n; ++j) out[(size_t)t * n + perm[j]] = z[j];
}
}  // namespace

extern "C" hfg_status hfg_pulay_solve_device(const double *dB, int32_t m1, int32_t batch, double *dC, void *stream) {
  if (!dB || !dC || m1 < 2 || m1 > kPulayMax || batch < 0)
    return hfg::fail_external(HFG_INVALID_ARG, "hfg_pulay_solve_device: arguments (2 <= m1 <= 8)");
  if (batch == 0) return HFG_OK;
  pulay_kernel<<<(batch + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(dB, m1, batch, dC);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return hfg::fail_external(HFG_DEVICE_ERROR, cudaGetErrorString(e));
  return HFG_OK;
}

extern "C" void hfg_release_thread(void) { g_eigh.release(); }
