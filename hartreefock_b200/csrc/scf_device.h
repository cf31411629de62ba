// Device-resident SCF state of one HartreeFockAlgorithm (see scf_device.cu).
// Internal to the library: the public surface stays include/hfgpu_host.hpp.
#pragma once

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <vector>

namespace hfgpu {
namespace detail {

// Least-squares solve of a small dense system by column-pivoted Householder
// QR (the Pulay system of DIIS.h:72); defined in host.cpp.
std::vector<double> pulay_solve(std::vector<double> A, int n, std::vector<double> b);

class DeviceScf {
 public:
  static constexpr int kDiisKeep = 6;   // DIIS.h:9 maxRetained
  static constexpr int kDiisFirst = 5;  // DIIS.h:31 firstEstimate

  DeviceScf(int n, int device);
  ~DeviceScf();
  DeviceScf(const DeviceScf &) = delete;
  DeviceScf &operator=(const DeviceScf &) = delete;

  int n() const { return n_; }
  cudaStream_t stream() const { return stream_; }
  // core Hamiltonian, overlap and S^-1/2 (row-major host n x n)
  void SetMatrices(const double *h, const double *S, const double *V);
  void SetDensity(int spin, const double *P);
  void SetFock(int spin, const double *F);
  void ResetDiis();
  // F = h + G[spin] (G = nullptr: F = h); optionally symmetrised
  void FockFromG(int spin, const double *G, bool symmetrize);
  bool DiisStep(int spin, double *err_est);
  void Diagonalize(int spin, const std::vector<bool> &occupied, double factor, double *eigenvalues);
  void EnergyAndChange(int spin, double *trace_ph, double *change2);
  void UpdateDensity(int spin, bool take_new, double alpha);
  void CopyOut(int spin, double *P, double *C);
  void Sync();

  double *density(int spin) { return P_[spin]; }
  double *g_buffer(int spin) { return G_[spin]; }
  double eigen_seconds() const { return eigen_seconds_; }
  void reset_timers() { eigen_seconds_ = 0; }

 private:
  void upload(double *dst, const double *src);
  void download(double *dst, const double *src);
  void gemm(bool ta, bool tb, int M, int N, int K, double alpha, const double *A, int lda, const double *B, int ldb,
            double beta, double *C, int ldc);

  int n_ = 0, device_ = 0;
  cudaStream_t stream_ = nullptr;
  cublasHandle_t blas_ = nullptr;
  cusolverDnHandle_t solver_ = nullptr;
  double *h_ = nullptr, *S_ = nullptr, *V_ = nullptr;
  double *T1_ = nullptr, *T2_ = nullptr, *Ft_ = nullptr, *W_ = nullptr, *err_ = nullptr;
  double *P_[2] = {}, *Pn_[2] = {}, *F_[2] = {}, *G_[2] = {}, *C_[2] = {};
  double *w_ = nullptr, *work_ = nullptr, *scalars_ = nullptr, *coef_ = nullptr;
  int *info_ = nullptr, *occ_dev_ = nullptr;
  int lwork_ = 0;
  double *host_scalars_ = nullptr, *host_w_ = nullptr;
  int *host_info_ = nullptr;
  double *diis_F_[2] = {}, *diis_E_[2] = {};
  int diis_head_[2] = {0, 0}, diis_count_[2] = {0, 0};
  cudaEvent_t ev_[4] = {};
  double eigen_seconds_ = 0;
};

}  // namespace detail
}  // namespace hfgpu
