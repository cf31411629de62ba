/* hfgpu driver: one-call SCF through the host API (include/hfgpu_host.hpp),
 * for callers that cannot link C++ (ctypes, cgo, JNI).  No reference
 * counterpart as a single function: it runs the reference's own call
 * sequence Basis::Load -> Molecule::Init -> {Restricted,Unrestricted}
 * HartreeFock::Init -> Calculate (README.md:41-70, HartreeFockThread.cpp:79-121). */
#ifndef HFGPU_DRIVER_H
#define HFGPU_DRIVER_H

#include <stdint.h>

#include "hfgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t unrestricted;      /* 0 RHF, 1 UHF */
  double alpha;              /* density mixing (HartreeFockAlgorithm::alpha) */
  double init_guess;         /* HartreeFockAlgorithm::initGuess */
  int32_t use_diis;          /* HartreeFockAlgorithm::UseDIIS */
  int32_t post_diis;         /* HartreeFockAlgorithm::normalIterAfterDIIS */
  int32_t alpha_electrons;   /* 0,0 = from nuclear charges (Molecule.cpp:135-139) */
  int32_t beta_electrons;
  int32_t eri_convention;    /* hfg_eri_convention */
  double schwarz_threshold;
  /* precision form of the Fock builds (HartreeFockAlgorithm::mixedCutoff
   * and friends in hfgpu_host.hpp); all 0 = the plain FP64 form */
  double mixed_cutoff;       /* FP32 below this density-weighted bound */
  double mixed_switch_energy;/* leave the incremental phase below this |dE| ... */
  double mixed_switch_density;/* ... and this rms density change ... */
  double mixed_switch_diis;  /* ... and this DIIS error estimate */
  int32_t fp64_final_iterations;
  int32_t fp64_final_converge;/* 1: the FP64 phase also meets the reference's test */
  int32_t incremental;       /* FP64 incremental builds (implied by mixed_cutoff > 0) */
  int32_t trace;             /* 1: one line per SCF step on stderr */
  int32_t stop_at_precision_test; /* plain builds, precision form's stopping rule */
  int32_t max_iterations;    /* the algorithm's iteration cap; 0 = 3000, the
                                reference's default (RestrictedHartreeFock.h:31) */
  int32_t mp2;               /* 1: RHF MP2 energy after the SCF (result.mp2_energy) */
  int32_t concurrent_classes;/* 1: a build's classes on concurrent streams
                                (HartreeFockAlgorithm::concurrentClasses); 2: also CUDA-graph
                                replay of plain builds (cudaGraphs), for one host thread
                                driving the device; 0: neither */
} hfd_scf_opts;

typedef struct {
  double energy;             /* HartreeFockAlgorithm::GetTotalEnergy */
  double homo;               /* HOMOEnergy */
  int32_t converged;
  int32_t iterations;
  int32_t nbf;
  int32_t fock_builds;       /* two-electron builds (iterations after the first) */
  double fock_ms_total;      /* device time spent in two-electron builds */
  int64_t fp32_quartets;     /* shell quartets evaluated in FP32, all builds */
  int64_t fp64_quartets;     /* shell quartets evaluated in FP64, all builds */
  int32_t mixed_steps;       /* builds of the incremental (first) phase */
  int32_t reserved;
  /* wall-clock split of the SCF (seconds) */
  double seconds_fock, seconds_eigen, seconds_diis, seconds_total;
  double seconds_init;       /* Init: one-electron matrices, engine context, S^-1/2 */
  double mp2_energy;         /* RestrictedHartreeFock::CalculateMp2Energy when opts.mp2 */
} hfd_scf_result;

void hfd_default_scf_opts(hfd_scf_opts *o);
/* Text of the calling thread's last hfd_* failure. */
const char *hfd_last_error(void);
/* Frees the calling host thread's handles and buffers (the SCF's host-side
 * cuBLAS / cuSOLVER state and hfg_release_thread's).  A worker thread that
 * ran hfd_scf calls it before it exits, so that nothing of it is freed by
 * thread-exit destructors while the process tears CUDA down. */
void hfd_release_thread(void);
/* The Pulay (DIIS) system of DIIS.h:72 for `batch` molecules: B holds batch
 * row-major m1 x m1 bordered matrices (error inner products, then the row
 * and column of ones), c receives batch x m1 solutions of B c = (0,..,0,1)
 * by the same column-pivoted Householder QR the SCF uses. */
hfg_status hfd_pulay_solve(const double *B, int32_t m1, int32_t batch, double *c);
/* atoms: Z[natoms], xyz[3*natoms] in bohr.  density (optional) receives
 * nbf*nbf (RHF) or 2*nbf*nbf (UHF: alpha then beta) doubles; pass its
 * capacity in `density_count`. */
hfg_status hfd_scf(const char *basis_path, int32_t natoms, const int32_t *Z, const double *xyz,
                   const hfd_scf_opts *opts, hfd_scf_result *result, double *density, int64_t density_count);
/* Core Hamiltonian h = T + V and overlap S from the host one-electron code
 * (row-major nbf x nbf); *nbf is set. */
hfg_status hfd_one_electron(const char *basis_path, int32_t natoms, const int32_t *Z, const double *xyz, double *S,
                            double *h, int64_t capacity, int32_t *nbf);

#ifdef __cplusplus
}
#endif
#endif
