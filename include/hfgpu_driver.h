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
} hfd_scf_opts;

typedef struct {
  double energy;             /* HartreeFockAlgorithm::GetTotalEnergy */
  double homo;               /* HOMOEnergy */
  int32_t converged;
  int32_t iterations;
  int32_t nbf;
  int32_t reserved;
  double fock_ms_total;      /* device time spent in two-electron builds */
} hfd_scf_result;

void hfd_default_scf_opts(hfd_scf_opts *o);
/* Text of the calling thread's last hfd_* failure. */
const char *hfd_last_error(void);
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
