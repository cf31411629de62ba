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

/* Sums a partial two-electron matrix over the shards of a sharded SCF, in
 * place: dG holds `count` doubles on the device, produced on `stream`. */
typedef void (*hfd_allreduce_fn)(double *dG, int64_t count, void *stream, void *user);

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
  int32_t mp2;               /* 1: MP2 energy after the SCF (result.mp2_energy), RHF or UHF */
  int32_t concurrent_classes;/* 1: a build's classes on concurrent streams
                                (HartreeFockAlgorithm::concurrentClasses); 2: also CUDA-graph
                                replay of plain builds (cudaGraphs), for one host thread
                                driving the device; 0: neither */
  double electric_field[3];  /* Molecule::ElectricField: h += E . dipole moments (HartreeFockAlgorithm.cpp:38) */
  /* sharded builds (HartreeFockAlgorithm::shardRank / shardCount / allReduce):
   * shard_count > 1 makes every build evaluate this rank's shard and
   * `allreduce(dG, count, stream, allreduce_user)` sum G over the ranks */
  int32_t shard_rank, shard_count;
  hfd_allreduce_fn allreduce;
  void *allreduce_user;
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
  double mp2_energy;         /* Restricted/UnrestrictedHartreeFock::CalculateMp2Energy when opts.mp2 */
  double dipole[3];          /* GetMoment(): nuclear minus electronic dipole about the origin (au) */
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
/* Core Hamiltonian h = T + V and overlap S from the device one-electron
 * kernels (hfg_one_electron), copied to the host row-major nbf x nbf; *nbf
 * is set. */
hfg_status hfd_one_electron(const char *basis_path, int32_t natoms, const int32_t *Z, const double *xyz, double *S,
                            double *h, int64_t capacity, int32_t *nbf);

/* Systems::Molecule::LoadXYZ (Molecule.cpp:143-199) against the basis file:
 * on success *natoms atoms with Z[i] and xyz[3 i ..] as written in the file
 * (up to `cap` atoms) and *nbf Cartesian functions; HFG_INVALID_ARG when
 * LoadXYZ returns false (short file, unknown symbol, element missing from
 * the basis, unparsable count line).  Host only, no device work. */
hfg_status hfd_load_xyz(const char *xyz_path, const char *basis_path, int32_t cap, int32_t *natoms, int32_t *Z,
                        double *xyz, int32_t *nbf);

/* ---------------------------------------------------------------------
 * Serving pool: RHF/UHF jobs submitted at any time, run by `slots` worker
 * threads whose SCFs share the device (each job's engine context, density,
 * Fock matrix, DIIS history and screening tables stay in device memory for
 * the life of the job), admitted in arrival order as soon as a slot is free
 * and the job's estimated footprint fits in what is left of the budget.
 * The reference's counterpart is its one-std::thread-per-job document
 * (HartreeFockDoc.cpp:372-405) with HartreeFockAlgorithm::terminate
 * (HartreeFockAlgorithm.h:57) as the stop: a cancelled or timed-out job
 * stops between two SCF iterations.
 * --------------------------------------------------------------------- */
typedef struct hfg_pool hfg_pool;

enum { HFG_JOB_QUEUED = 0, HFG_JOB_RUNNING = 1, HFG_JOB_DONE = 2, HFG_JOB_FAILED = 3, HFG_JOB_CANCELLED = 4,
       HFG_JOB_TIMEOUT = 5 };

typedef struct {
  const char *basis_path;   /* copied at submission, as are Z and xyz */
  int32_t natoms;
  const int32_t *Z;
  const double *xyz;        /* bohr, 3 per atom */
  hfd_scf_opts opts;        /* the job's SCF (hfd_scf's options) */
  double timeout_s;         /* > 0: bound on submission-to-end time */
} hfg_job_spec;

typedef struct {
  int32_t state;            /* HFG_JOB_* */
  hfg_status status;        /* HFG_OK, the SCF's error, HFG_CANCELLED or HFG_TIMEOUT */
  double queue_s, run_s, latency_s;  /* submission to start, start to end, submission to end */
  int64_t footprint_bytes;  /* the admission estimate */
  hfd_scf_result result;    /* set once the job has ended (energy so far when stopped) */
} hfg_job_info;

/* slots >= 1 worker threads; hbm_budget_bytes bounds the admitted jobs' summed estimates. */
hfg_status hfg_pool_create(int32_t slots, int64_t hbm_budget_bytes, hfg_pool **out);
/* Queues a job; HFG_OOM_BUDGET when its estimate exceeds the whole budget. */
hfg_status hfg_job_submit(hfg_pool *pool, const hfg_job_spec *spec, int64_t *job_id);
/* Non-blocking state of a job. */
hfg_status hfg_job_poll(hfg_pool *pool, int64_t job_id, hfg_job_info *info);
/* Waits until the job has ended (timeout_s <= 0: no bound); HFG_TIMEOUT if it has not. */
hfg_status hfg_job_wait(hfg_pool *pool, int64_t job_id, double timeout_s, hfg_job_info *info);
/* A queued job leaves the queue; a running one stops between SCF iterations;
 * both end as HFG_JOB_CANCELLED.  No effect on an ended job. */
hfg_status hfg_job_cancel(hfg_pool *pool, int64_t job_id);
/* Jobs running and queued now, and the budget they hold. */
hfg_status hfg_pool_stats(hfg_pool *pool, int32_t *running, int32_t *queued, int64_t *used_bytes);
const char *hfg_pool_last_error(void);
/* Cancels queued and running jobs, waits for the workers, frees the pool. */
void hfg_pool_destroy(hfg_pool *pool);

#ifdef __cplusplus
}
#endif
#endif
