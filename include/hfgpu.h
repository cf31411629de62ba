/* hfgpu -- B200 (sm_100a) two-electron-integral and Fock-build engine.
 *
 * C ABI: plain pointers and sizes, no CUDA or C++ types, never throws.
 * Every entry point returns an hfg_status; hfg_last_error() gives text for
 * the calling thread's most recent failure.  Host matrices are row-major
 * nbf x nbf doubles in the reference's atomic-orbital order: atoms in
 * molecule order -> shells in basis-file order -> Cartesian components in
 * canonical order (xx, xy, xz, yy, yz, zz), the s part of an SP shell before
 * its p part.
 *
 * The reference interface each call replaces is cited as
 * file:line of aromanro/HartreeFock (HartreeFock/ directory).
 *
 * Threading: a context is used by one host thread at a time; distinct
 * contexts are independent (each owns its own CUDA stream), matching the
 * reference's one-algorithm-per-thread model (HartreeFockDoc.cpp:372-405).
 */
#ifndef HFGPU_H
#define HFGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  HFG_OK = 0,
  HFG_INVALID_ARG = 1,
  HFG_UNSUPPORTED_L = 2, /* a shell above the compiled angular momentum (d) */
  HFG_OOM_BUDGET = 3,    /* device allocation or memory budget exceeded */
  HFG_DEVICE_ERROR = 4,  /* CUDA error; context must be destroyed */
  HFG_TIMEOUT = 5,
  HFG_CANCELLED = 6,
  HFG_NO_DEVICE = 7      /* no CUDA device / kernels not loadable */
} hfg_status;

/* Which electron-transfer rows the (dd|dd) class computes.
 * HFG_ERI_REFERENCE reproduces GaussianTwoElectrons::ElectronTransfer
 * (GaussianTwoElectrons.cpp:162), whose ket column f starts at total L(f)-1;
 * for (dd|dd) quartets with a two-centre bra the reference therefore omits
 * the [d0|g0] terms.  HFG_ERI_EXACT evaluates the full recursion. */
typedef enum { HFG_ERI_REFERENCE = 0, HFG_ERI_EXACT = 1 } hfg_eri_convention;

/* Basis of one molecule, shell by shell (structure of arrays).  One entry per
 * shell letter: an SP line of the basis file is two shells (L=0 and L=1)
 * sharing exponents.  Replaces the walk over Molecule::atoms -> shells ->
 * basisFunctions (IntegralsRepository.cpp:566-578, Molecule.cpp:41-72). */
typedef struct {
  int32_t nshells;
  const double *center;      /* [3*nshells], bohr */
  const int32_t *L;          /* [nshells], 0..2 */
  const int32_t *nprim;      /* [nshells] */
  const int32_t *prim_offset; /* [nshells] into exponent/coefficient */
  const int32_t *ao_offset;  /* [nshells] first AO index of the shell */
  const double *exponent;    /* [sum nprim] */
  const double *coefficient; /* [sum nprim] contraction coefficients from the
                                basis file; the per-component primitive
                                normalisation of GaussianOrbital.cpp:25-30 is
                                applied inside */
  int32_t nbf;               /* number of Cartesian basis functions */
} hfg_shells;

/* Direct Fock builds come in two forms.  The plain form (all fields below
 * at their defaults) evaluates every quartet that survives the Schwarz test
 * in FP64 from the full density, as the reference does.  The precision form
 * is switched on by any of density_screening, incremental or a positive
 * mixed_cutoff:
 *   - density screening: a quartet is skipped when its density-weighted
 *     bound Q_ab Q_cd max|D| (max over the six shell blocks of D that its
 *     J/K digestion reads) is below density_threshold;
 *   - mixed precision: of the kept quartets, those of a task (one bra shell
 *     pair and up to 32 ket pairs) whose largest density-weighted bound is
 *     below mixed_cutoff are evaluated with FP32 recursions (FP64 Boys
 *     function, prefactor and J/K accumulation); the others in FP64;
 *   - incremental: the context keeps the previous density and two-electron
 *     matrix; each build evaluates G[P - P_prev] and returns
 *     G_prev + G[P - P_prev].  hfg_fock_reset() starts over from P_prev = 0. */
typedef struct {
  double schwarz_threshold; /* skip quartets with Q_ab*Q_cd below this (1e-12) */
  double mixed_cutoff;      /* FP32 below this density-weighted bound; 0 = all
                               FP64 (default 0; the precision form uses 1e-4) */
  int32_t eri_convention;   /* hfg_eri_convention, default HFG_ERI_REFERENCE */
  int32_t device;           /* CUDA ordinal, default 0 */
  int32_t density_screening;/* 1: skip quartets below density_threshold */
  int32_t incremental;      /* 1: build from the density difference */
  double density_threshold; /* density screening cutoff; 0 = schwarz_threshold */
  int32_t cuda_graphs;      /* 1: plain-form direct builds replay a CUDA graph
                               (hfg_set_graphs); default 0 */
  int32_t concurrent_classes; /* 1: a build's class kernels run concurrently
                               on the build stream and twelve auxiliary streams
                               (hfg_set_streams); default 0 */
} hfg_opts;

typedef struct hfg_ctx hfg_ctx;

typedef struct {
  int64_t shell_pairs;         /* significant shell pairs */
  int64_t shell_quartets;      /* Schwarz-surviving quartets of the last build */
  int64_t function_quartets;   /* 8-fold unique function quartets, same build */
  int64_t primitive_quartets;  /* primitive quartets, same build */
  int64_t fp32_shell_quartets; /* precision form: quartets evaluated in FP32 */
  int64_t fp64_shell_quartets; /* precision form: quartets evaluated in FP64
                                  (plain form: = shell_quartets) */
  double flops;                /* algorithmic flops of the last build */
  double last_build_ms;        /* device time of the last build (events) */
  int32_t kernel_launches;     /* kernels launched by the last build */
  int32_t reserved;
} hfg_stats;

void hfg_default_opts(hfg_opts *opts);
const char *hfg_last_error(void);
/* Number of CUDA devices visible (0 if none). */
int32_t hfg_device_count(void);

/* Builds the shell pairs, primitive-pair tables, Schwarz bounds and class
 * lists on the device.  Replaces IntegralsRepository(Molecule*) / Reset
 * (IntegralsRepository.h:49-51, IntegralsRepository.cpp:19-27). */
hfg_status hfg_ctx_create(const hfg_shells *shells, const hfg_opts *opts, hfg_ctx **out);
void hfg_ctx_destroy(hfg_ctx *ctx);
int32_t hfg_ctx_nbf(const hfg_ctx *ctx);

/* Number of doubles of the packed 8-fold table: GetElectronElectronIndex(n-1,
 * n-1, n-1, n-1) + 1 (IntegralsRepository.h:151-162). */
int64_t hfg_packed_size(int32_t nbf);

/* Stored mode: the packed ERI table, index T(T(i,j),T(k,l)) with
 * T(a,b) = max(max+1)/2 + min.  Replaces
 * IntegralsRepository::CalculateElectronElectronIntegrals
 * (IntegralsRepository.cpp:566-584); entries of screened-out quartets are 0.
 * host_out holds `count` doubles (hfg_packed_size). */
hfg_status hfg_eri_packed(hfg_ctx *ctx, double *host_out, int64_t count);
/* Same, into device memory on `stream` (a cudaStream_t, 0 = context stream). */
hfg_status hfg_eri_packed_device(hfg_ctx *ctx, double *dev_out, int64_t count, void *stream);

/* One contracted integral (i j | k l).  Replaces
 * IntegralsRepository::getElectronElectron(contracted x4)
 * (IntegralsRepository.cpp:372-433). */
hfg_status hfg_eri_quartet(hfg_ctx *ctx, int32_t i, int32_t j, int32_t k, int32_t l, double *out);

/* Direct RHF two-electron matrix G = J[P] - K[P]/2 from the density P,
 * G_ij = sum_kl P_kl[(ij|kl) - 1/2 (il|kj)], without storing integrals.
 * Replaces the iter > 0 branch of RestrictedHartreeFock::InitFockMatrix
 * (RestrictedHartreeFock.cpp:187-203); the caller forms F = h + G. */
hfg_status hfg_fock_rhf(hfg_ctx *ctx, const double *P, double *G);
/* Direct UHF: G+ = J[P+ + P-] - K[P+], G- = J[P+ + P-] - K[P-].  Replaces
 * UnrestrictedHartreeFock::InitFockMatrices (UnrestrictedHartreeFock.cpp:223-240). */
hfg_status hfg_fock_uhf(hfg_ctx *ctx, const double *Pa, const double *Pb, double *Ga, double *Gb);
/* Device-pointer forms on `stream` (cudaStream_t or 0). */
hfg_status hfg_fock_rhf_device(hfg_ctx *ctx, const double *dP, double *dG, void *stream);
hfg_status hfg_fock_uhf_device(hfg_ctx *ctx, const double *dPa, const double *dPb, double *dGa, double *dGb,
                               void *stream);

/* Precision form controls (see hfg_opts).  No reference counterpart: the
 * reference rebuilds the full two-electron matrix in FP64 every iteration
 * (RestrictedHartreeFock.cpp:168-207).
 * hfg_fock_reset: drop the incremental history, so that the next build
 * evaluates G from the full density (P_prev = 0, G_prev = 0).
 * hfg_set_mixed_cutoff: FP32 cutoff of the following builds (0 = all FP64);
 * an SCF driver finishes with hfg_set_mixed_cutoff(ctx, 0) plus
 * hfg_fock_reset(ctx), so that its last iterations run all-FP64.
 * hfg_set_incremental: switch incremental builds on or off (resets). */
hfg_status hfg_fock_reset(hfg_ctx *ctx);
hfg_status hfg_set_mixed_cutoff(hfg_ctx *ctx, double cutoff);
hfg_status hfg_set_incremental(hfg_ctx *ctx, int32_t on);

/* Sharded direct builds (one molecule over several GPUs; no reference
 * counterpart): with shard (rank, count) set, hfg_fock_rhf/uhf[_device]
 * evaluate only the rank-th of `count` contiguous task ranges of each
 * quartet class, ranges of equal estimated cost (primitive quartets times the
 * class's per-primitive flops, plus its per-quartet horizontal recursions),
 * and return that shard's partial G.  The partial G of the `count` shards
 * sum to the full G (G is linear in the J/K sums); the caller reduces them,
 * e.g. with one NCCL all-reduce (hartreefock_b200/shards.py).  Incremental
 * builds keep a per-shard history.  Stored builds (hfg_eri_packed) and
 * hfg_fock_rhf_noalloc are not sharded.  Default (0, 1). */
hfg_status hfg_set_shard(hfg_ctx *ctx, int32_t rank, int32_t count);
/* The shard partition itself (host arithmetic, no device): given the
 * running cost of a class's `ntasks` tasks (cost_prefix[0] = 0,
 * cost_prefix[t + 1] = cost of tasks 0..t, ntasks + 1 entries), the
 * contiguous task range [*first, *first + *ntasks_out) of shard `rank` of
 * `count`: shard r starts at the first task whose prefix reaches
 * r / count of the total.  The ranges of ranks 0..count-1 tile the tasks. */
hfg_status hfg_shard_range(const double *cost_prefix, int64_t ntasks, int32_t rank, int32_t count, int64_t *first,
                           int64_t *ntasks_out);
/* Device-to-device copy of `bytes` on `stream`, finished when the call
 * returns (for callers that move a sharded G into their own buffers). */
hfg_status hfg_copy_device(void *dst, const void *src, int64_t bytes, void *stream);

/* Batched contexts (many independent molecules; no reference counterpart:
 * the reference runs one molecule per algorithm object).  hfg_batch_create
 * takes one hfg_shells per molecule (AO offsets local to the molecule) and
 * builds shell pairs and quartets within each molecule only; every direct
 * build then runs one launch per quartet class over the tasks of all
 * molecules.  Matrices of the batch live in flat device buffers, molecule m's
 * nbf[m] x nbf[m] row-major block at offset[m] (hfg_batch_layout; `total`
 * doubles in all).  `active` (host, one byte per molecule, or NULL = all)
 * selects the molecules a build serves; the G blocks of the others are left
 * untouched.  Plain FP64 form only; sharding applies.  The single-molecule
 * entry points reject batched contexts. */
hfg_status hfg_batch_create(const hfg_shells *mols, int32_t nmol, const hfg_opts *opts, hfg_ctx **out);
int32_t hfg_batch_size(const hfg_ctx *ctx);
hfg_status hfg_batch_layout(const hfg_ctx *ctx, int32_t *nbf, int64_t *offset, int64_t *total);
hfg_status hfg_fock_rhf_batch_device(hfg_ctx *ctx, const double *dP, double *dG, const uint8_t *active, void *stream);
hfg_status hfg_fock_uhf_batch_device(hfg_ctx *ctx, const double *dPa, const double *dPb, double *dGa, double *dGb,
                                     const uint8_t *active, void *stream);
/* The same builds with the active mask in device memory (d_active[nmol],
 * 0 = skip the molecule) and no host synchronisation: the active molecules'
 * tasks are compacted on the device and the class kernels take them from a
 * device work queue (one atomic task counter per class, a fixed grid), so a
 * caller can capture a whole batched SCF iteration in a CUDA graph.  The
 * large classes always run on the warp-cooperative kernels here (no scratch
 * sized on the host).  The first call allocates the context's work buffers;
 * capture after it.  No
 * reference counterpart (one molecule per algorithm object there). */
hfg_status hfg_fock_rhf_batch_async(hfg_ctx *ctx, const double *dP, double *dG, const uint8_t *d_active,
                                    void *stream);
hfg_status hfg_fock_uhf_batch_async(hfg_ctx *ctx, const double *dPa, const double *dPb, double *dGa, double *dGb,
                                    const uint8_t *d_active, void *stream);

/* One-electron matrices on `device`: overlap S, kinetic energy T and
 * nuclear attraction V (h = T + V), each row-major nbf x nbf in host memory,
 * for the shells `shells` and the nuclei (xyz[3*natoms] bohr, charges Z).
 * Replaces IntegralsRepository's one-electron part and QuantumMatrix
 * (IntegralsRepository.cpp:34-321, QuantumMatrix.cpp:34-155).  Needs no
 * context; allocates and frees its own device buffers. */
hfg_status hfg_one_electron(const hfg_shells *shells, const double *xyz, const int32_t *Z, int32_t natoms,
                            int32_t device, double *S, double *T, double *V);

/* Dipole moment matrices about the origin, <a|x|b>, <a|y|b>, <a|z|b>
 * (row-major nbf x nbf): MomentMatrix::Calculate (QuantumMatrix.cpp:61-98)
 * through GaussianMoment (GaussianMoment.cpp:44-90), on the device. */
hfg_status hfg_moments(const hfg_shells *shells, int32_t device, double *Mx, double *My, double *Mz);

/* AO -> MO transform for the post-HF consumers (no allocation-free form):
 * dX receives the (ia|jb) block, i in [i0, i0+ni), a in [a0, a0+na), as a
 * row-major (ni*na) x (ni*na) matrix with row i*na + a, from the MO
 * coefficients dC (device, row-major nbf x nbf: AO rows, MO columns, the
 * reference's C).  Replaces MolecularOrbitalsIntegralsRepository::
 * getElectronElectron (IntegralsRepository.h:190-291) for that block.  Uses
 * the context's stored-mode table (its screening and ERI convention),
 * unpacked on the device: needs about 9/8 nbf^4 doubles free, else
 * HFG_OOM_BUDGET.  Single-molecule contexts only. */
hfg_status hfg_mo_eri_ovov(hfg_ctx *ctx, const double *dC, int32_t i0, int32_t ni, int32_t a0, int32_t na, double *dX,
                           void *stream);
/* The whole MO tensor (pq|rs) for every orbital of dC (device, row-major
 * nbf x nbf), as dX[(p q),(r s)] (nbf^2 x nbf^2, row-major): the elements
 * MolecularOrbitalsIntegralsRepository::getElectronElectron(p, q, r, s, C)
 * returns (IntegralsRepository.h:190-291).  Needs about 11/8 nbf^4 doubles
 * free.  Single-molecule contexts only. */
hfg_status hfg_mo_eri_full(hfg_ctx *ctx, const double *dC, double *dX, void *stream);
/* SpinOrbitalsElectronElectronIntegralsRepository::Compute
 * (SpinOrbitalsElectronElectronIntegralsRepository.cpp:30-52) for host C
 * (row-major nbf x nbf): out[((p m + q) m + r) m + s], m = 2 nbf, spin orbital
 * p = spatial orbital p / 2 with spin p % 2, receives
 *   (p/2 r/2 | q/2 s/2) [p, r and q, s of one spin] - (p/2 s/2 | q/2 r/2) [p, s and q, r of one spin],
 * the antisymmetrised integrals of the CCSD and CIS consumers; `count` >= m^4. */
hfg_status hfg_spin_orbital_eri(hfg_ctx *ctx, const double *C, double *out, int64_t count);
/* RHF MP2 correlation energy from host C (row-major nbf x nbf) and orbital
 * energies eps[nbf], the lowest nocc orbitals occupied:
 * sum (ia|jb)[2(ia|jb) - (ib|ja)] / (e_i + e_j - e_a - e_b).  Replaces
 * RestrictedHartreeFock::CalculateMp2Energy (RestrictedHartreeFock.cpp:251-288). */
hfg_status hfg_mp2_rhf(hfg_ctx *ctx, const double *C, const double *eps, int32_t nocc, double *e_mp2);
/* UHF MP2 energy as UnrestrictedHartreeFock::CalculateMp2Energy computes it
 * (UnrestrictedHartreeFock.cpp:295-375): 0.25 (S+ + S-), S = sum over the
 * spin's occupied i, j and virtual a, b of (ia|jb)^2 / (e_i + e_j - e_a - e_b),
 * from host C+ / C- (row-major nbf x nbf), orbital energies e+ / e- and the
 * occupied counts 0 <= n+, n- <= nbf (lowest orbitals; either may be the
 * larger -- Molecule::Init, Molecule.cpp:132-139, gives the odd electron to
 * the minus spin).  The reference evaluates both sums through one
 * MolecularOrbitalsIntegralsRepository whose caches are keyed by orbital
 * indices only (IntegralsRepository.h:190-291), so its S- reuses values
 * cached with C+; this reproduces that: in S- index b takes C+ when virtual+,
 * j when also occupied+, a when also virtual+, i when also occupied+, and
 * every other index C-. */
hfg_status hfg_mp2_uhf(hfg_ctx *ctx, const double *Cplus, const double *eplus, int32_t nplus, const double *Cminus,
                       const double *eminus, int32_t nminus, double *e_mp2);

/* Frees the calling host thread's library state (the batched eigensolver's
 * handle and workspace).  For worker threads that exit while the process
 * goes on: call it before the thread ends. */
void hfg_release_thread(void);

/* Eigen-decomposition of `batch` symmetric n x n matrices (device, FP64,
 * contiguous) on `stream`: dW receives batch x n ascending eigenvalues, dV
 * batch x n x n eigenvectors with eigenvector k of matrix b in row k of block
 * b (dV may equal dA).  method 0: one batched cuSOLVER call (Jacobi);
 * method 1: one divide-and-conquer solve (dsyevd) per matrix, the solver of
 * the single-molecule SCF -- within a degenerate level the two return
 * different bases, which decides the occupied orbitals of open shells.  The batched SCF's
 * counterpart of the per-molecule Eigen::SelfAdjointEigenSolver step
 * (RestrictedHartreeFock.cpp:121-124).  Workspace is kept per host thread. */
hfg_status hfg_eigh_batched(const double *dA, double *dV, double *dW, int32_t n, int32_t batch, int32_t method,
                            void *stream);

/* The DIIS systems of a batch of molecules on the device: for each of
 * `batch` row-major m1 x m1 matrices in dB (the Pulay matrix bordered by
 * ones, DIIS.h:34-96), dC receives the m1 solution entries of
 * B c = (0, ..., 0, 1) by column-pivoted Householder QR with a rank cut-off
 * (the role of colPivHouseholderQr, DIIS.h:72), the same algorithm as the
 * host SCF's solve.  2 <= m1 <= 8.  Asynchronous on `stream`. */
hfg_status hfg_pulay_solve_device(const double *dB, int32_t m1, int32_t batch, double *dC, void *stream);

/* Allocation-free variant of hfg_fock_rhf_device, for callers that must not
 * allocate device memory while they run: a serving loop under a fixed HBM
 * budget, code that cannot afford the implicit synchronisation of
 * cudaMalloc/cudaFree, or a host without allocator access on that path.
 * No counterpart in the reference.  The J/K accumulators live in a
 * file-scope device array of 2 x 1024 x 1024 doubles (16 MiB) that every GPU
 * loading the library keeps until exit; contexts above 1024 basis functions
 * are rejected with HFG_INVALID_ARG.  The large classes run on the
 * warp-cooperative kernels (shared memory only), so no other scratch is
 * used: the context (created beforehand with hfg_ctx_create, which does
 * allocate) and the caller's device buffers dP, dG are the only other memory.
 * The call always does a plain full FP64 build; a context with
 * precision-form settings (density screening, an FP32 cutoff or incremental
 * builds) is rejected with HFG_INVALID_ARG.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress) and should come
 * before any stream capture; the CUDA driver also sizes its per-thread
 * local-memory reservation on a kernel's first launch in the process, so a
 * caller that must see no allocation inside the call makes one call (or one
 * hfg_fock_rhf_device build) beforehand.  All calls share the array: calls
 * that overlap on the GPU (different streams or contexts at the same time)
 * race on it. */
hfg_status hfg_fock_rhf_noalloc(hfg_ctx *ctx, const double *dP, double *dG, void *stream);

/* Schwarz bounds sqrt(max (ij|ij)) per shell pair (a >= b), in pair order
 * a*(a+1)/2 + b; `count` = nshells*(nshells+1)/2. */
hfg_status hfg_schwarz(hfg_ctx *ctx, double *host_out, int64_t count);

hfg_status hfg_ctx_stats(const hfg_ctx *ctx, hfg_stats *out);

/* CUDA graphs for the plain-form direct build (no reference counterpart):
 * with `on`, the second hfg_fock_*_device / hfg_fock_* call with the same
 * buffers, stream and settings is captured into a graph and later ones
 * replay it (one launch instead of ~30).  Needs a created stream (not the
 * legacy default stream; 0 selects the context's own).  Any setter
 * (autotune, shard, precision settings, profiling) starts over. */
hfg_status hfg_set_graphs(hfg_ctx *ctx, int32_t on);
/* Concurrent class kernels (no reference counterpart): with `on`, the
 * quartet classes of a direct or batched build are spread over the build
 * stream and twelve auxiliary streams of the context (forked and joined by
 * events; J/K accumulate by atomics, each split class stream has its own
 * scratch region), so small molecules' class kernels overlap. */
hfg_status hfg_set_streams(hfg_ctx *ctx, int32_t on);
/* Task shape of the thread-per-quartet classes (no reference counterpart):
 * a quartet whose primitive quartets exceed `target` per lane is spread over
 * a group of 2..32 lanes that split its primitive loop and sum the
 * contraction with warp shuffles, and tasks carry correspondingly fewer kets
 * (0: one lane per quartet; default 96).  Rebuilds the task lists. */
hfg_status hfg_set_prim_target(hfg_ctx *ctx, int32_t target);
/* Picks that target per class (0, 48, 96, 192, 384) by timing each class's
 * J/K kernel on the caller's device density dP; `chosen` receives
 * (La, Lb, Lc, Ld, target) per tuned class.  Single-molecule contexts. */
hfg_status hfg_autotune_tasks(hfg_ctx *ctx, const double *dP, int32_t *chosen, int32_t cap, int32_t *count,
                              void *stream);

/* Kernel of the large classes that have two (no reference counterpart):
 * `path` 1 runs quartet class (La Lb | Lc Ld) on the warp-cooperative kernel
 * (one warp per shell quartet, recursions from a level-ordered program in
 * shared memory, no scratch), 0 on the split path (primitive kernel, then the
 * HRR / digestion kernel over scratch).  Default: warp for (dd|dd), split for
 * the rest.  HFG_INVALID_ARG for a class without both kernels.  Batched
 * asynchronous builds and hfg_fock_rhf_noalloc always use the warp kernel. */
hfg_status hfg_set_class_path(hfg_ctx *ctx, int32_t la, int32_t lb, int32_t lc, int32_t ld, int32_t path);
/* Picks that kernel per class by timing both on the caller's device density
 * dP (one warm-up, two timed launches each, CUDA events); `chosen` receives
 * (La, Lb, Lc, Ld, path) per tuned class.  Single-molecule contexts. */
hfg_status hfg_autotune_paths(hfg_ctx *ctx, const double *dP, int32_t *chosen, int32_t cap, int32_t *count,
                              void *stream);

/* Grid autotuner (no reference counterpart): times every fused quartet
 * class's J/K kernel at 1, 2, 4, 8 and 16 blocks per SM on the density dP
 * (device; a flat batch buffer for batched contexts) and keeps the fastest
 * grid per class for this context's later builds.  `chosen` (optional)
 * receives up to cap/5 records (La, Lb, Lc, Ld, blocks per SM); *count the
 * records written.  Costs about 15 launches per class.  With concurrent
 * class streams (hfg_set_streams) on a single-molecule plain-form context,
 * the classes share the SMs, so one cap for all classes (1, 2 or 4 blocks
 * per SM) is chosen from whole builds instead; its record is
 * (-1, -1, -1, -1, blocks per SM).  The classes whose kernels hold no
 * shared memory (their Boys rows read from global memory) then try twice
 * and four times that cap, again on whole builds; a higher cap that wins
 * adds one record per such class. */
hfg_status hfg_autotune(hfg_ctx *ctx, const double *dP, int32_t *chosen, int32_t cap, int32_t *count, void *stream);

/* Per-class timing of the builds (no reference counterpart: instrumentation
 * for the roofline accounting).  With profiling on, every class launch of a
 * build is bracketed by CUDA events on the build's stream. */
typedef struct {
  int32_t la, lb, lc, ld;   /* class (La Lb | Lc Ld) */
  int64_t shell_quartets;
  int64_t function_quartets;
  int64_t primitive_quartets;
  double flops;             /* algorithmic flops of the class in one build */
  double ms;                /* device time of the class kernel, last build */
  int64_t tasks;            /* tasks (one bra pair, <= 32 ket pairs) of the class */
  double lane_occupancy;    /* primitive quartets the lanes evaluate / (32 x the longest
                               lane loop) over the tasks, for a thread per quartet */
  int32_t warp_kernel;      /* 1: one warp per quartet (the large classes) */
  int32_t reserved;
} hfg_class_time;
hfg_status hfg_set_profiling(hfg_ctx *ctx, int32_t on);
/* Writes up to `cap` entries (largest flops first); *count = entries written. */
hfg_status hfg_class_profile(const hfg_ctx *ctx, hfg_class_time *out, int32_t cap, int32_t *count);

/* Device peak of dependent-free FP64 FMA issue, measured by a short
 * microbenchmark on `device` (TFLOP/s, 2 flops per FMA).  Instrumentation
 * for the roofline denominator; no reference counterpart. */
hfg_status hfg_measure_fp64_peak(int32_t device, double *tflops);
/* The same for FP32 FMA (the precision form's FP32 quartets); no counterpart
 * in the reference. */
hfg_status hfg_measure_fp32_peak(int32_t device, double *tflops);

#ifdef __cplusplus
}
#endif
#endif
