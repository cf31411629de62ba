// Internal definitions shared by the class kernels and the host context.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hfg {

constexpr int kMaxL = 2;                      // compiled shells: s, p, d
constexpr int kMaxLtot = 4 * kMaxL;           // highest Boys order used
constexpr int kBoysTaylor = 7;                // Taylor terms around a grid point
constexpr double kBoysStep = 0.05;            // grid spacing in T
constexpr double kBoysTmax = 36.0;            // above: asymptotic F_0 + upward recursion
constexpr int kBoysGrid = 721;                // 36 / 0.05 + 1 grid points
constexpr int kBoysOrders = kMaxLtot + kBoysTaylor;  // orders 0 .. 14 tabulated
// staged row: 7 Taylor terms and exp(-T_i), 8 doubles.  Word k of row i is
// stored at k ^ ((i >> 1) & 7) within the row: rows start on bank 0 or 16
// only, and the swizzle spreads one column of 16 consecutive rows over all
// 32 banks (plain rows put a whole warp's column on one bank pair).
constexpr int kBoysRow = kBoysTaylor + 1;
__host__ __device__ constexpr int boys_swizzle(int i, int k) { return i * kBoysRow + (k ^ ((i >> 1) & 7)); }
// Per-order rows ready for evaluation, after the e^-T tail of the table:
// table L (L = 0 .. kMaxLtot) holds in each grid row F_{L+k}(T_i) / k!
// (k < kBoysTaylor) and e^-T_i, swizzled as boys_swizzle places them.
constexpr int kBoysFoldedOff = kBoysGrid * kBoysOrders + kBoysGrid;
constexpr int kBoysFoldedSize = kBoysGrid * kBoysRow;

constexpr int kWarpsPerBlock = 4;
constexpr int kThreads = 32 * kWarpsPerBlock;
__host__ __device__ constexpr int ncart(int L) { return (L + 1) * (L + 2) / 2; }

// Warps per block of the fused class kernel.  The staged Boys table (46 KB)
// admits 4 blocks per SM: the light classes (<= 9 integrals per quartet,
// <= ~120 registers) run 8 warps per block so that the table is shared by
// more warps; the register-heavy ones keep 4, where the register file, not
// the table, sets the residency.
__host__ __device__ constexpr int fused_warps(int la, int lb, int lc, int ld) {
  return ncart(la) * ncart(lb) * ncart(lc) * ncart(ld) <= 9 ? 8 : 4;
}
// Resident blocks per SM the compiler must allow (1: the register
// allocation is free).  A 64-register cap (four 8-warp blocks per SM) fits
// (ss|ss) and (ps|ss) without spills but made (ps|ss) 20% slower alone
// (1.20 -> 1.43 ms per (H2O)16 launch) for a change within noise in the
// concurrent build; the other light classes spill under it.
__host__ __device__ constexpr int fused_min_blocks(int, int, int, int) { return 1; }
// Unroll factor of the inner (bra) primitive loop of the thread-per-quartet
// kernels (two primitive quartets in flight per lane).  Measured per class on
// the (H2O)32 / 6-31G* build: unrolling by 2 takes (ds|ps) from 2.68 to
// 2.14 ms and (ps|ss) from 4.44 to 4.34 ms, but slows (ss|ss) (2.59 -> 3.80)
// and (ps|ps) (1.75 -> 2.22), so it is per class.
__host__ __device__ constexpr int prim_unroll(int la, int lb, int lc, int ld) {
  return (la == 2 && lb == 0 && lc == 1 && ld == 0) || (la == 1 && lb == 0 && lc == 0 && ld == 0) ||
                 (la == 2 && lb == 0 && lc == 0 && ld == 0)
             ? 2
             : 1;
}
// Where a class kernel reads its Boys slice: staged into shared memory
// (46 KB per block, which also caps an SM at four such blocks over all the
// classes running at once) or straight from the per-order rows in global
// memory through L1 (kBoysFoldedOff; no shared memory).  Measured per class
// on the (H2O)32 / 6-31G* build, classes one after another: from global
// memory (ss|ss) 3.13 -> 2.66 ms, (pp|pp) 0.25 -> 0.21, (dd|ss) 0.33 -> 0.30,
// (ds|ds) 0.68 -> 0.66, (ds|pp) 0.61 -> 0.59, but (ps|ss) 4.35 -> 4.58 and
// (ds|ps), (ds|ss) 1-2% slower.
__host__ __device__ constexpr bool boys_from_global(int la, int lb, int lc, int ld) {
  return (la == 0 && lb == 0 && lc == 0 && ld == 0) || (la == 1 && lb == 1 && lc == 1 && ld == 1) ||
         (la == 2 && lb == 2 && lc == 0 && ld == 0) || (la == 2 && lb == 0 && lc == 2 && ld == 0) ||
         (la == 2 && lb == 0 && lc == 1 && ld == 1);
}
// Fused class kernels whose warps load their next task record while they
// work on the current one (every class but (ss|ss): with its Boys slice in
// global memory the prefetch made it slower, 2.66 -> 3.15 ms per (H2O)32
// build; without the prefetch the class is 4% slower with the staged slice
// and 15% faster with the global one).
__host__ __device__ constexpr bool task_prefetch(int la, int lb, int lc, int ld) {
  return la + lb + lc + ld > 0;
}
// The same choice for the split path's primitive kernel: from global memory
// (dp|ds) 1.78 -> 1.33 ms, (dp|pp) 0.95 -> 0.74, (dd|ps) 1.15 -> 0.90, (dp|dp)
// 0.87 -> 0.77, (dd|ds) 0.81 -> 0.71, (dd|pp) 0.55 -> 0.50; (dd|dp) 0.91 ->
// 2.13 ms, so it keeps the staged slice, as does (dd|dd).
__host__ __device__ constexpr bool boys_from_global_split(int la, int lb, int lc, int ld) {
  return !(la == 2 && lb == 2 && lc == 2 && (ld == 1 || ld == 2));
}

enum Mode { kStorePacked = 0, kJkRhf = 1, kJkUhf = 2, kSchwarz = 3, kBlock = 4 };

// Density screening and precision of a J/K launch.  kScreenNone: every
// Schwarz-surviving quartet in FP64.  kScreenFp64 / kScreenMixed: quartets
// whose density-weighted bound Q_ab Q_cd max|D| falls below the launch's
// density threshold are skipped.  kScreenFp64 evaluates the rest in FP64;
// kScreenMixed decides per task (one bra pair, <= 32 kets, a warp-uniform
// test): FP64 when the task's largest bound reaches the mixed cutoff, else
// FP32 primitive pairs, geometry, Boys interpolation and recursions (the
// Boys function's edges in FP64) with the J/K digestion in FP64.
enum Screen { kScreenNone = 0, kScreenFp64 = 1, kScreenMixed = 2 };

// One primitive pair of a shell pair (first shell A with exponent a, second
// B with exponent b): zeta = a+b, P = (aA+bB)/zeta, PA = P-A,
// bAB = b(A-B) and K = N_a c_a N_b c_b exp(-ab/zeta |AB|^2) sqrt(2) pi^(5/4) / zeta,
// so that the quartet prefactor 2 pi^(5/2) / (zeta eta sqrt(zeta+eta))
// exp(...) of GaussianTwoElectrons.cpp:44-45 is K_ab K_cd / sqrt(zeta+eta).
struct __align__(16) PrimPair {
  double zeta, Px, Py, Pz, PAx, PAy, PAz, bABx, bABy, bABz, K, inv_zeta;
};
// FP32 copy of a PrimPair for the mixed-precision kernels (48 B)
struct __align__(16) PrimPairF {
  float zeta, Px, Py, Pz, PAx, PAy, PAz, bABx, bABy, bABz, K, inv_zeta;
};

// Device view of one context's tables.
struct EngineView {
  const PrimPair *prim;       // all primitive pairs, pair-major
  const PrimPairF *primf;     // the same in FP32
  const int *pair_prim_off;   // per pair
  const int *pair_nprim;
  const int *pair_sa;         // first shell (higher L; higher index on ties)
  const int *pair_sb;
  const int *pair_ao_a;       // first AO of each shell of the pair
  const int *pair_ao_b;
  const double *pair_AB;      // [3*npairs] A - B
  const double *pair_Q;       // Schwarz bound
  const float *shell_dmax;    // [nshells][nshells] max |D| over each shell block (density screening)
  int nshells;
  const double *boys_table;   // [kBoysGrid][kBoysOrders] F_m(T_i), e^-T_i, then the per-order rows
  int nbf;
  int reference_convention;   // 1: reproduce the reference's (dd|dd) ET rows
  // batched contexts (many molecules, one launch per class); null otherwise
  const int *pair_mol;             // molecule of each shell pair
  const int *mol_nbf;              // basis functions per molecule
  const long long *mol_off;        // offset of each molecule's n x n matrices
  const unsigned char *mol_active; // 0: skip the molecule in this build
};

// The molecule a task belongs to (its bra pair's): its size, the offset of
// its matrices in the batch buffers, and whether this build skips it.
struct MolView {
  int n;
  long long base;
  bool skip;
};
__device__ __forceinline__ MolView task_molecule(const EngineView &v, int bp) {
  if (!v.pair_mol) return MolView{v.nbf, 0, false};
  const int m = v.pair_mol[bp];
  return MolView{v.mol_nbf[m], v.mol_off[m], v.mol_active != nullptr && v.mol_active[m] == 0};
}

// One unit of work: a bra pair position in the class's pair list and a
// range of at most 32 ket positions (kets of one primitive-count bucket).
// lg: the thread-per-quartet kernels give each quartet 2^lg lanes, which
// split its primitive quartets and sum them with warp shuffles (tasks with
// fewer kets than lanes, and long contractions); 0 = one lane per quartet.
struct __align__(16) Task {
  int bra_pos;
  int ket_start;
  int ket_end;
  int lg = 0;
};

struct ClassLaunch {
  const int *bra_list;   // pair indices of the bra class, sorted by Q desc
  const int *ket_list;   // pair indices of the ket class, sorted by Q desc
  const Task *tasks;
  int ntasks;            // tasks of this launch (of this shard)
  int task_offset;       // shard: launch task t is tasks[task_offset + t * task_stride]
  int task_stride;
  int same_class;        // bra class == ket class
  double threshold;
  // outputs by mode
  double *packed;        // kStorePacked
  const double *Da, *Db; // kJk*: densities (Db for UHF)
  const double *Dt;      // total density for J in UHF
  double *J, *Ka, *Kb;   // accumulators (n x n)
  double *Qout;          // kSchwarz: per pair
  // density screening (kScreenFp64 / kScreenMixed launches)
  float dens_threshold;  // skip quartets whose density-weighted bound is below
  float mixed_cutoff;    // tasks whose largest bound is below run in FP32
  unsigned long long *counters;  // [0] FP64, [1] FP32 quartets evaluated
  // device work queue (batched builds without host synchronisation): the
  // task count lives in device memory (written by the compaction of the
  // active molecules' tasks) and warps take the next task from an atomic
  // counter that starts at 0; null = ntasks above, static grid-stride order
  const int *ntasks_dev;
  int *queue;
};

// task t of a launch (shards take every task_stride-th task of the class)
__device__ __forceinline__ Task launch_task(const ClassLaunch &cl, int t) {
  return cl.tasks[cl.task_offset + (long long)t * cl.task_stride];
}

// Tasks of the launch: the device count when the queue is on.
__device__ __forceinline__ int launch_ntasks(const ClassLaunch &cl) {
  return cl.ntasks_dev ? *cl.ntasks_dev : cl.ntasks;
}
// A warp's first task and its next one after t: the grid-stride order
// (start, start + stride, ...) or, with the queue, one atomic per warp.
__device__ __forceinline__ int warp_fetch(int *queue, int step) {
  int t = 0;
  if ((threadIdx.x & 31) == 0) t = atomicAdd(queue, step);
  return __shfl_sync(0xffffffffu, t, 0);
}
__device__ __forceinline__ int first_task(const ClassLaunch &cl, int start) {
  return cl.queue ? warp_fetch(cl.queue, 1) : start;
}
__device__ __forceinline__ int next_task(const ClassLaunch &cl, int t, int stride) {
  return cl.queue ? warp_fetch(cl.queue, 1) : t + stride;
}

// One chunk of a split-path class launch (see eri_split.cuh): scratch for
// the contracted [e0|f0] blocks of `ntasks` tasks starting at `task0`.
struct SplitChunk {
  double *scr_fwd;   // [kAcc][slots]: block with bra = task's bra pair
  double *scr_rev;   // [kAcc][slots]: reference-convention (dd|dd) only, bra = ket pair
  long long stride;  // slots in the chunk (ntasks * 32)
  int task0;         // first task of the chunk
  int ntasks;
};

// component normalisation f(l,m,n) = 1/sqrt((2l-1)!!(2m-1)!!(2n-1)!!) in the
// canonical component order; the L-dependent part of the primitive
// normalisation sits in the contraction coefficients
template <int L>
__device__ __forceinline__ double comp_norm(int c);
template <>
__device__ __forceinline__ double comp_norm<0>(int) { return 1.0; }
template <>
__device__ __forceinline__ double comp_norm<1>(int) { return 1.0; }
template <>
__device__ __forceinline__ double comp_norm<2>(int c) {
  // xx xy xz yy yz zz
  return (c == 0 || c == 3 || c == 5) ? 0.57735026918962576451 : 1.0;
}

// Packed 8-fold index (IntegralsRepository.h:151-162)
__device__ __forceinline__ long long tri(long long a, long long b) {
  return a < b ? b * (b + 1) / 2 + a : a * (a + 1) / 2 + b;
}

// Nearest Boys grid point of 0 <= T < kBoysTmax: index i = round(T / step)
// and dT = i * step - T.  The integer comes out of the low mantissa bits of
// T / step + 1.5 * 2^52 (the sum rounds to an integer there), so no
// float-integer conversion is issued either way.
struct BoysGridPoint {
  int i;
  double dt;
};
__device__ __forceinline__ BoysGridPoint boys_grid_point(double T) {
  constexpr double kShift = 6755399441055744.0;  // 1.5 * 2^52
  const double y = fma(T, 1.0 / kBoysStep, kShift);
  return {__double2loint(y), (y - kShift) * kBoysStep - T};
}

// e^-T for T >= kBoysTmax (36), to ~1.2e-7 relative: there e^-T enters F_m
// only through the upward recursion below, where it is under 1e-6 of
// (2m+1) F_m for m <= 8, so single precision in this factor moves F_m by less
// than 1e-13 relative.  2^y with y = -T log2(e) in FP64: the integer part
// goes into the exponent field, the fraction through exp2f (underflows to
// ~2^-1022 and below, far under anything that survives the recursion).
__device__ __forceinline__ double exp_neg_far(double T) {
  const double y = -T * 1.4426950408889634074;  // log2(e)
  const double n = floor(y);
  const int ni = max((int)n, -1022);
  return (double)exp2f((float)(y - n)) * __hiloint2double((ni + 1023) << 20, 0);
}

// Boys function F_0..F_M at T.  Below kBoysTmax: 7-term Taylor expansion of
// F_M about the nearest grid point, F_M(T) = sum_k F_{M+k}(T_i) (-dT)^k / k!,
// from the shared-memory slice tab[i][k] = F_{M+k}(T_i)/k! (k < 7), then the
// downward recursion F_m = (2T F_{m+1} + e^-T) / (2m+1) (BoysFunctions.cpp:17-20)
// with e^-T = e^-T_i * e^(T_i - T), tab[i][7] = e^-T_i and the second factor
// from its 8-term Taylor series (|T_i - T| <= 0.025: truncation < 4e-18);
// both polynomials evaluated in Estrin's scheme.
// Above: F_0 = sqrt(pi/T)/2 (erfc(sqrt T) < 3e-17 there) and the upward
// recursion F_{m+1} = ((2m+1) F_m - e^-T) / (2T), 1/T as rsqrt(T)^2 and e^-T
// from exp_neg_far.  The scale folds the quartet prefactor into every order.
template <int M, class R>
__device__ __forceinline__ void boys_eval(R *F, double T, double scale, const double *__restrict__ tab) {
  if (T < kBoysTmax) {
    const BoysGridPoint gp = boys_grid_point(T);
    const int i = gp.i;
    const double dt = gp.dt;  // -(T - T_i)
    const double *t = tab + i * kBoysRow;
    const int sw = (i >> 1) & 7;
    // both polynomials in Estrin's scheme (pairs, then powers dt^2 and dt^4):
    // three dependent multiply-adds instead of six and seven in Horner's
    const double d2 = dt * dt, d4 = d2 * d2;
    const double p01 = fma(t[1 ^ sw], dt, t[0 ^ sw]), p23 = fma(t[3 ^ sw], dt, t[2 ^ sw]);
    const double p45 = fma(t[5 ^ sw], dt, t[4 ^ sw]);
    double fm[M + 1];
    fm[M] = fma(fma(t[6 ^ sw], d2, p45), d4, fma(p23, d2, p01));
    if (M > 0) {
      const double a01 = 1.0 + dt, a23 = fma(dt, 1.0 / 6.0, 0.5);
      const double a45 = fma(dt, 1.0 / 120.0, 1.0 / 24.0), a67 = fma(dt, 1.0 / 5040.0, 1.0 / 720.0);
      const double x = fma(fma(a67, d2, a45), d4, fma(a23, d2, a01));
      const double e = t[7 ^ sw] * x;
      const double t2 = 2.0 * T;
#pragma unroll
      for (int m = M - 1; m >= 0; --m) fm[m] = fma(t2, fm[m + 1], e) * (1.0 / (2 * m + 1));
    }
#pragma unroll
    for (int m = 0; m <= M; ++m) F[m] = (R)(fm[m] * scale);
  } else {
    const double r = rsqrt(T);
    double f = 0.88622692545275801365 * r;  // sqrt(pi)/2 / sqrt(T)
    F[0] = (R)(f * scale);
    if (M > 0) {
      const double e = exp_neg_far(T);
      const double h = 0.5 * r * r;
#pragma unroll
      for (int m = 0; m < M; ++m) {
        f = ((2 * m + 1) * f - e) * h;
        F[m + 1] = (R)(f * scale);
      }
    }
  }
}

}  // namespace hfg
