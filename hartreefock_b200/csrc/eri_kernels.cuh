// Shell-quartet class kernels: one thread per contracted shell quartet, one
// warp per (bra pair, 32 consecutive ket pairs).  The bra pair is shared by
// the warp (its primitive pairs are broadcast loads), the ket pairs come from
// the Schwarz-sorted ket list of the class.  The Boys table slice the class
// needs is staged into shared memory once per block, or read from global
// memory through L1 (boys_from_global).
#pragma once

#include <type_traits>

#include "eri_gen.cuh"
#include "hfg_internal.cuh"

namespace hfg {

// full unrolling for blocks whose values fit in registers, rolled loops above
template <int N>
constexpr int kUnrollBlock = N <= 81 ? 64 : 1;

__device__ __forceinline__ double inv_factorial(int k) {
  // 1/k! for k = 0..6 as a select chain (an indexed array would live in
  // local memory and be rebuilt on every call)
  return k <= 1 ? 1.0 : k == 2 ? 0.5 : k == 3 ? 1.0 / 6.0 : k == 4 ? 1.0 / 24.0 : k == 5 ? 1.0 / 120.0 : 1.0 / 720.0;
}

template <int LTOT>
__device__ __forceinline__ void stage_boys(double *tab, const double *__restrict__ g) {
  for (int x = threadIdx.x; x < kBoysGrid * kBoysRow; x += blockDim.x) {
    const int i = x / kBoysRow, k = x - i * kBoysRow;
    // Taylor coefficients F_{LTOT+k}(T_i)/k!, then e^-T_i from the table's
    // tail, each at its swizzled place in the row
    tab[boys_swizzle(i, k)] =
        k < kBoysTaylor ? g[i * kBoysOrders + LTOT + k] * inv_factorial(k) : g[kBoysGrid * kBoysOrders + i];
  }
  __syncthreads();
}

// FP64 Boys function for the two edges the FP32 paths do not serve:
// T < kBoysStep (series F_M(T) = sum_k (-T)^k / (k! (2M+2k+1)), 9 terms,
// truncation below 1e-17 there, then the downward recursion) and the band
// just above the asymptotic switch (asymptotic F_0 and the upward
// recursion, as boys_eval).
template <int M>
__device__ __noinline__ void boys_edges_fp64(double *F, double T, double scale) {
  if (T < kBoysStep) {
    double term = 1.0, f = 0.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      f += term / (2 * M + 2 * k + 1);
      term *= -T / (k + 1);
    }
    double fm[M + 1];
    fm[M] = f;
    const double e = exp(-T), t2 = 2.0 * T;
#pragma unroll
    for (int m = M - 1; m >= 0; --m) fm[m] = fma(t2, fm[m + 1], e) * (1.0 / (2 * m + 1));
#pragma unroll
    for (int m = 0; m <= M; ++m) F[m] = fm[m] * scale;
  } else {
    const double r = rsqrt(T);
    double f = 0.88622692545275801365 * r;
    F[0] = f * scale;
    const double e = exp_neg_far(T), h = 0.5 * r * r;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      f = ((2 * m + 1) * f - e) * h;
      F[m + 1] = f * scale;
    }
  }
}

// FP32 Boys function: the 7-term Taylor expansion and the downward recursion
// of boys_eval in single precision on [kBoysStep, kBoysTmax) (coefficients
// rounded from the staged FP64 table), the asymptotic form in single
// precision from kBoysTmax + kBoysF32Band on, FP64 near T = 0 and in the band
// at the switch.  (The far, small quartets that run in FP32 are mostly at
// large T: the asymptotic branch is their common case.)
constexpr float kBoysF32Band = 4.0f;
template <int M>
__device__ __forceinline__ void boys_eval_f32(float *F, float T, float scale, const double *__restrict__ tab) {
  if (T >= (float)kBoysTmax + kBoysF32Band) {
    const float r = rsqrtf(T);
    float f = 0.88622692545275801365f * r;  // sqrt(pi)/2 / sqrt(T)
    F[0] = f * scale;
    if (M > 0) {
      const float e = __expf(-T), h = 0.5f * r * r;
#pragma unroll
      for (int m = 0; m < M; ++m) {
        f = ((2 * m + 1) * f - e) * h;
        F[m + 1] = f * scale;
      }
    }
  } else if (T >= (float)kBoysStep && T < (float)kBoysTmax) {
    const int i = __float2int_rn(T * (float)(1.0 / kBoysStep));
    const float dt = (float)i * (float)kBoysStep - T;
    const double *t = tab + i * kBoysRow;
    const int sw = (i >> 1) & 7;
    float f = (float)t[6 ^ sw];
#pragma unroll
    for (int k = 5; k >= 0; --k) f = fmaf(f, dt, (float)t[k ^ sw]);
    float fm[M + 1];
    fm[M] = f;
    if (M > 0) {
      // e^(T_i - T), |dt| <= 0.025: five terms reach float precision
      float x = 1.0f / 120.0f;
      x = fmaf(x, dt, 1.0f / 24.0f);
      x = fmaf(x, dt, 1.0f / 6.0f);
      x = fmaf(x, dt, 0.5f);
      x = fmaf(x, dt, 1.0f);
      x = fmaf(x, dt, 1.0f);
      const float e = (float)t[7 ^ sw] * x, t2 = 2.0f * T;
#pragma unroll
      for (int m = M - 1; m >= 0; --m) fm[m] = fmaf(t2, fm[m + 1], e) * (1.0f / (2 * m + 1));
    }
#pragma unroll
    for (int m = 0; m <= M; ++m) F[m] = fm[m] * scale;
  } else {
    double Fd[M + 1];
    boys_edges_fp64<M>(Fd, (double)T, (double)scale);
#pragma unroll
    for (int m = 0; m <= M; ++m) F[m] = (float)Fd[m];
  }
}

// Contracted [e0|f0] of one shell quartet (bra pair `bp`, ket pair `kp`)
// accumulated into acc: the primitive loops.  R = double: FP64 throughout;
// R = float: the FP32 primitive pairs and FP32 arithmetic (mixed
// precision), with the Boys function's edges in FP64.
// lg > 0: the 2^lg lanes of an aligned lane group share the quartet; lane gl
// of the group takes the primitive quartets gl, gl + 2^lg, ... of the
// (ket primitive, bra primitive) grid and the group sums its accumulators
// with shuffles afterwards (warp-shuffle contraction), so every lane of the
// group ends with the whole contracted block.  lg is warp-uniform.
template <int LA, int LB, int LC, int LD, bool REF, class R>
__device__ __forceinline__ void accumulate_primitives_grouped(const EngineView &v, const double *tab, int bp, int kp,
                                                              int npk, R *acc, int lg) {
  constexpr int LTOT = LA + LB + LC + LD;
  using Cls = EriClass<LA, LB, LC, LD, REF>;
  const int G = 1 << lg, gl = threadIdx.x & (G - 1);
  const int offb = v.pair_prim_off[bp], npb = v.pair_nprim[bp];
  const int offk = v.pair_prim_off[kp];
  const int total = npk * npb;
  int ik = npb > 0 ? gl / npb : 0, ib = npb > 0 ? gl - ik * npb : 0;
  for (int w = gl; w < total; w += G) {
    if constexpr (std::is_same<R, float>::value) {
      const PrimPairF pk = v.primf[offk + ik], pb = v.primf[offb + ib];
      const float rs = rsqrtf(pb.zeta + pk.zeta);
      const float rho = pb.zeta * pk.zeta * (rs * rs);
      const float PQx = pb.Px - pk.Px, PQy = pb.Py - pk.Py, PQz = pb.Pz - pk.Pz;
      const float T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
      float F[LTOT + 1];
      boys_eval_f32<LTOT>(F, T, pb.K * pk.K * rs, tab);
      const float roz = rho * pb.inv_zeta, ie = pk.inv_zeta;
      Cls::template prim<float>(acc, F, pb.PAx, pb.PAy, pb.PAz, -roz * PQx, -roz * PQy, -roz * PQz,
                                0.5f * pb.inv_zeta, roz, -(pb.bABx + pk.bABx) * ie, -(pb.bABy + pk.bABy) * ie,
                                -(pb.bABz + pk.bABz) * ie, pb.zeta * ie, 0.5f * ie);
    } else {
      const PrimPair pk = v.prim[offk + ik], pb = v.prim[offb + ib];
      const double rs = rsqrt(pb.zeta + pk.zeta);
      const double rho = pb.zeta * pk.zeta * (rs * rs);
      const double PQx = pb.Px - pk.Px, PQy = pb.Py - pk.Py, PQz = pb.Pz - pk.Pz;
      const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
      double F[LTOT + 1];
      boys_eval<LTOT, double>(F, T, pb.K * pk.K * rs, tab);
      const double roz = rho * pb.inv_zeta, ie = pk.inv_zeta;
      Cls::template prim<double>(acc, F, pb.PAx, pb.PAy, pb.PAz, -roz * PQx, -roz * PQy, -roz * PQz,
                                 0.5 * pb.inv_zeta, roz, -(pb.bABx + pk.bABx) * ie, -(pb.bABy + pk.bABy) * ie,
                                 -(pb.bABz + pk.bABz) * ie, pb.zeta * ie, 0.5 * ie);
    }
    ib += G;
    while (ib >= npb) {
      ib -= npb;
      ++ik;
    }
  }
  for (int o = 1; o < G; o <<= 1)
#pragma unroll
    for (int x = 0; x < Cls::kAcc; ++x) acc[x] += __shfl_xor_sync(0xffffffffu, acc[x], o);
}

// `acc`: the block's accumulators, a register array (R*) or any indexable
// accumulator type (lane groups need the register array).
template <int LA, int LB, int LC, int LD, bool REF, class R, class A>
__device__ __forceinline__ void accumulate_primitives(const EngineView &v, const double *tab, int bp, int kp, int npk,
                                                      A acc, int lg = 0) {
  if constexpr (std::is_pointer<A>::value) {
    if (lg > 0) {
      accumulate_primitives_grouped<LA, LB, LC, LD, REF, R>(v, tab, bp, kp, npk, acc, lg);
      return;
    }
  }
  constexpr int LTOT = LA + LB + LC + LD;
  using Cls = EriClass<LA, LB, LC, LD, REF>;
  const int offb = v.pair_prim_off[bp], npb = v.pair_nprim[bp];
  const int offk = v.pair_prim_off[kp];
  // ket primitive pairs differ across the warp's lanes: load each once; the
  // bra primitive pairs are shared by the warp (broadcast loads).  Staging
  // them in shared memory per task was measured slower (generic loads).
  if constexpr (std::is_same<R, float>::value) {
    const PrimPairF *bsrc = v.primf + offb;
    for (int ik = 0; ik < npk; ++ik) {
      const PrimPairF pk = v.primf[offk + ik];
      for (int ib = 0; ib < npb; ++ib) {
        const PrimPairF pb = bsrc[ib];
        const float rs = rsqrtf(pb.zeta + pk.zeta);
        const float rho = pb.zeta * pk.zeta * (rs * rs);
        const float PQx = pb.Px - pk.Px, PQy = pb.Py - pk.Py, PQz = pb.Pz - pk.Pz;
        const float T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
        float F[LTOT + 1];
        boys_eval_f32<LTOT>(F, T, pb.K * pk.K * rs, tab);
        const float roz = rho * pb.inv_zeta;
        const float ie = pk.inv_zeta;
        Cls::template prim<float>(acc, F, pb.PAx, pb.PAy, pb.PAz, -roz * PQx, -roz * PQy, -roz * PQz,
                                  0.5f * pb.inv_zeta, roz, -(pb.bABx + pk.bABx) * ie, -(pb.bABy + pk.bABy) * ie,
                                  -(pb.bABz + pk.bABz) * ie, pb.zeta * ie, 0.5f * ie);
      }
    }
  } else {
    const PrimPair *bsrc = v.prim + offb;
    for (int ik = 0; ik < npk; ++ik) {
      const PrimPair pk = v.prim[offk + ik];
#pragma unroll prim_unroll(LA, LB, LC, LD)
      for (int ib = 0; ib < npb; ++ib) {
        const PrimPair pb = bsrc[ib];
        const double rs = rsqrt(pb.zeta + pk.zeta);
        const double inv_zpe = rs * rs;
        const double rho = pb.zeta * pk.zeta * inv_zpe;
        const double PQx = pb.Px - pk.Px, PQy = pb.Py - pk.Py, PQz = pb.Pz - pk.Pz;
        const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
        double F[LTOT + 1];
        boys_eval<LTOT, double>(F, T, pb.K * pk.K * rs, tab);
        const double roz = rho * pb.inv_zeta;
        const double ie = pk.inv_zeta;
        Cls::template prim<double>(acc, F, pb.PAx, pb.PAy, pb.PAz, -roz * PQx, -roz * PQy, -roz * PQz,
                                   0.5 * pb.inv_zeta, roz, -(pb.bABx + pk.bABx) * ie, -(pb.bABy + pk.bABy) * ie,
                                   -(pb.bABz + pk.bABz) * ie, pb.zeta * ie, 0.5 * ie);
      }
    }
  }
}

// Contracted (ab|cd) block of one shell quartet, bra pair `bp`, ket pair
// `kp`, components in canonical order, normalisation applied.  `npk` = 0
// yields an all-zero block (inactive lanes).  R is the arithmetic type
// (see accumulate_primitives).
template <int LA, int LB, int LC, int LD, bool REF, class R = double>
__device__ __forceinline__ void quartet_block(const EngineView &v, const double *tab, int bp, int kp, int npk, R *out,
                                              int lg = 0) {
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  using Cls = EriClass<LA, LB, LC, LD, REF>;
  R acc[Cls::kAcc];
#pragma unroll
  for (int x = 0; x < Cls::kAcc; ++x) acc[x] = R(0);
  accumulate_primitives<LA, LB, LC, LD, REF, R>(v, tab, bp, kp, npk, acc, lg);
  Cls::template hrr<R>(out, acc, R(v.pair_AB[3 * bp]), R(v.pair_AB[3 * bp + 1]), R(v.pair_AB[3 * bp + 2]),
                       R(v.pair_AB[3 * kp]), R(v.pair_AB[3 * kp + 1]), R(v.pair_AB[3 * kp + 2]));
  constexpr int U = kUnrollBlock<NA * NB * NC * ND>;
#pragma unroll U
  for (int a = 0; a < NA; ++a)
#pragma unroll U
    for (int b = 0; b < NB; ++b)
#pragma unroll U
      for (int c = 0; c < NC; ++c)
#pragma unroll U
        for (int d = 0; d < ND; ++d)
          out[((a * NB + b) * NC + c) * ND + d] *= R(comp_norm<LA>(a) * comp_norm<LB>(b) * comp_norm<LC>(c) *
                                                     comp_norm<LD>(d));
}

// Density-weighted Schwarz bound of the quartet (bp|kp): Q_ab Q_cd times the
// largest |D| over the six shell blocks a J/K digestion reads (ab, cd for J;
// ac, ad, bc, bd for K).
__device__ __forceinline__ float density_bound(const EngineView &v, int bp, int kp) {
  const int a = v.pair_sa[bp], b = v.pair_sb[bp], c = v.pair_sa[kp], d = v.pair_sb[kp];
  const float *S = v.shell_dmax;
  const int ns = v.nshells;
  const float m = fmaxf(fmaxf(fmaxf(S[a * ns + b], S[c * ns + d]), fmaxf(S[a * ns + c], S[a * ns + d])),
                        fmaxf(S[b * ns + c], S[b * ns + d]));
  return (float)(v.pair_Q[bp] * v.pair_Q[kp]) * m;
}

// Warp-level density screening of one task.  Sets *keep for the lane's
// quartet (active and bound >= threshold) and *fp64 for the task (the warp's
// largest kept bound reaches the mixed cutoff; always true for kScreenFp64),
// identically in every lane; returns false when no quartet is kept.  Counts
// the kept quartets per precision.
template <int SCR>
__device__ __forceinline__ bool screen_task(const EngineView &v, const ClassLaunch &cl, int bp, int kp, bool active,
                                            bool *keep, bool *fp64, bool leader = true) {
  const float bnd = active ? density_bound(v, bp, kp) : 0.0f;
  const bool k = active && bnd >= cl.dens_threshold;
  *keep = k;
  const unsigned kept = __ballot_sync(0xffffffffu, k);
  if (!kept) return false;
  bool hi = true;
  if constexpr (SCR == kScreenMixed) {
    float m = k ? bnd : 0.0f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    hi = m >= cl.mixed_cutoff;
  }
  *fp64 = hi;
  const unsigned counted = __ballot_sync(0xffffffffu, k && leader);  // one lane per quartet
  if ((threadIdx.x & 31) == 0 && cl.counters) atomicAdd(&cl.counters[hi ? 0 : 1], (unsigned long long)__popc(counted));
  return true;
}

// The reference evaluates each function quartet of a (dd|dd) shell quartet
// with the bra/ket orientation its SwapOrbitals picks from function IDs
// (IntegralsRepository.cpp:344-370); under the reference's electron-transfer
// row range the orientation changes the value.  This reproduces the choice
// per element (AO index == function ID).  Kept out of line: it holds three
// (dd|dd) blocks and is only reached by the rare two-d-shell quartets.
template <class R>
static __device__ __noinline__ void dddd_reference_values(const EngineView &v, const double *tab, int bp, int kp,
                                                          int npk, R *out) {
  constexpr int N = 6;
  const int sab = v.pair_sa[bp], skt = v.pair_sa[kp];
  if (sab > skt || npk == 0) {
    quartet_block<2, 2, 2, 2, true, R>(v, tab, bp, kp, npk, out);
    return;
  }
  R sw[N * N * N * N];
  quartet_block<2, 2, 2, 2, true, R>(v, tab, kp, bp, v.pair_nprim[bp], sw);
  if (sab < skt) {
    for (int a = 0; a < N; ++a)
      for (int b = 0; b < N; ++b)
        for (int c = 0; c < N; ++c)
          for (int d = 0; d < N; ++d) out[((a * N + b) * N + c) * N + d] = sw[((c * N + d) * N + a) * N + b];
    return;
  }
  // same first shell: per-element orientation
  quartet_block<2, 2, 2, 2, true, R>(v, tab, bp, kp, npk, out);
  const int aoa = v.pair_ao_a[bp], aob = v.pair_ao_b[bp], aoc = v.pair_ao_a[kp], aod = v.pair_ao_b[kp];
  const bool bdiag = v.pair_sa[bp] == v.pair_sb[bp], kdiag = v.pair_sa[kp] == v.pair_sb[kp];
  for (int a = 0; a < N; ++a)
    for (int b = 0; b < N; ++b)
      for (int c = 0; c < N; ++c)
        for (int d = 0; d < N; ++d) {
          const int I = aoa + a, J = aob + b, K = aoc + c, L = aod + d;
          const int o1 = bdiag ? max(I, J) : I, o2 = bdiag ? min(I, J) : J;
          const int o3 = kdiag ? max(K, L) : K, o4 = kdiag ? min(K, L) : L;
          const bool bra_first = o1 > o3 || (o1 == o3 && o2 >= o4);
          if (!bra_first) out[((a * N + b) * N + c) * N + d] = sw[((c * N + d) * N + a) * N + b];
        }
}

template <int LA, int LB, int LC, int LD, bool REF, class R>
__device__ __forceinline__ void quartet_values(const EngineView &v, const double *tab, int bp, int kp, int npk,
                                               R *out, int lg) {
  if constexpr (REF && LA == 2 && LB == 2 && LC == 2 && LD == 2) {
    dddd_reference_values<R>(v, tab, bp, kp, npk, out);  // single-quartet queries only: lg == 0
  } else {
    quartet_block<LA, LB, LC, LD, REF, R>(v, tab, bp, kp, npk, out, lg);
  }
}

// SCR (enum Screen) selects plain FP64, or a density-screened FP64 or mixed
// FP64/FP32 J/K build (kJkRhf, kJkUhf only).
template <int LA, int LB, int LC, int LD, int MODE, bool REF, int SCR = kScreenNone>
__global__ void __launch_bounds__(32 * fused_warps(LA, LB, LC, LD), fused_min_blocks(LA, LB, LC, LD))
    eri_class_kernel(const EngineView v, const ClassLaunch cl) {
  constexpr int kW = fused_warps(LA, LB, LC, LD);
  constexpr int LTOT = LA + LB + LC + LD;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int N = NA * NB * NC * ND;
  static_assert(SCR == kScreenNone || MODE == kJkRhf || MODE == kJkUhf, "screening applies to J/K builds");
  // the class's Boys slice: per-order rows in global memory, or staged
  __shared__ double tab_sh[boys_from_global(LA, LB, LC, LD) ? 1 : kBoysGrid * kBoysRow];
  const double *__restrict__ tab = tab_sh;
  if constexpr (boys_from_global(LA, LB, LC, LD)) {
    tab = v.boys_table + kBoysFoldedOff + LTOT * kBoysFoldedSize;
  } else {
    stage_boys<LTOT>(tab_sh, v.boys_table);
  }

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int ntasks = launch_ntasks(cl);
  // task_prefetch: the warp's next task record is loaded while it works on
  // this one (the task lists stream from DRAM once per build: a miss on
  // every task)
  constexpr bool kPrefetch = task_prefetch(LA, LB, LC, LD);
  int t = first_task(cl, blockIdx.x * kW + warp);
  Task task_next;
  if (kPrefetch && t < ntasks) task_next = launch_task(cl, t);
  for (int tn; t < ntasks; t = tn) {
    Task task;
    if constexpr (kPrefetch) {
      task = task_next;
      tn = next_task(cl, t, gridDim.x * kW);
      if (tn < ntasks) task_next = launch_task(cl, tn);
    } else {
      task = launch_task(cl, t);
      tn = next_task(cl, t, gridDim.x * kW);
    }
    const int bp = cl.bra_list[task.bra_pos];
    // the task's molecule (batched contexts): its matrices and size
    const MolView mv = task_molecule(v, bp);
    if (mv.skip) continue;  // warp-uniform: the warp shares the bra pair
    const int n = mv.n;
    const double *Da = cl.Da + mv.base, *Db = cl.Db ? cl.Db + mv.base : nullptr;
    const double *Dt = cl.Dt ? cl.Dt + mv.base : nullptr;
    double *Jm = cl.J ? cl.J + mv.base : nullptr, *Kam = cl.Ka ? cl.Ka + mv.base : nullptr;
    double *Kbm = cl.Kb ? cl.Kb + mv.base : nullptr;
    // 2^lg lanes per quartet (lg warp-uniform): lane group `lane >> lg`
    // takes that ket of the task, and only its first lane digests the result
    const int lg = task.lg;
    const int gl = lane & ((1 << lg) - 1);
    const int kpos = task.ket_start + (lane >> lg);
    bool active = kpos < task.ket_end;
    const int kp = active ? cl.ket_list[kpos] : bp;
    bool fp64 = true;
    if constexpr (SCR != kScreenNone) {
      bool keep;
      if (!screen_task<SCR>(v, cl, bp, kp, active, &keep, &fp64, gl == 0)) continue;  // warp-uniform
      active = keep;
    }
    const int npk = active ? v.pair_nprim[kp] : 0;

    double out[N];
    if (SCR != kScreenMixed || fp64) {
      quartet_values<LA, LB, LC, LD, REF, double>(v, tab, bp, kp, npk, out, lg);
    } else if constexpr (SCR == kScreenMixed) {
      // FP32 evaluation, FP64 from here on (digestion, accumulation)
      float o32[N];
      quartet_values<LA, LB, LC, LD, REF, float>(v, tab, bp, kp, npk, o32, lg);
#pragma unroll kUnrollBlock<N>
      for (int x = 0; x < N; ++x) out[x] = (double)o32[x];
    }
    active = active && gl == 0;
    // blocks above 81 integrals live in local memory anyway: keep their
    // epilogue loops rolled (code size, compile time)
    constexpr int U = kUnrollBlock<NA * NB * NC * ND>;

    const int aoa = v.pair_ao_a[bp], aob = v.pair_ao_b[bp], aoc = v.pair_ao_a[kp], aod = v.pair_ao_b[kp];
    const bool bdiag = v.pair_sa[bp] == v.pair_sb[bp], kdiag = v.pair_sa[kp] == v.pair_sb[kp];
    const bool same = bp == kp;

    if constexpr (MODE == kBlock) {
      // raw block of the first quartet (single-integral queries)
      if (t == 0 && lane == 0 && active)
        for (int x = 0; x < NA * NB * NC * ND; ++x) cl.packed[x] = out[x];
    } else if constexpr (MODE == kStorePacked) {
      if (active) {
#pragma unroll U
        for (int a = 0; a < NA; ++a)
#pragma unroll U
          for (int b = 0; b < NB; ++b)
#pragma unroll U
            for (int c = 0; c < NC; ++c)
#pragma unroll U
              for (int d = 0; d < ND; ++d) {
                const int I = aoa + a, J = aob + b, K = aoc + c, L = aod + d;
                if (bdiag && I < J) continue;
                if (kdiag && K < L) continue;
                const long long ij = tri(I, J), kl = tri(K, L);
                if (same && ij < kl) continue;
                cl.packed[tri(ij, kl)] = out[((a * NB + b) * NC + c) * ND + d];
              }
      }
    } else {
      // degeneracy of the unique quartet among its 8 permutations
      const double s = (bdiag ? 0.5 : 1.0) * (kdiag ? 0.5 : 1.0) * (same ? 0.5 : 1.0);
      constexpr bool kUhf = MODE == kJkUhf;
      const double *DJ = kUhf ? Dt : Da;
      double jab[NA * NB], jcd[NC * ND];
      double kac[NA * NC], kad[NA * ND], kbc[NB * NC], kbd[NB * ND];
      double kac2[kUhf ? NA * NC : 1], kad2[kUhf ? NA * ND : 1], kbc2[kUhf ? NB * NC : 1], kbd2[kUhf ? NB * ND : 1];
#pragma unroll U
      for (int x = 0; x < NA * NB; ++x) jab[x] = 0.0;
#pragma unroll U
      for (int x = 0; x < NC * ND; ++x) jcd[x] = 0.0;
#pragma unroll U
      for (int x = 0; x < NA * NC; ++x) kac[x] = 0.0;
#pragma unroll U
      for (int x = 0; x < NA * ND; ++x) kad[x] = 0.0;
#pragma unroll U
      for (int x = 0; x < NB * NC; ++x) kbc[x] = 0.0;
#pragma unroll U
      for (int x = 0; x < NB * ND; ++x) kbd[x] = 0.0;
      if constexpr (kUhf) {
#pragma unroll U
        for (int x = 0; x < NA * NC; ++x) kac2[x] = 0.0;
#pragma unroll U
        for (int x = 0; x < NA * ND; ++x) kad2[x] = 0.0;
#pragma unroll U
        for (int x = 0; x < NB * NC; ++x) kbc2[x] = 0.0;
#pragma unroll U
        for (int x = 0; x < NB * ND; ++x) kbd2[x] = 0.0;
      }
      if (active) {
#pragma unroll U
        for (int a = 0; a < NA; ++a)
#pragma unroll U
          for (int b = 0; b < NB; ++b)
#pragma unroll U
            for (int c = 0; c < NC; ++c)
#pragma unroll U
              for (int d = 0; d < ND; ++d) {
                const int I = aoa + a, J = aob + b, K = aoc + c, L = aod + d;
                const double val = s * out[((a * NB + b) * NC + c) * ND + d];
                jab[a * NB + b] += 2.0 * val * __ldg(&DJ[K * n + L]);
                jcd[c * ND + d] += 2.0 * val * __ldg(&DJ[I * n + J]);
                kac[a * NC + c] += val * __ldg(&Da[J * n + L]);
                kad[a * ND + d] += val * __ldg(&Da[J * n + K]);
                kbc[b * NC + c] += val * __ldg(&Da[I * n + L]);
                kbd[b * ND + d] += val * __ldg(&Da[I * n + K]);
                if constexpr (kUhf) {
                  kac2[a * NC + c] += val * __ldg(&Db[J * n + L]);
                  kad2[a * ND + d] += val * __ldg(&Db[J * n + K]);
                  kbc2[b * NC + c] += val * __ldg(&Db[I * n + L]);
                  kbd2[b * ND + d] += val * __ldg(&Db[I * n + K]);
                }
              }
#pragma unroll U
        for (int c = 0; c < NC; ++c)
#pragma unroll U
          for (int d = 0; d < ND; ++d) atomicAdd(&Jm[(aoc + c) * n + aod + d], jcd[c * ND + d]);
#pragma unroll U
        for (int a = 0; a < NA; ++a) {
#pragma unroll U
          for (int c = 0; c < NC; ++c) atomicAdd(&Kam[(aoa + a) * n + aoc + c], kac[a * NC + c]);
#pragma unroll U
          for (int d = 0; d < ND; ++d) atomicAdd(&Kam[(aoa + a) * n + aod + d], kad[a * ND + d]);
        }
#pragma unroll U
        for (int b = 0; b < NB; ++b) {
#pragma unroll U
          for (int c = 0; c < NC; ++c) atomicAdd(&Kam[(aob + b) * n + aoc + c], kbc[b * NC + c]);
#pragma unroll U
          for (int d = 0; d < ND; ++d) atomicAdd(&Kam[(aob + b) * n + aod + d], kbd[b * ND + d]);
        }
        if constexpr (kUhf) {
#pragma unroll U
          for (int a = 0; a < NA; ++a) {
#pragma unroll U
            for (int c = 0; c < NC; ++c) atomicAdd(&Kbm[(aoa + a) * n + aoc + c], kac2[a * NC + c]);
#pragma unroll U
            for (int d = 0; d < ND; ++d) atomicAdd(&Kbm[(aoa + a) * n + aod + d], kad2[a * ND + d]);
          }
#pragma unroll U
          for (int b = 0; b < NB; ++b) {
#pragma unroll U
            for (int c = 0; c < NC; ++c) atomicAdd(&Kbm[(aob + b) * n + aoc + c], kbc2[b * NC + c]);
#pragma unroll U
            for (int d = 0; d < ND; ++d) atomicAdd(&Kbm[(aob + b) * n + aod + d], kbd2[b * ND + d]);
          }
        }
      }
      // the warp shares the bra pair: reduce its J block across lanes first
#pragma unroll U
      for (int x = 0; x < NA * NB; ++x) {
        double r = jab[x];
#pragma unroll U
        for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
        jab[x] = r;
      }
      if (lane == 0) {
#pragma unroll U
        for (int a = 0; a < NA; ++a)
#pragma unroll U
          for (int b = 0; b < NB; ++b) atomicAdd(&Jm[(aoa + a) * n + aob + b], jab[a * NB + b]);
      }
    }
  }
}

// Schwarz bounds: thread per pair of the class, (ab|ab) with the exact
// recursion, Q = sqrt(max_ij |(ij|ij)|).
template <int LA, int LB>
__global__ void __launch_bounds__(kThreads) schwarz_kernel(const EngineView v, const int *pairs, int npairs,
                                                           double *Q) {
  constexpr int NA = ncart(LA), NB = ncart(LB);
  __shared__ double tab[kBoysGrid * kBoysRow];
  stage_boys<2 * (LA + LB)>(tab, v.boys_table);
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < npairs; x += gridDim.x * blockDim.x) {
    const int p = pairs[x];
    double out[NA * NB * NA * NB];
    quartet_block<LA, LB, LA, LB, false>(v, tab, p, p, v.pair_nprim[p], out);
    double m = 0.0;
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int b = 0; b < NB; ++b) m = fmax(m, fabs(out[((a * NB + b) * NA + a) * NB + b]));
    Q[p] = sqrt(m);
  }
}

// Host: launch one fused class kernel (block size per class).
template <int LA, int LB, int LC, int LD, int MODE, bool REF, int SCR = kScreenNone>
void launch_fused(const EngineView &v, const ClassLaunch &cl, int grid, cudaStream_t s) {
  eri_class_kernel<LA, LB, LC, LD, MODE, REF, SCR><<<grid, 32 * fused_warps(LA, LB, LC, LD), 0, s>>>(v, cl);
}

}  // namespace hfg
