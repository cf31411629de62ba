// Split path for the large classes (more than 100 integrals per shell
// quartet): the fused kernel's per-thread state (the contracted [e0|f0]
// block plus the full (ab|cd) block plus the J/K partials) does not fit the
// register file there and spills heavily.  Here
//   1. eri_prim_split_kernel: thread per shell quartet runs the primitive
//      loops (Boys, vertical recursion, electron transfer, contraction) and
//      streams the contracted [e0|f0] block to scratch, column-major across
//      the quartets of a chunk so that a warp's stores coalesce;
//   2. eri_hrr_digest_kernel: one block per task (32 quartets sharing the
//      bra pair); each warp expands bra rows (a b) of all 32 quartets with the
//      linear horizontal recursion (<= 4 terms per output), then stores them
//      (packed table) or digests them into J/K.
// Density-screened builds run step 1 twice (FP64 and FP32 halves, each
// taking its own tasks) and step 2 once over the quartets either kept.
#pragma once

#include "eri_kernels.cuh"
#include "eri_split_gen.cuh"

namespace hfg {

// contracted [e0|f0] of one shell quartet, written to scr[x * stride]
template <int LA, int LB, int LC, int LD, bool REF, class R>
__device__ __forceinline__ void prim_block_to_scratch(const EngineView &v, const double *tab, int bp, int kp, int npk,
                                                      double *scr, long long stride) {
  using Cls = EriClass<LA, LB, LC, LD, REF>;
  R acc[Cls::kAcc];
#pragma unroll
  for (int x = 0; x < Cls::kAcc; ++x) acc[x] = R(0);
  accumulate_primitives<LA, LB, LC, LD, REF, R>(v, tab, bp, kp, npk, acc);
#pragma unroll
  for (int x = 0; x < Cls::kAcc; ++x) scr[x * stride] = (double)acc[x];
}

// One quartet's contracted [e0|f0] block(s) in precision R, to its slot.
template <int LA, int LB, int LC, int LD, bool REF, class R>
__device__ __forceinline__ void prim_to_scratch(const EngineView &v, const double *tab, int bp, int kp,
                                                const SplitChunk &ch, long long slot) {
  constexpr bool kOrient = REF && LA == 2 && LB == 2 && LC == 2 && LD == 2;
  if constexpr (kOrient) {
    // bra/ket orientation the reference picks (see dddd_reference_values)
    const int sab = v.pair_sa[bp], skt = v.pair_sa[kp];
    if (sab >= skt)
      prim_block_to_scratch<LA, LB, LC, LD, true, R>(v, tab, bp, kp, v.pair_nprim[kp], ch.scr_fwd + slot, ch.stride);
    if (sab <= skt)
      prim_block_to_scratch<LA, LB, LC, LD, true, R>(v, tab, kp, bp, v.pair_nprim[bp], ch.scr_rev + slot, ch.stride);
  } else {
    prim_block_to_scratch<LA, LB, LC, LD, REF, R>(v, tab, bp, kp, v.pair_nprim[kp], ch.scr_fwd + slot, ch.stride);
  }
}

// SCR (enum Screen): plain FP64, density-screened FP64, or density-screened
// with the per-task FP64/FP32 choice.  A warp is one task (blockDim and the
// slot count are multiples of 32).
template <int LA, int LB, int LC, int LD, bool REF, int SCR = kScreenNone>
__global__ void __launch_bounds__(kThreads) eri_prim_split_kernel(const EngineView v, const ClassLaunch cl,
                                                                  const SplitChunk ch) {
  constexpr int LTOT = LA + LB + LC + LD;
  __shared__ double tab[kBoysGrid * kBoysRow];
  stage_boys<LTOT>(tab, v.boys_table);
  const long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (slot >= (long long)ch.ntasks * 32) return;  // whole warps
  const Task task = launch_task(cl, ch.task0 + (int)(slot >> 5));
  const int kpos = task.ket_start + (int)(slot & 31);
  bool active = kpos < task.ket_end;
  const int bp = cl.bra_list[task.bra_pos], kp = active ? cl.ket_list[kpos] : bp;
  bool fp64 = true;
  if constexpr (SCR != kScreenNone) {
    bool keep;
    if (!screen_task<SCR>(v, cl, bp, kp, active, &keep, &fp64)) return;  // warp-uniform
    active = keep;
  }
  if (!active) return;
  if constexpr (SCR == kScreenMixed) {
    if (!fp64) {
      prim_to_scratch<LA, LB, LC, LD, REF, float>(v, tab, bp, kp, ch, slot);
      return;
    }
  }
  prim_to_scratch<LA, LB, LC, LD, REF, double>(v, tab, bp, kp, ch, slot);
}

// Host: launch one primitive-split kernel.
template <int LA, int LB, int LC, int LD, bool REF, int SCR = kScreenNone>
void launch_prim_split(const EngineView &v, const ClassLaunch &cl, const SplitChunk &ch, int grid, cudaStream_t s) {
  eri_prim_split_kernel<LA, LB, LC, LD, REF, SCR><<<grid, kThreads, 0, s>>>(v, cl, ch);
}

// One block per task (32 quartets sharing the bra pair); warp w of the block
// expands rows ab = w, w + 4, ... of all 32 quartets.  The J_cd partials of a
// quartet accumulate in registers across a warp's rows and across the
// block's warps in shared memory before one atomic per element; J_ab reduces
// across the warp; the K partials go out per row.  SCREENED: only the
// quartets the density screening kept (the same test as step 1).
template <int LA, int LB, int LC, int LD, int MODE, bool REF, bool SCREENED = false>
__global__ void __launch_bounds__(kThreads) eri_hrr_digest_kernel(const EngineView v, const ClassLaunch cl,
                                                                  const SplitChunk ch) {
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int NAB = NA * NB, NCD = NC * ND;
  constexpr bool kOrient = REF && LA == 2 && LB == 2 && LC == 2 && LD == 2;
  constexpr bool kJk = MODE != kStorePacked;
  constexpr bool kUhf = MODE == kJkUhf;
  __shared__ double jcd_sh[kJk ? kWarpsPerBlock * 32 * NCD : 1];
  const int tloc = blockIdx.x;
  if (tloc >= ch.ntasks) return;  // whole block
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long slot = (long long)tloc * 32 + lane;
  const Task task = launch_task(cl, ch.task0 + tloc);
  const int kpos = task.ket_start + lane;
  bool active = kpos < task.ket_end;
  const int bp = cl.bra_list[task.bra_pos];
  const int kp = active ? cl.ket_list[kpos] : bp;
  if constexpr (SCREENED) {
    // every warp of the block sees the same task: block-uniform return
    active = active && density_bound(v, bp, kp) >= cl.dens_threshold;
    if (!__any_sync(0xffffffffu, active)) return;
  }
  const MolView mv = task_molecule(v, bp);
  if (mv.skip) return;  // block-uniform: one task per block
  const int n = mv.n;
  const double *Da = cl.Da + mv.base, *Db = cl.Db ? cl.Db + mv.base : nullptr;
  const double *Dt = cl.Dt ? cl.Dt + mv.base : nullptr;
  double *Jm = cl.J ? cl.J + mv.base : nullptr, *Kam = cl.Ka ? cl.Ka + mv.base : nullptr;
  double *Kbm = cl.Kb ? cl.Kb + mv.base : nullptr;
  const double X0 = v.pair_AB[3 * bp], X1 = v.pair_AB[3 * bp + 1], X2 = v.pair_AB[3 * bp + 2];
  const double Y0 = v.pair_AB[3 * kp], Y1 = v.pair_AB[3 * kp + 1], Y2 = v.pair_AB[3 * kp + 2];
  const int aoa = v.pair_ao_a[bp], aob = v.pair_ao_b[bp], aoc = v.pair_ao_a[kp], aod = v.pair_ao_b[kp];
  const bool bdiag = v.pair_sa[bp] == v.pair_sb[bp], kdiag = v.pair_sa[kp] == v.pair_sb[kp];
  const bool same = bp == kp;
  const double s = (bdiag ? 0.5 : 1.0) * (kdiag ? 0.5 : 1.0) * (same ? 0.5 : 1.0);
  const double *DJ = kUhf ? Dt : Da;

  double jcd[kJk ? NCD : 1];
#pragma unroll
  for (int x = 0; x < (kJk ? NCD : 1); ++x) jcd[x] = 0.0;

  for (int ab = warp; ab < NAB; ab += kWarpsPerBlock) {
    const int a = ab / NB, b = ab - a * NB;
    const int I = aoa + a, J = aob + b;
    double out[NCD];
#pragma unroll
    for (int x = 0; x < NCD; ++x) out[x] = 0.0;
    if (active) {
      if constexpr (kOrient) {
        const int sab = v.pair_sa[bp], skt = v.pair_sa[kp];
        if (sab > skt) {
          EriRows<LA, LB, LC, LD>::template row<double>(out, ab, ch.scr_fwd + slot, ch.stride, X0, X1, X2, Y0, Y1,
                                                        Y2);
        } else if (sab < skt) {
          EriRows<LA, LB, LC, LD>::template col<double>(out, ab, ch.scr_rev + slot, ch.stride, Y0, Y1, Y2, X0, X1,
                                                        X2);
        } else {
          double sw[NCD];
          EriRows<LA, LB, LC, LD>::template row<double>(out, ab, ch.scr_fwd + slot, ch.stride, X0, X1, X2, Y0, Y1,
                                                        Y2);
          EriRows<LA, LB, LC, LD>::template col<double>(sw, ab, ch.scr_rev + slot, ch.stride, Y0, Y1, Y2, X0, X1,
                                                        X2);
          const int o1 = bdiag ? max(I, J) : I, o2 = bdiag ? min(I, J) : J;
#pragma unroll
          for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int d = 0; d < ND; ++d) {
              const int K = aoc + c, L = aod + d;
              const int o3 = kdiag ? max(K, L) : K, o4 = kdiag ? min(K, L) : L;
              if (!(o1 > o3 || (o1 == o3 && o2 >= o4))) out[c * ND + d] = sw[c * ND + d];
            }
        }
      } else {
        EriRows<LA, LB, LC, LD>::template row<double>(out, ab, ch.scr_fwd + slot, ch.stride, X0, X1, X2, Y0, Y1, Y2);
      }
      const double nab = comp_norm<LA>(a) * comp_norm<LB>(b);
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int d = 0; d < ND; ++d) out[c * ND + d] *= nab * comp_norm<LC>(c) * comp_norm<LD>(d);
    }

    if constexpr (!kJk) {
      if (active && !(bdiag && I < J)) {
        const long long ij = tri(I, J);
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            const int K = aoc + c, L = aod + d;
            if (kdiag && K < L) continue;
            const long long kl = tri(K, L);
            if (same && ij < kl) continue;
            cl.packed[tri(ij, kl)] = out[c * ND + d];
          }
      }
    } else {
      double jab = 0.0;
      if (active) {
        const double dij = 2.0 * s * __ldg(&DJ[I * n + J]);
        double kac[NC], kbc[NC], kad[ND], kbd[ND];
        double kac2[kUhf ? NC : 1], kbc2[kUhf ? NC : 1], kad2[kUhf ? ND : 1], kbd2[kUhf ? ND : 1];
#pragma unroll
        for (int c = 0; c < NC; ++c) kac[c] = kbc[c] = 0.0;
#pragma unroll
        for (int d = 0; d < ND; ++d) kad[d] = kbd[d] = 0.0;
        if constexpr (kUhf) {
#pragma unroll
          for (int c = 0; c < NC; ++c) kac2[c] = kbc2[c] = 0.0;
#pragma unroll
          for (int d = 0; d < ND; ++d) kad2[d] = kbd2[d] = 0.0;
        }
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            const int K = aoc + c, L = aod + d;
            const double val = s * out[c * ND + d];
            jab += 2.0 * val * __ldg(&DJ[K * n + L]);
            jcd[c * ND + d] += dij * out[c * ND + d];
            kac[c] += val * __ldg(&Da[J * n + L]);
            kad[d] += val * __ldg(&Da[J * n + K]);
            kbc[c] += val * __ldg(&Da[I * n + L]);
            kbd[d] += val * __ldg(&Da[I * n + K]);
            if constexpr (kUhf) {
              kac2[c] += val * __ldg(&Db[J * n + L]);
              kad2[d] += val * __ldg(&Db[J * n + K]);
              kbc2[c] += val * __ldg(&Db[I * n + L]);
              kbd2[d] += val * __ldg(&Db[I * n + K]);
            }
          }
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          atomicAdd(&Kam[I * n + aoc + c], kac[c]);
          atomicAdd(&Kam[J * n + aoc + c], kbc[c]);
          if constexpr (kUhf) {
            atomicAdd(&Kbm[I * n + aoc + c], kac2[c]);
            atomicAdd(&Kbm[J * n + aoc + c], kbc2[c]);
          }
        }
#pragma unroll
        for (int d = 0; d < ND; ++d) {
          atomicAdd(&Kam[I * n + aod + d], kad[d]);
          atomicAdd(&Kam[J * n + aod + d], kbd[d]);
          if constexpr (kUhf) {
            atomicAdd(&Kbm[I * n + aod + d], kad2[d]);
            atomicAdd(&Kbm[J * n + aod + d], kbd2[d]);
          }
        }
      }
      // the warp's 32 quartets share the bra pair and this (a b) row
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) jab += __shfl_xor_sync(0xffffffffu, jab, o);
      if (lane == 0) atomicAdd(&Jm[I * n + J], jab);
    }
  }

  if constexpr (kJk) {
    // sum the J_cd partials of the block's warps, one atomic per element
#pragma unroll
    for (int x = 0; x < NCD; ++x) jcd_sh[(warp * NCD + x) * 32 + lane] = jcd[x];
    __syncthreads();
    if (active) {
      for (int x = warp; x < NCD; x += kWarpsPerBlock) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kWarpsPerBlock; ++w) t += jcd_sh[(w * NCD + x) * 32 + lane];
        const int c = x / ND, d = x - c * ND;
        atomicAdd(&Jm[(aoc + c) * n + aod + d], t);
      }
    }
  }
}

}  // namespace hfg
