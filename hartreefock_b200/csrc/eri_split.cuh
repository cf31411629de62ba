// Split path for the large classes (more than 100 integrals per shell
// quartet): the fused kernel's per-thread state (the contracted [e0|f0]
// block plus the full (ab|cd) block plus the J/K partials) does not fit the
// register file there and spills heavily.  Here
//   1. eri_prim_split_kernel: thread per shell quartet runs the primitive
//      loops (Boys, vertical recursion, electron transfer, contraction) and
//      streams the contracted [e0|f0] block to scratch, column-major across
//      the quartets of a chunk so that a warp's stores coalesce;
//   2. one block per task (32 quartets sharing the bra pair); warps expand
//      bra rows (a b) of all 32 quartets with the linear horizontal recursion
//      (<= 4 terms per output), then store them (packed table,
//      eri_hrr_store_kernel) or digest them into J/K (eri_hrr_jk_kernel).
// Density-screened builds run step 1 twice (FP64 and FP32 halves, each
// taking its own tasks) and step 2 once over the quartets either kept.
#pragma once

#include <atomic>

#include "eri_kernels.cuh"
#include "eri_split_gen.cuh"

namespace hfg {

// contracted [e0|f0] of one shell quartet, written to scr[x * stride]
// (accumulating in place in scratch instead of registers removes the
// spills of the large blocks but made the classes 1.3-2x slower: global
// read-modify-writes per primitive quartet cost more than local-memory
// spills, which stay in L1)
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
  __shared__ double tab_sh[boys_from_global_split(LA, LB, LC, LD) ? 1 : kBoysGrid * kBoysRow];
  const double *__restrict__ tab = tab_sh;
  if constexpr (boys_from_global_split(LA, LB, LC, LD)) {
    tab = v.boys_table + kBoysFoldedOff + LTOT * kBoysFoldedSize;
  } else {
    stage_boys<LTOT>(tab_sh, v.boys_table);
  }
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

// Row (a b) of one quartet's normalised (ab|cd) block from its contracted
// [e0|f0] block(s) in scratch (slot `slot` of the chunk): the linear
// horizontal recursion, for the reference's (dd|dd) convention in the
// orientation the reference picks per element (see dddd_reference_values).
template <int LA, int LB, int LC, int LD, bool REF>
__device__ __forceinline__ void split_row(double *out, int ab, const EngineView &v, const SplitChunk &ch,
                                          long long slot, int bp, int kp, double X0, double X1, double X2,
                                          double Y0, double Y1, double Y2) {
  constexpr int NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int NCD = NC * ND;
  constexpr bool kOrient = REF && LA == 2 && LB == 2 && LC == 2 && LD == 2;
  const int a = ab / NB, b = ab - a * NB;
  if constexpr (kOrient) {
    const int sab = v.pair_sa[bp], skt = v.pair_sa[kp];
    if (sab > skt) {
      EriRows<LA, LB, LC, LD>::template row<double>(out, ab, ch.scr_fwd + slot, ch.stride, X0, X1, X2, Y0, Y1, Y2);
    } else if (sab < skt) {
      EriRows<LA, LB, LC, LD>::template col<double>(out, ab, ch.scr_rev + slot, ch.stride, Y0, Y1, Y2, X0, X1, X2);
    } else {
      double sw[NCD];
      EriRows<LA, LB, LC, LD>::template row<double>(out, ab, ch.scr_fwd + slot, ch.stride, X0, X1, X2, Y0, Y1, Y2);
      EriRows<LA, LB, LC, LD>::template col<double>(sw, ab, ch.scr_rev + slot, ch.stride, Y0, Y1, Y2, X0, X1, X2);
      const bool bdiag = v.pair_sa[bp] == v.pair_sb[bp], kdiag = v.pair_sa[kp] == v.pair_sb[kp];
      const int I = v.pair_ao_a[bp] + a, J = v.pair_ao_b[bp] + b;
      const int aoc = v.pair_ao_a[kp], aod = v.pair_ao_b[kp];
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

// Stored-table mode: one block per task (32 quartets sharing the bra pair);
// warp w of the block expands rows ab = w, w + 4, ... of all 32 quartets
// and writes the 8-fold-unique elements to the packed table.
template <int LA, int LB, int LC, int LD, bool REF>
__global__ void __launch_bounds__(kThreads) eri_hrr_store_kernel(const EngineView v, const ClassLaunch cl,
                                                                 const SplitChunk ch) {
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int NAB = NA * NB, NCD = NC * ND;
  const int tloc = blockIdx.x;
  if (tloc >= ch.ntasks) return;  // whole block
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long slot = (long long)tloc * 32 + lane;
  const Task task = launch_task(cl, ch.task0 + tloc);
  const int kpos = task.ket_start + lane;
  if (kpos >= task.ket_end) return;  // no barrier below
  const int bp = cl.bra_list[task.bra_pos];
  const int kp = cl.ket_list[kpos];
  const double X0 = v.pair_AB[3 * bp], X1 = v.pair_AB[3 * bp + 1], X2 = v.pair_AB[3 * bp + 2];
  const double Y0 = v.pair_AB[3 * kp], Y1 = v.pair_AB[3 * kp + 1], Y2 = v.pair_AB[3 * kp + 2];
  const int aoa = v.pair_ao_a[bp], aob = v.pair_ao_b[bp], aoc = v.pair_ao_a[kp], aod = v.pair_ao_b[kp];
  const bool bdiag = v.pair_sa[bp] == v.pair_sb[bp], kdiag = v.pair_sa[kp] == v.pair_sb[kp];
  const bool same = bp == kp;
  for (int ab = warp; ab < NAB; ab += kWarpsPerBlock) {
    const int a = ab / NB, b = ab - a * NB;
    const int I = aoa + a, J = aob + b;
    if (bdiag && I < J) continue;
    double out[NCD];
    split_row<LA, LB, LC, LD, REF>(out, ab, v, ch, slot, bp, kp, X0, X1, X2, Y0, Y1, Y2);
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
}

// J/K digestion of one task, tiled over the bra rows.  The block has NB warps
// (one per bra component b); warp w owns the bra components a = w, w + NB, ...
// (NA / NB of them) and walks b = (w + s) mod NB in steps s = 0 .. NB-1, so
// that in every step the block's warps hold distinct b.  Per row (a b) and
// lane (ket quartet):
//   J_ab  warp sum -> one atomic per row;
//   J_cd  the warp's own shared-memory slots, summed over the warps at the
//         end -> one atomic per (c d);
//   K_ac, K_ad  registers over b -> NC + ND atomics per a;
//   K_bc, K_bd  shared-memory slots per b, summed over a across the steps
//         (one warp per slot per step, a block barrier between steps) ->
//         NC + ND atomics per b.
// Global atomics per quartet: NCD + (NA + NB)(NC + ND) + NAB / 32, against
// NCD + 2 NAB (NC + ND) + NAB / 32 when every row sends its own K partials.
// The density entries the K terms need -- D[I][ket c, d] and D[J][ket c, d]
// -- are read once per row or step into registers (a ket shell's AO indices
// are contiguous), not once per integral.
template <int LA, int LB, int LC, int LD, int MODE>
__host__ __device__ constexpr int jk_tile_doubles() {
  constexpr int NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  return ((MODE == kJkUhf ? 2 : 1) * NB * (NC + ND) + NB * NC * ND) * 32;
}

// at least 12 warps per SM: <= 170 registers per thread
__host__ __device__ constexpr int jk_min_blocks(int LB) { return ncart(LB) >= 6 ? 2 : 4; }

template <int LA, int LB, int LC, int LD, int MODE, bool REF, bool SCREENED = false>
__global__ void __launch_bounds__(32 * ncart(LB), jk_min_blocks(LB))
    eri_hrr_jk_kernel(const EngineView v, const ClassLaunch cl, const SplitChunk ch) {
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int NCD = NC * ND, NK = NC + ND;
  constexpr int APW = NA / NB;  // bra components a per warp
  static_assert(NA % NB == 0, "bra components a split evenly over the warps");
  static_assert(MODE == kJkRhf || MODE == kJkUhf, "J/K builds only");
  constexpr bool kUhf = MODE == kJkUhf;
  constexpr int NS = kUhf ? 2 : 1;  // spins with K matrices
  // K_bc / K_bd slots [spin][b][c or d][lane], then J_cd [warp][cd][lane]
  extern __shared__ double tile_sh[];
  double *kb_sh = tile_sh;
  double *jcd_sh = tile_sh + NS * NB * NK * 32;
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
  const double *Dm[2] = {cl.Da + mv.base, kUhf ? cl.Db + mv.base : nullptr};
  const double *DJ = kUhf ? cl.Dt + mv.base : Dm[0];
  double *Jm = cl.J + mv.base;
  double *Km[2] = {cl.Ka + mv.base, kUhf ? cl.Kb + mv.base : nullptr};
  const double X0 = v.pair_AB[3 * bp], X1 = v.pair_AB[3 * bp + 1], X2 = v.pair_AB[3 * bp + 2];
  const double Y0 = v.pair_AB[3 * kp], Y1 = v.pair_AB[3 * kp + 1], Y2 = v.pair_AB[3 * kp + 2];
  const int aoa = v.pair_ao_a[bp], aob = v.pair_ao_b[bp], aoc = v.pair_ao_a[kp], aod = v.pair_ao_b[kp];
  const bool bdiag = v.pair_sa[bp] == v.pair_sb[bp], kdiag = v.pair_sa[kp] == v.pair_sb[kp];
  const bool same = bp == kp;
  const double s = (bdiag ? 0.5 : 1.0) * (kdiag ? 0.5 : 1.0) * (same ? 0.5 : 1.0);

  for (int x = threadIdx.x; x < jk_tile_doubles<LA, LB, LC, LD, MODE>(); x += blockDim.x) tile_sh[x] = 0.0;
  double *jcd_w = jcd_sh + warp * NCD * 32 + lane;  // this warp's J_cd slots
  double kac[NS][APW][NC], kad[NS][APW][ND];
#pragma unroll
  for (int sp = 0; sp < NS; ++sp)
#pragma unroll
    for (int k = 0; k < APW; ++k) {
#pragma unroll
      for (int c = 0; c < NC; ++c) kac[sp][k][c] = 0.0;
#pragma unroll
      for (int d = 0; d < ND; ++d) kad[sp][k][d] = 0.0;
    }
  __syncthreads();

  for (int st = 0; st < NB; ++st) {
    const int b = (warp + st) % NB;
    const int J = aob + b;
    double kbc[NS][NC], kbd[NS][ND];
#pragma unroll
    for (int sp = 0; sp < NS; ++sp) {
#pragma unroll
      for (int c = 0; c < NC; ++c) kbc[sp][c] = 0.0;
#pragma unroll
      for (int d = 0; d < ND; ++d) kbd[sp][d] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < APW; ++k) {
      const int a = warp + k * NB, ab = a * NB + b;
      const int I = aoa + a;
      double jab = 0.0;
      if (active) {
        double out[NCD];
        split_row<LA, LB, LC, LD, REF>(out, ab, v, ch, slot, bp, kp, X0, X1, X2, Y0, Y1, Y2);
        const double dij = 2.0 * s * __ldg(&DJ[I * n + J]);
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            const double o = out[c * ND + d];
            jab += o * __ldg(&DJ[(aoc + c) * n + aod + d]);
            jcd_w[(c * ND + d) * 32] += dij * o;
          }
        jab *= 2.0 * s;
#pragma unroll
        for (int sp = 0; sp < NS; ++sp) {
          double dic[NC], did[ND], djc[NC], djd[ND];
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            dic[c] = __ldg(&Dm[sp][I * n + aoc + c]);
            djc[c] = __ldg(&Dm[sp][J * n + aoc + c]);
          }
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            did[d] = __ldg(&Dm[sp][I * n + aod + d]);
            djd[d] = __ldg(&Dm[sp][J * n + aod + d]);
          }
#pragma unroll
          for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int d = 0; d < ND; ++d) {
              const double val = s * out[c * ND + d];
              kac[sp][k][c] += val * djd[d];  // K_IK += (IJ|KL) D_JL
              kad[sp][k][d] += val * djc[c];  // K_IL += (IJ|KL) D_JK
              kbc[sp][c] += val * did[d];     // K_JK += (IJ|KL) D_IL
              kbd[sp][d] += val * dic[c];     // K_JL += (IJ|KL) D_IK
            }
        }
      }
      // the warp's 32 quartets share the bra pair and this (a b) row
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) jab += __shfl_xor_sync(0xffffffffu, jab, o);
      if (lane == 0 && jab != 0.0) atomicAdd(&Jm[I * n + J], jab);
    }
    // this step's b slot belongs to this warp alone
#pragma unroll
    for (int sp = 0; sp < NS; ++sp) {
      double *slotb = kb_sh + ((sp * NB + b) * NK) * 32 + lane;
#pragma unroll
      for (int c = 0; c < NC; ++c) slotb[c * 32] += kbc[sp][c];
#pragma unroll
      for (int d = 0; d < ND; ++d) slotb[(NC + d) * 32] += kbd[sp][d];
    }
    __syncthreads();
  }
  if (active) {
#pragma unroll
    for (int sp = 0; sp < NS; ++sp)
#pragma unroll
      for (int k = 0; k < APW; ++k) {
        const int I = aoa + warp + k * NB;
#pragma unroll
        for (int c = 0; c < NC; ++c) atomicAdd(&Km[sp][I * n + aoc + c], kac[sp][k][c]);
#pragma unroll
        for (int d = 0; d < ND; ++d) atomicAdd(&Km[sp][I * n + aod + d], kad[sp][k][d]);
      }
    for (int x = warp; x < NCD; x += NB) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < NB; ++w) t += jcd_sh[(w * NCD + x) * 32 + lane];
      const int c = x / ND, d = x - c * ND;
      atomicAdd(&Jm[(aoc + c) * n + aod + d], t);
    }
    for (int x = warp; x < NS * NB * NK; x += NB) {
      const int sp = x / (NB * NK), r = x - sp * NB * NK, b = r / NK, e = r - b * NK;
      const int col = e < NC ? aoc + e : aod + (e - NC);
      atomicAdd(&Km[sp][(aob + b) * n + col], kb_sh[x * 32 + lane]);
    }
  }
}

// Host: launch the tiled J/K digestion (NB warps per block, one block per
// task, the tile in dynamic shared memory; the first launch of each
// instantiation raises its shared-memory limit).
template <int LA, int LB, int LC, int LD, int MODE, bool REF, bool SCREENED = false>
void launch_hrr_jk(const EngineView &v, const ClassLaunch &cl, const SplitChunk &ch, int grid, cudaStream_t s) {
  constexpr size_t bytes = sizeof(double) * jk_tile_doubles<LA, LB, LC, LD, MODE>();
  if constexpr (bytes > 48 * 1024) {
    static std::atomic<unsigned> sized{0};  // one bit per device
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned bit = 1u << (dev & 31);
    if (!(sized.load() & bit)) {
      cudaFuncSetAttribute(eri_hrr_jk_kernel<LA, LB, LC, LD, MODE, REF, SCREENED>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
      sized.fetch_or(bit);
    }
  }
  eri_hrr_jk_kernel<LA, LB, LC, LD, MODE, REF, SCREENED><<<grid, 32 * ncart(LB), bytes, s>>>(v, cl, ch);
}

}  // namespace hfg
