// Warp-cooperative kernel for the large classes (more than 100 integrals per
// shell quartet: (dp|ds), (dd|ps), (dp|pp), (dp|dp), (dd|pp), (dd|ds),
// (dd|dp), (dd|dd)).  A thread per shell quartet cannot hold these classes'
// recursion intermediates in registers (the per-thread kernels spilled up to
// 38 KB per thread), so here one warp evaluates one shell quartet:
//
//   1. primitive quartets one after another; per primitive quartet every lane
//      forms the same prefactors and Boys values (FP64, from the global
//      table), then the lanes run the class's vertical-recursion and
//      electron-transfer program (WarpProg, generated) level by level on
//      intermediates in shared memory, and add the [e0|f0] entries they own
//      to register accumulators (the contraction);
//   2. the contracted [e0|f0] block goes to shared memory and the lanes
//      expand bra rows (a b) of the (ab|cd) block with the row-wise
//      horizontal recursion (EriRows), normalised, into a shared block;
//   3. the lanes digest the block: every element of J_ab, J_cd, K_ac, K_ad,
//      K_bc, K_bd is one lane's dot product over the block, then one atomic
//      (or the packed-table store).
//
// Work units are single quartets: unit u of a launch is ket u % 32 of task
// u / 32 (units past a task's last ket are skipped), walked grid-stride by
// the warps, so a class with few large quartets still spreads over every SM.
// Nothing is written to global memory but the outputs: no scratch.
#pragma once

#include "eri_kernels.cuh"
#include "eri_split_gen.cuh"
#include "eri_warp_gen.cuh"

namespace hfg {

// Boys function F_0..F_M at T from the global FP64 table
// (g[i * kBoysOrders + m] = F_m(T_i), tail g[kBoysGrid * kBoysOrders + i] =
// e^-T_i): the expansion and recursions of boys_eval, without the staged
// shared-memory slice (one evaluation per primitive quartet per warp).
template <int M>
__device__ __forceinline__ void boys_global(double *F, double T, double scale, const double *__restrict__ g) {
  if (T < kBoysTmax) {
    const BoysGridPoint gp = boys_grid_point(T);
    const int i = gp.i;
    const double dt = gp.dt;
    const double *t = g + i * kBoysOrders + M;
    // sum_k F_{M+k}(T_i) dt^k / k!, k < 7, nested as F_M + dt (F_{M+1} + dt/2 (F_{M+2} + ...))
    double f = __ldg(t + 6);
#pragma unroll
    for (int k = 6; k >= 1; --k) f = fma(f, dt * (1.0 / k), __ldg(t + k - 1));
    double fm[M + 1];
    fm[M] = f;
    if (M > 0) {
      double x = 1.0 / 5040.0;
      x = fma(x, dt, 1.0 / 720.0);
      x = fma(x, dt, 1.0 / 120.0);
      x = fma(x, dt, 1.0 / 24.0);
      x = fma(x, dt, 1.0 / 6.0);
      x = fma(x, dt, 0.5);
      x = fma(x, dt, 1.0);
      x = fma(x, dt, 1.0);
      const double e = __ldg(g + kBoysGrid * kBoysOrders + i) * x;
      const double t2 = 2.0 * T;
#pragma unroll
      for (int m = M - 1; m >= 0; --m) fm[m] = fma(t2, fm[m + 1], e) * (1.0 / (2 * m + 1));
    }
#pragma unroll
    for (int m = 0; m <= M; ++m) F[m] = fm[m] * scale;
  } else {
    const double r = rsqrt(T);
    double f = 0.88622692545275801365 * r;
    F[0] = f * scale;
    if (M > 0) {
      const double e = exp_neg_far(T), h = 0.5 * r * r;
#pragma unroll
      for (int m = 0; m < M; ++m) {
        f = ((2 * m + 1) * f - e) * h;
        F[m + 1] = f * scale;
      }
    }
  }
}

// Shared-memory footprint of one warp, in bytes: the program's slots and the
// contracted block(s) in R, the normalised (ab|cd) block in FP64 with rows
// padded to an odd length (conflict-free column reads).
template <int LA, int LB, int LC, int LD, bool REF>
struct WarpShape {
  using P = WarpProg<LA, LB, LC, LD, REF>;
  static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  static constexpr int NAB = NA * NB, NCD = NC * ND, NCDP = NCD | 1;
  static constexpr bool kOrient = REF && LA == 2 && LB == 2 && LC == 2 && LD == 2;
  static constexpr int kAccRegs = (P::kAcc + 31) / 32;
  // R-typed part sized for FP64 (the mixed kernel runs both precisions)
  static constexpr int kWork = P::kSlots;
  static constexpr int kAccs = P::kAcc * (kOrient ? 2 : 1);
  static constexpr int kRDoubles = (kWork + kAccs + 1) & ~1;
  static constexpr int kBytes = (kRDoubles + NAB * NCDP) * 8;
  // warps per block: keep a block near a third of the SM's shared memory
  static constexpr int kWarps = kBytes * 8 <= 72 * 1024 ? 8 : kBytes * 4 <= 72 * 1024 ? 4 : kBytes * 2 <= 80 * 1024 ? 2 : 1;
};

// Contracted [e0|f0] block of the quartet (bra pair bp, ket pair kp) in
// precision R, into acc_sh[x] (x = e * NF + f).  Every lane of the warp takes
// part; w is the warp's slot array (w[0] == 0).
template <int LA, int LB, int LC, int LD, bool REF, class R>
__device__ __forceinline__ void warp_contract(const EngineView &v, int bp, int kp, R *w, R *acc_sh) {
  using P = WarpProg<LA, LB, LC, LD, REF>;
  using S = WarpShape<LA, LB, LC, LD, REF>;
  constexpr int LTOT = LA + LB + LC + LD;
  const int lane = threadIdx.x & 31;
  R racc[S::kAccRegs];
#pragma unroll
  for (int j = 0; j < S::kAccRegs; ++j) racc[j] = R(0);
  const uint4 *__restrict__ ops = P::ops();
  const uint16_t *__restrict__ accmap = P::acc();
  const int offb = v.pair_prim_off[bp], npb = v.pair_nprim[bp];
  const int offk = v.pair_prim_off[kp], npk = v.pair_nprim[kp];
  // slot 0 reads as zero (absent operands); rewritten per quartet because
  // the FP32 and FP64 views of the slots overlap
  if (lane == 0) w[0] = R(0);
  for (int ik = 0; ik < npk; ++ik) {
    const PrimPair pk = v.prim[offk + ik];
    for (int ib = 0; ib < npb; ++ib) {
      const PrimPair pb = v.prim[offb + ib];
      // prefactors and Boys values: the same in every lane (broadcast loads)
      const double rs = rsqrt(pb.zeta + pk.zeta);
      const double rho = pb.zeta * pk.zeta * (rs * rs);
      const double PQx = pb.Px - pk.Px, PQy = pb.Py - pk.Py, PQz = pb.Pz - pk.Pz;
      const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
      double F[LTOT + 1];
      boys_global<LTOT>(F, T, pb.K * pk.K * rs, v.boys_table);
      const double roz = rho * pb.inv_zeta, ie = pk.inv_zeta;
      const R PA0 = R(pb.PAx), PA1 = R(pb.PAy), PA2 = R(pb.PAz);
      const R WP0 = R(-roz * PQx), WP1 = R(-roz * PQy), WP2 = R(-roz * PQz);
      const R oo2z = R(0.5 * pb.inv_zeta), mroz = R(-roz);
      const R DL0 = R(-(pb.bABx + pk.bABx) * ie), DL1 = R(-(pb.bABy + pk.bABy) * ie), DL2 = R(-(pb.bABz + pk.bABz) * ie);
      const R mzoe = R(-pb.zeta * ie), oo2e = R(0.5 * ie);
#pragma unroll
      for (int m = 0; m <= LTOT; ++m)
        if (lane == m) w[P::fslot(m)] = R(F[m]);
      __syncwarp();
#pragma unroll
      for (int l = 1; l <= P::kLevels; ++l) {
#pragma unroll 2
        for (int k = P::bound(l - 1) + lane; k < P::bound(l); k += 32) {
          const uint4 op = __ldg(&ops[k]);
          const unsigned x = op.x;
          const int dir = (x >> 16) & 3;
          const bool et = (x >> 18) & 1;
          const R n1 = R((x >> 20) & 15), n2 = R((x >> 24) & 15);
          const R a = w[op.y & 0xffff], b = w[op.y >> 16], c = w[op.z & 0xffff], d = w[op.z >> 16];
          const R pa = dir == 0 ? PA0 : dir == 1 ? PA1 : PA2;
          const R wp = dir == 0 ? WP0 : dir == 1 ? WP1 : WP2;
          const R dl = dir == 0 ? DL0 : dir == 1 ? DL1 : DL2;
          // vertical: PA a + WP b + n1 oo2z (c - roz d)
          // transfer: delta a - zoe b + oo2e (n1 c + n2 d)
          // (the class kernels' association: the pair difference is formed
          // before its prefactor, so near-cancelling terms keep their bits)
          const R c1 = et ? dl : pa;
          const R c2 = et ? mzoe : wp;
          const R c3 = et ? oo2e : n1 * oo2z;
          const R t = (et ? n1 : R(1)) * c + (et ? n2 : mroz) * d;
          w[x & 0xffff] = c1 * a + c2 * b + c3 * t;
        }
        __syncwarp();
      }
#pragma unroll
      for (int j = 0; j < S::kAccRegs; ++j) {
        const int xi = lane + 32 * j;
        if (xi < P::kAcc) racc[j] += w[__ldg(&accmap[xi])];
      }
      __syncwarp();  // the next primitive quartet overwrites the slots
    }
  }
#pragma unroll
  for (int j = 0; j < S::kAccRegs; ++j) {
    const int xi = lane + 32 * j;
    if (xi < P::kAcc) acc_sh[xi] = racc[j];
  }
  __syncwarp();
}

// The normalised (ab|cd) block of the quartet into o[ab * NCDP + cd] (FP64),
// with the reference's per-element bra/ket orientation for its (dd|dd)
// convention (see dddd_reference_values).
template <int LA, int LB, int LC, int LD, bool REF, class R>
__device__ __forceinline__ void warp_block(const EngineView &v, int bp, int kp, R *w, R *acc_sh, double *o) {
  using S = WarpShape<LA, LB, LC, LD, REF>;
  constexpr int NB = S::NB, NC = S::NC, ND = S::ND, NCD = S::NCD, NCDP = S::NCDP;
  const int lane = threadIdx.x & 31;
  const R X0 = R(v.pair_AB[3 * bp]), X1 = R(v.pair_AB[3 * bp + 1]), X2 = R(v.pair_AB[3 * bp + 2]);
  const R Y0 = R(v.pair_AB[3 * kp]), Y1 = R(v.pair_AB[3 * kp + 1]), Y2 = R(v.pair_AB[3 * kp + 2]);
  int mode = 0;  // 0: (bp|kp) only, 1: (kp|bp) only, 2: both, chosen per element
  if constexpr (S::kOrient) {
    const int sab = v.pair_sa[bp], skt = v.pair_sa[kp];
    mode = sab > skt ? 0 : sab < skt ? 1 : 2;
  }
  R *acc_f = acc_sh, *acc_r = acc_sh + WarpProg<LA, LB, LC, LD, REF>::kAcc;
  if (mode != 1) warp_contract<LA, LB, LC, LD, REF, R>(v, bp, kp, w, acc_f);
  if constexpr (S::kOrient) {
    if (mode != 0) warp_contract<LA, LB, LC, LD, REF, R>(v, kp, bp, w, acc_r);
  }
  const int aoa = v.pair_ao_a[bp], aob = v.pair_ao_b[bp], aoc = v.pair_ao_a[kp], aod = v.pair_ao_b[kp];
  const bool bdiag = v.pair_sa[bp] == v.pair_sb[bp], kdiag = v.pair_sa[kp] == v.pair_sb[kp];
  for (int ab = lane; ab < S::NAB; ab += 32) {
    const int a = ab / NB, b = ab - a * NB;
    R out[NCD];
    if (mode == 1) {
      if constexpr (S::kOrient)
        EriRows<LA, LB, LC, LD>::template col<R>(out, ab, acc_r, 1, Y0, Y1, Y2, X0, X1, X2);
    } else {
      EriRows<LA, LB, LC, LD>::template row<R>(out, ab, acc_f, 1, X0, X1, X2, Y0, Y1, Y2);
    }
    if constexpr (S::kOrient) {
      if (mode == 2) {
        R sw[NCD];
        EriRows<LA, LB, LC, LD>::template col<R>(sw, ab, acc_r, 1, Y0, Y1, Y2, X0, X1, X2);
        const int I = aoa + a, J = aob + b;
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
    }
    const double nab = comp_norm<LA>(a) * comp_norm<LB>(b);
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int d = 0; d < ND; ++d)
        o[ab * NCDP + c * ND + d] = double(out[c * ND + d]) * (nab * comp_norm<LC>(c) * comp_norm<LD>(d));
  }
  __syncwarp();
}

template <int LA, int LB, int LC, int LD, int MODE, bool REF, int SCR>
__global__ void __launch_bounds__(32 * WarpShape<LA, LB, LC, LD, REF>::kWarps)
    eri_warp_kernel(const EngineView v, const ClassLaunch cl) {
  using S = WarpShape<LA, LB, LC, LD, REF>;
  constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND, NAB = S::NAB, NCD = S::NCD, NCDP = S::NCDP;
  constexpr bool kUhf = MODE == kJkUhf;
  extern __shared__ __align__(16) double warp_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double *base = warp_smem + (size_t)warp * (S::kBytes / 8);
  double *o = base + S::kRDoubles;
  unsigned long long n64 = 0, n32 = 0;
  const long long nunits = (long long)launch_ntasks(cl) * 32;
  const long long ustride = (long long)gridDim.x * S::kWarps;
  for (long long u = cl.queue ? warp_fetch(cl.queue, 1) : (long long)blockIdx.x * S::kWarps + warp; u < nunits;
       u = cl.queue ? warp_fetch(cl.queue, 1) : u + ustride) {
    const Task task = launch_task(cl, (int)(u >> 5));
    const int kpos = task.ket_start + (int)(u & 31);
    if (kpos >= task.ket_end) continue;  // warp-uniform
    const int bp = cl.bra_list[task.bra_pos], kp = cl.ket_list[kpos];
    const MolView mv = task_molecule(v, bp);
    if (mv.skip) continue;
    bool fp64 = true;
    if constexpr (SCR != kScreenNone) {
      const float bnd = density_bound(v, bp, kp);
      if (!(bnd >= cl.dens_threshold)) continue;
      if constexpr (SCR == kScreenMixed) fp64 = bnd >= cl.mixed_cutoff;
      if (fp64) ++n64;
      else ++n32;
    }
    if (fp64) {
      warp_block<LA, LB, LC, LD, REF, double>(v, bp, kp, base, base + S::kWork, o);
    } else if constexpr (SCR == kScreenMixed) {
      float *wf = reinterpret_cast<float *>(base);
      warp_block<LA, LB, LC, LD, REF, float>(v, bp, kp, wf, wf + S::kWork, o);
    }
    const int n = mv.n;
    const int aoa = v.pair_ao_a[bp], aob = v.pair_ao_b[bp], aoc = v.pair_ao_a[kp], aod = v.pair_ao_b[kp];
    const bool bdiag = v.pair_sa[bp] == v.pair_sb[bp], kdiag = v.pair_sa[kp] == v.pair_sb[kp];
    const bool same = bp == kp;
    if constexpr (MODE == kStorePacked) {
      for (int x = lane; x < NAB * NCD; x += 32) {
        const int ab = x / NCD, cd = x - ab * NCD;
        const int a = ab / NB, b = ab - a * NB, c = cd / ND, d = cd - c * ND;
        const int I = aoa + a, J = aob + b, K = aoc + c, L = aod + d;
        if (bdiag && I < J) continue;
        if (kdiag && K < L) continue;
        const long long ij = tri(I, J), kl = tri(K, L);
        if (same && ij < kl) continue;
        cl.packed[tri(ij, kl)] = o[ab * NCDP + cd];
      }
    } else {
      // every element of J_ab, J_cd, K_ac, K_ad, K_bc, K_bd (and the beta K
      // blocks for UHF) is one lane's dot product over the block
      const double s = (bdiag ? 0.5 : 1.0) * (kdiag ? 0.5 : 1.0) * (same ? 0.5 : 1.0);
      const double *Da = cl.Da + mv.base, *Db = kUhf ? cl.Db + mv.base : nullptr;
      const double *DJ = kUhf ? cl.Dt + mv.base : Da;
      double *Jm = cl.J + mv.base, *Kam = cl.Ka + mv.base, *Kbm = kUhf ? cl.Kb + mv.base : nullptr;
      constexpr int nK = NA * NC + NA * ND + NB * NC + NB * ND;
      constexpr int total = NAB + NCD + nK * (kUhf ? 2 : 1);
      for (int x = lane; x < total; x += 32) {
        double t = 0.0;
        if (x < NAB) {
          const int a = x / NB, b = x - a * NB;
#pragma unroll 4
          for (int cd = 0; cd < NCD; ++cd) {
            const int c = cd / ND, d = cd - c * ND;
            t += o[x * NCDP + cd] * __ldg(&DJ[(aoc + c) * n + aod + d]);
          }
          atomicAdd(&Jm[(aoa + a) * n + aob + b], 2.0 * s * t);
        } else if (x < NAB + NCD) {
          const int cd = x - NAB, c = cd / ND, d = cd - c * ND;
#pragma unroll 4
          for (int ab = 0; ab < NAB; ++ab) {
            const int a = ab / NB, b = ab - a * NB;
            t += o[ab * NCDP + cd] * __ldg(&DJ[(aoa + a) * n + aob + b]);
          }
          atomicAdd(&Jm[(aoc + c) * n + aod + d], 2.0 * s * t);
        } else {
          int y = x - NAB - NCD;
          const bool beta = kUhf && y >= nK;
          if (beta) y -= nK;
          const double *D = beta ? Db : Da;
          double *Km = beta ? Kbm : Kam;
          if (y < NA * NC) {  // K_ac = sum_bd (ab|cd) D_bd
            const int a = y / NC, c = y - a * NC;
            for (int b = 0; b < NB; ++b)
#pragma unroll
              for (int d = 0; d < ND; ++d) t += o[(a * NB + b) * NCDP + c * ND + d] * __ldg(&D[(aob + b) * n + aod + d]);
            atomicAdd(&Km[(aoa + a) * n + aoc + c], s * t);
          } else if ((y -= NA * NC) < NA * ND) {  // K_ad = sum_bc (ab|cd) D_bc
            const int a = y / ND, d = y - a * ND;
            for (int b = 0; b < NB; ++b)
#pragma unroll
              for (int c = 0; c < NC; ++c) t += o[(a * NB + b) * NCDP + c * ND + d] * __ldg(&D[(aob + b) * n + aoc + c]);
            atomicAdd(&Km[(aoa + a) * n + aod + d], s * t);
          } else if ((y -= NA * ND) < NB * NC) {  // K_bc = sum_ad (ab|cd) D_ad
            const int b = y / NC, c = y - b * NC;
            for (int a = 0; a < NA; ++a)
#pragma unroll
              for (int d = 0; d < ND; ++d) t += o[(a * NB + b) * NCDP + c * ND + d] * __ldg(&D[(aoa + a) * n + aod + d]);
            atomicAdd(&Km[(aob + b) * n + aoc + c], s * t);
          } else {  // K_bd = sum_ac (ab|cd) D_ac
            y -= NB * NC;
            const int b = y / ND, d = y - b * ND;
            for (int a = 0; a < NA; ++a)
#pragma unroll
              for (int c = 0; c < NC; ++c) t += o[(a * NB + b) * NCDP + c * ND + d] * __ldg(&D[(aoa + a) * n + aoc + c]);
            atomicAdd(&Km[(aob + b) * n + aod + d], s * t);
          }
        }
      }
    }
    __syncwarp();  // the block is rewritten by the warp's next quartet
  }
  if constexpr (SCR != kScreenNone) {
    if (lane == 0 && cl.counters && (n64 | n32)) {
      atomicAdd(&cl.counters[0], n64);
      atomicAdd(&cl.counters[1], n32);
    }
  }
}

// Host: launch one warp-cooperative class kernel; `grid` caps the blocks
// (0: as many as are resident at once on every SM).
template <int LA, int LB, int LC, int LD, int MODE, bool REF, int SCR>
void launch_warp(const EngineView &v, const ClassLaunch &cl, int grid, cudaStream_t s) {
  using S = WarpShape<LA, LB, LC, LD, REF>;
  auto kern = eri_warp_kernel<LA, LB, LC, LD, MODE, REF, SCR>;
  static int resident = 0;  // blocks per SM, set once per instantiation
  static int num_sms = 0;
  if (resident == 0) {
    if (S::kBytes * S::kWarps > 48 * 1024)
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kBytes * S::kWarps);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
    int r = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, kern, 32 * S::kWarps, S::kBytes * S::kWarps);
    resident = r > 0 ? r : 1;
  }
  const long long units = (long long)cl.ntasks * 32;
  const long long need = (units + S::kWarps - 1) / S::kWarps;
  long long g = (long long)num_sms * resident;
  if (grid > 0) g = std::min<long long>(g, grid);
  g = std::max<long long>(1, std::min(g, need));
  kern<<<(int)g, 32 * S::kWarps, S::kBytes * S::kWarps, s>>>(v, cl);
}

}  // namespace hfg
