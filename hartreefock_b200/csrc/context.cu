// Host side of the engine: context construction (shell pairs, primitive-pair
// tables, Schwarz bounds, class lists), the stored and direct builds, and the
// C ABI declared in include/hfgpu.h.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <cstdlib>
#include <mutex>
#include <numeric>
#include <set>
#include <string>
#include <vector>

#include "../../include/hfgpu.h"
#include "eri_dispatch.cuh"
#include "eri_split_dispatch.cuh"
#include "eri_warp_dispatch.cuh"

namespace hfg {

static thread_local std::string g_last_error;

static hfg_status fail(hfg_status st, const std::string &msg) {
  g_last_error = msg;
  return st;
}

// for entry points defined in other translation units (hfg_eigh_batched,
// hfg_one_electron)
hfg_status fail_external(hfg_status st, const std::string &msg) { return fail(st, msg); }
static const std::vector<double> &boys_table_host();
const std::vector<double> &boys_table_for_external() { return boys_table_host(); }

#define HFG_CUDA(call)                                                                        \
  do {                                                                                        \
    cudaError_t err__ = (call);                                                               \
    if (err__ != cudaSuccess)                                                                 \
      return fail(err__ == cudaErrorMemoryAllocation ? HFG_OOM_BUDGET : HFG_DEVICE_ERROR,      \
                  std::string(#call) + ": " + cudaGetErrorString(err__));                     \
  } while (0)

// ---------------------------------------------------------------------------
// Boys table F_m(T_i), T_i = i * kBoysStep, m = 0 .. kBoysOrders-1, from the
// convergent series F_m(T) = e^-T sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1))
// evaluated in extended precision (all terms positive, no cancellation).
// ---------------------------------------------------------------------------
static const std::vector<double> &boys_table_host() {
  static std::vector<double> tab;
  static std::once_flag once;
  std::call_once(once, [] {
    tab.resize((size_t)kBoysGrid * kBoysOrders + kBoysGrid);
    for (int i = 0; i < kBoysGrid; ++i) {
      const long double T = (long double)i * (long double)kBoysStep;
      for (int m = 0; m < kBoysOrders; ++m) {
        long double term = 1.0L / (2 * m + 1), sum = 0;
        for (int k = 0; k < 2000; ++k) {
          sum += term;
          term *= 2.0L * T / (2 * m + 2 * k + 3);
          if (term < sum * 1e-21L) break;
        }
        tab[(size_t)i * kBoysOrders + m] = (double)(expl(-T) * sum);
      }
      tab[(size_t)kBoysGrid * kBoysOrders + i] = (double)expl(-T);  // e^-T_i
    }
    // the per-order rows (the same products the kernels form when they
    // stage a slice into shared memory)
    const double inv_fact[kBoysTaylor] = {1.0, 1.0, 0.5, 1.0 / 6.0, 1.0 / 24.0, 1.0 / 120.0, 1.0 / 720.0};
    tab.resize((size_t)kBoysFoldedOff + (size_t)(kMaxLtot + 1) * kBoysFoldedSize);
    for (int L = 0; L <= kMaxLtot; ++L)
      for (int i = 0; i < kBoysGrid; ++i)
        for (int k = 0; k < kBoysRow; ++k)
          tab[(size_t)kBoysFoldedOff + (size_t)L * kBoysFoldedSize + boys_swizzle(i, k)] =
              k < kBoysTaylor ? tab[(size_t)i * kBoysOrders + L + k] * inv_fact[k]
                              : tab[(size_t)kBoysGrid * kBoysOrders + i];
  });
  return tab;
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
struct HostShell {
  double c[3];
  int L, nprim, prim_off, ao;
};

// Pairs of one class, grouped into buckets of similar primitive-pair count
// (so that the 32 kets of a warp run equal primitive loops), each bucket
// sorted by Schwarz bound descending (so that screening cuts a prefix).
constexpr int kBuckets = 6;
static inline int prim_bucket(int np) { return np <= 1 ? 0 : np <= 3 ? 1 : np <= 6 ? 2 : np <= 12 ? 3 : np <= 24 ? 4 : 5; }
struct PairClassList {
  std::vector<int> pairs;  // concatenated buckets
  // segment starts in `pairs`, molecule-major then bucket: molecule m's
  // bucket k is [seg_start[m * kBuckets + k], seg_start[m * kBuckets + k + 1])
  std::vector<int> seg_start;
  int *d_pairs = nullptr;
};

struct QuartetClass {
  int cls;       // index into kClasses
  int bra_pc, ket_pc;
  std::vector<Task> tasks;
  Task *d_tasks = nullptr;
  int64_t shell_quartets = 0, function_quartets = 0, prim_quartets = 0;
  double flops = 0;
  // lane occupancy of the thread-per-quartet layout: primitive quartets the
  // lanes evaluate over the lanes x the longest lane loop of each task
  double lane_work = 0, warp_work = 0;
  // estimated flops of tasks [0, t): shards take contiguous ranges of equal cost
  std::vector<double> cost_prefix;
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;  // per-class timing (profiling on)
  float last_ms = 0;
};

template <class T>
static hfg_status upload(T **dst, const std::vector<T> &src) {
  *dst = nullptr;
  if (src.empty()) return HFG_OK;
  HFG_CUDA(cudaMalloc((void **)dst, src.size() * sizeof(T)));
  HFG_CUDA(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
  // a pageable-to-device cudaMemcpy returns once the data is staged; the DMA
  // itself is queued on the legacy default stream, which the context's
  // non-blocking streams do not wait for: let it land before any kernel of
  // ours reads the table
  HFG_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
  return HFG_OK;
}

}  // namespace hfg

using namespace hfg;

struct hfg_ctx {
  hfg_opts opts{};
  int device = 0;
  int nbf = 0;
  std::vector<HostShell> shells;
  int npairs = 0;
  std::vector<int> pair_sa, pair_sb, pair_cls, pair_nprim;
  std::vector<double> pair_Q;
  PairClassList pclass[kNumPairClasses];
  std::vector<QuartetClass> qclasses;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // class kernels of one build are independent (J/K by atomics): they run on
  // the build stream and kAux more, forked and joined by events, so small
  // molecules' classes overlap instead of queueing
  static constexpr int kAux = 12;
  cudaStream_t aux[kAux] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[kAux] = {};
  int num_sms = 148;
  // grid cap of the fused class kernels, in blocks per SM; 0 = automatic: 4
  // with every class on the build stream, 1 with concurrent class streams
  // (where other classes share the SMs)
  int blocks_per_sm = 0;
  int tuned_bps[kNumClasses] = {};  // per class, from hfg_autotune (0 = blocks_per_sm)
  // primitive quartets per lane that the task builder aims for when it
  // spreads a quartet over a lane group (0: one lane per quartet); per class
  // from hfg_autotune, else prim_target
  int prim_target = 96;
  int class_prim_target[kNumClasses] = {};
  // CUDA graph of the plain direct build (hfg_set_graphs): captured on the
  // second build with the same buffers, stream and settings, replayed after
  bool use_graphs = false;
  bool use_streams = false;  // class kernels over the auxiliary streams (hfg_set_streams)
  // large classes with both kernels: 1 = the warp-cooperative kernel, 0 =
  // the split path (primitive kernel + HRR/digest over scratch); per class,
  // from hfg_autotune_paths / hfg_set_class_path, else the default below
  int8_t warp_class[kNumClasses] = {};
  // direct builds: the fused and warp-cooperative class kernels take their
  // tasks from a device work queue (one counter per class, one atomic per
  // warp and task) instead of a grid-stride walk
  bool use_queue = false;
  // density-screened builds compact the live tasks before the class kernels
  // (HFG_NO_COMPACT=1: every task goes to the class kernels, which skip the
  // dead ones themselves)
  bool use_compaction = true;
  cudaEvent_t ev_done = nullptr;  // end of the last build on its stream
  unsigned config_version = 0;  // bumped by every setter that changes a build
  struct GraphKey {
    bool uhf = false;
    const void *pa = nullptr, *pb = nullptr, *ga = nullptr, *gb = nullptr, *s = nullptr;
    unsigned version = 0;
    bool operator==(const GraphKey &o) const {
      return uhf == o.uhf && pa == o.pa && pb == o.pb && ga == o.ga && gb == o.gb && s == o.s && version == o.version;
    }
  };
  GraphKey graph_key, graph_seen;
  bool graph_seen_valid = false;
  cudaGraphExec_t graph_exec = nullptr;
  hfg_stats graph_stats{};
  // device tables
  PrimPair *d_prim = nullptr;
  PrimPairF *d_primf = nullptr;
  int *d_pair_prim_off = nullptr, *d_pair_nprim = nullptr, *d_pair_sa = nullptr, *d_pair_sb = nullptr;
  int *d_pair_ao_a = nullptr, *d_pair_ao_b = nullptr;
  double *d_pair_AB = nullptr, *d_pair_Q = nullptr, *d_boys = nullptr;
  // work buffers
  double *d_J = nullptr, *d_Ka = nullptr, *d_Kb = nullptr, *d_P = nullptr, *d_Pb = nullptr, *d_Pt = nullptr;
  double *d_G = nullptr, *d_Gb = nullptr, *d_block = nullptr;
  // split-path [e0|f0] blocks, one region per auxiliary stream (the split
  // classes of a build run on those streams concurrently)
  double *d_scratch[kAux] = {};
  size_t scratch_doubles[kAux] = {};
  size_t scratch_budget_bytes = size_t(512) << 20;
  // precision form: density screening, FP32 cutoff, incremental history
  int nshells = 0;
  int *d_shell_ao = nullptr, *d_shell_nf = nullptr;
  float *d_shell_dmax = nullptr;                 // [nshells][nshells]
  unsigned long long *d_counters = nullptr;      // FP64 / FP32 quartets of the last build
  double *d_prev_P[2] = {}, *d_prev_G[2] = {};   // incremental history (alpha, beta)
  double *d_dP[2] = {};                          // density difference of the build
  bool inc_valid = false, inc_uhf = false;
  double mixed_cutoff = 0;
  bool counted = false;                          // d_counters hold the last build's counts
  int shard_rank = 0, shard_count = 1;           // direct builds: this shard of every class's tasks
  // batched contexts: many molecules, shell pairs and quartets only within a
  // molecule, each molecule's n x n matrices at mol_off[m] in flat buffers
  bool batch = false;
  int nmol = 1;
  std::vector<int> pair_mol, mol_nbf;
  std::vector<long long> mol_off;
  long long batch_elems = 0;
  int *d_pair_mol = nullptr, *d_mol_nbf = nullptr;
  long long *d_mol_off = nullptr;
  unsigned char *d_mol_active = nullptr;
  // batched builds with converged molecules: the active molecules' tasks of
  // every class, compacted on the device, and their counts
  Task *d_task_active = nullptr;
  int *d_task_counts = nullptr;
  int *d_queue = nullptr;  // per quartet class: the device work queue's counter
  std::vector<int> task_base;  // per quartet class, offset into d_task_active
  hfg_stats stats{};
  bool profiling = false;
  bool precision_form() const { return opts.density_screening || opts.incremental || mixed_cutoff > 0; }
  double density_threshold() const {
    return opts.density_threshold > 0 ? opts.density_threshold : opts.schwarz_threshold;
  }
  EngineView view() const {
    EngineView v{};
    v.prim = d_prim;
    v.primf = d_primf;
    v.pair_prim_off = d_pair_prim_off;
    v.pair_nprim = d_pair_nprim;
    v.pair_sa = d_pair_sa;
    v.pair_sb = d_pair_sb;
    v.pair_ao_a = d_pair_ao_a;
    v.pair_ao_b = d_pair_ao_b;
    v.pair_AB = d_pair_AB;
    v.pair_Q = d_pair_Q;
    v.shell_dmax = d_shell_dmax;
    v.nshells = nshells;
    v.boys_table = d_boys;
    v.nbf = nbf;
    v.reference_convention = opts.eri_convention == HFG_ERI_REFERENCE;
    if (batch) {
      v.pair_mol = d_pair_mol;
      v.mol_nbf = d_mol_nbf;
      v.mol_off = d_mol_off;
      v.mol_active = d_mol_active;
    }
    return v;
  }
  ~hfg_ctx() {
    cudaSetDevice(device);
    // the last build may still be queued (on the caller's stream and ours):
    // let it finish before its buffers go
    if (ev_done) cudaEventSynchronize(ev_done);
    for (int i = 0; i < kAux; ++i)
      if (aux[i]) cudaStreamSynchronize(aux[i]);
    if (stream) cudaStreamSynchronize(stream);
    for (auto &q : qclasses) {
      cudaFree(q.d_tasks);
      if (q.ev_a) cudaEventDestroy(q.ev_a);
      if (q.ev_b) cudaEventDestroy(q.ev_b);
    }
    for (auto &p : pclass) cudaFree(p.d_pairs);
    void *bufs[] = {d_prim,       d_pair_prim_off, d_pair_nprim, d_pair_sa,  d_pair_sb,    d_pair_ao_a, d_pair_ao_b,
                    d_pair_AB,    d_pair_Q,        d_boys,       d_J,        d_Ka,         d_Kb,        d_P,
                    d_Pb,         d_Pt,            d_G,          d_Gb,       d_block,      d_scratch[0], d_shell_ao,
                    d_shell_nf,   d_shell_dmax,    d_counters,   d_prev_P[0], d_prev_P[1], d_prev_G[0], d_prev_G[1],
                    d_dP[0],      d_dP[1],         d_primf,      d_pair_mol, d_mol_nbf,    d_mol_off,   d_mol_active,
                    d_task_active, d_task_counts, d_queue};
    for (void *b : bufs) cudaFree(b);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    for (int i = 0; i < kAux; ++i) {
      if (aux[i]) cudaStreamDestroy(aux[i]);
      if (ev_join[i]) cudaEventDestroy(ev_join[i]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_done) cudaEventDestroy(ev_done);
    for (int i = 1; i < kAux; ++i) cudaFree(d_scratch[i]);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }
};

// the large class runs on the warp-cooperative kernel (classes with only
// that kernel always do)
static bool class_on_warp(const hfg_ctx *c, int cls) { return kWarp[cls] && (c->warp_class[cls] || !kSplit[cls]); }

namespace hfg {

static int pair_class_index(int la, int lb) {
  for (int i = 0; i < kNumPairClasses; ++i)
    if (kPairClasses[i][0] == la && kPairClasses[i][1] == lb) return i;
  return -1;
}

static int class_index(int la, int lb, int lc, int ld) {
  for (int i = 0; i < kNumClasses; ++i)
    if (kClasses[i].la == la && kClasses[i].lb == lb && kClasses[i].lc == lc && kClasses[i].ld == ld) return i;
  return -1;
}

static double prim_flops(int cls, bool reference) {
  for (const auto &f : kEriClassFlops)
    if (f.la == kClasses[cls].la && f.lb == kClasses[cls].lb && f.lc == kClasses[cls].lc &&
        f.ld == kClasses[cls].ld)
      return reference ? f.prim_reference : f.prim_exact;
  return 0;
}
static double hrr_flops(int cls) {
  for (const auto &f : kEriClassFlops)
    if (f.la == kClasses[cls].la && f.lb == kClasses[cls].lb && f.lc == kClasses[cls].lc &&
        f.ld == kClasses[cls].ld)
      return f.hrr;
  return 0;
}
// Boys (7-term Horner, exp, downward recursion) + prefactor/geometry per
// primitive quartet, counted as 2 flops per FMA, exp as 1
static double boys_geom_flops(int ltot) { return 14 + 3 * ltot + 40; }

static inline int ncart_h(int L) { return (L + 1) * (L + 2) / 2; }

// number of 8-fold unique function quartets in a pair's function block
static inline int64_t pair_functions(const hfg_ctx *c, int p) {
  const int na = ncart_h(c->shells[c->pair_sa[p]].L), nb = ncart_h(c->shells[c->pair_sb[p]].L);
  return c->pair_sa[p] == c->pair_sb[p] ? (int64_t)na * (na + 1) / 2 : (int64_t)na * nb;
}

// Build per-class quartet task lists with Schwarz screening at `threshold`.
// Every unordered pair of pairs appears once: for different classes all
// (bra, ket) combinations, for the same class the kets at positions <= the
// bra's position in the concatenated bucket list.
static void build_quartet_classes(hfg_ctx *c, double threshold) {
  c->qclasses.clear();
  for (int ci = 0; ci < kNumClasses; ++ci) {
    const ClassEntry &ce = kClasses[ci];
    QuartetClass q;
    q.cls = ci;
    q.bra_pc = pair_class_index(ce.la, ce.lb);
    q.ket_pc = pair_class_index(ce.lc, ce.ld);
    const PairClassList &BL = c->pclass[q.bra_pc], &KL = c->pclass[q.ket_pc];
    const auto &bras = BL.pairs;
    const auto &kets = KL.pairs;
    if (bras.empty() || kets.empty()) continue;
    const bool same = q.bra_pc == q.ket_pc;
    std::vector<int64_t> kfun(kets.size() + 1, 0), kprim(kets.size() + 1, 0);
    std::vector<double> kq(kets.size());
    for (size_t k = 0; k < kets.size(); ++k) {
      kfun[k + 1] = kfun[k] + pair_functions(c, kets[k]);
      kprim[k + 1] = kprim[k] + c->pair_nprim[kets[k]];
      kq[k] = c->pair_Q[kets[k]];
    }
    const double pf = prim_flops(ci, c->opts.eri_convention == HFG_ERI_REFERENCE);
    const double hf = hrr_flops(ci);
    const int ltot = ce.la + ce.lb + ce.lc + ce.ld;
    // the longest ket contraction of each bucket segment
    std::vector<int> segmax(KL.seg_start.size(), 0);
    for (size_t g = 0; g + 1 < KL.seg_start.size(); ++g)
      for (int64_t k2 = KL.seg_start[g]; k2 < KL.seg_start[g + 1]; ++k2)
        segmax[g] = std::max(segmax[g], c->pair_nprim[kets[k2]]);
    // fused thread-per-quartet classes: lanes per quartet so that a lane's
    // share of a quartet's primitive quartets stays near the target (long
    // contractions spread over 2..32 lanes, fewer kets per task); the large
    // classes (split path: one lane per quartet; warp kernel: one warp per
    // quartet) keep 32 kets per task
    const bool grouped = !kSplit[ci] && !kWarp[ci];
    const int target = c->class_prim_target[ci] > 0 ? c->class_prim_target[ci]
                       : c->class_prim_target[ci] < 0 ? 0 : c->prim_target;
    for (size_t b = 0; b < bras.size(); ++b) {
      const double qb = c->pair_Q[bras[b]];
      if (!(qb > 0)) continue;
      const double need = threshold / qb;
      const int64_t bf = pair_functions(c, bras[b]);
      const int64_t bprim = c->pair_nprim[bras[b]];
      // kets come from the bra's own molecule only
      const int mol = c->pair_mol.empty() ? 0 : c->pair_mol[bras[b]];
      for (int k = 0; k < kBuckets; ++k) {
        const int64_t s0 = KL.seg_start[mol * kBuckets + k], s1 = KL.seg_start[mol * kBuckets + k + 1];
        // kets of the bucket with qb * qk >= threshold form a prefix
        int64_t lo = s0, hi = s1;
        while (lo < hi) {
          const int64_t mid = (lo + hi) / 2;
          if (kq[mid] >= need) lo = mid + 1;
          else hi = mid;
        }
        int64_t end = lo;
        if (same) end = std::min<int64_t>(end, (int64_t)b + 1);
        if (end <= s0) continue;
        int per_task = 32;
        if (grouped && target > 0) {
          const double work = (double)bprim * segmax[mol * kBuckets + k];
          int G = 1;
          while (G < 32 && work / G > target) G <<= 1;
          per_task = 32 / G;
        }
        for (int64_t st = s0; st < end; st += per_task) {
          const int64_t e1 = std::min<int64_t>(st + per_task, end);
          Task tk{(int)b, (int)st, (int)e1};
          int m2 = 1;
          while (m2 < e1 - st) m2 <<= 1;
          if (grouped)
            while ((32 >> tk.lg) > m2) ++tk.lg;  // 32 / 2^lg lane groups, at least the task's kets
          q.tasks.push_back(tk);
          int64_t mx = 0;
          for (int64_t k2 = st; k2 < e1; ++k2) mx = std::max<int64_t>(mx, c->pair_nprim[kets[k2]]);
          q.lane_work += (double)bprim * (double)(kprim[e1] - kprim[st]);
          q.warp_work += 32.0 * std::ceil((double)bprim * (double)mx / (double)(1 << tk.lg));
          if (q.cost_prefix.empty()) q.cost_prefix.push_back(0.0);
          q.cost_prefix.push_back(q.cost_prefix.back() +
                                  (double)bprim * (double)(kprim[e1] - kprim[st]) * (pf + boys_geom_flops(ltot)) +
                                  (double)(e1 - st) * hf);
        }
        q.shell_quartets += end - s0;
        if (same && end == (int64_t)b + 1) {
          // the diagonal quartet (bra == ket) counts its unique half
          q.function_quartets += bf * (kfun[end - 1] - kfun[s0]) + bf * (bf + 1) / 2;
        } else {
          q.function_quartets += bf * (kfun[end] - kfun[s0]);
        }
        q.prim_quartets += bprim * (kprim[end] - kprim[s0]);
      }
    }
    q.flops = (double)q.prim_quartets * (pf + boys_geom_flops(ltot)) + (double)q.shell_quartets * hf;
    if (!q.tasks.empty()) c->qclasses.push_back(std::move(q));
  }
  // largest classes first
  std::sort(c->qclasses.begin(), c->qclasses.end(),
            [](const QuartetClass &a, const QuartetClass &b) { return a.flops > b.flops; });
}

static hfg_status upload_classes(hfg_ctx *c) {
  for (auto &q : c->qclasses) {
    const hfg_status st = upload(&q.d_tasks, q.tasks);
    if (st != HFG_OK) return st;
  }
  return HFG_OK;
}

// blocks of a fused class launch: one warp per task, fused_warps() per block
static int grid_for(const hfg_ctx *c, int ntasks, int cls) {
  const ClassEntry &e = kClasses[cls];
  const int w = fused_warps(e.la, e.lb, e.lc, e.ld);
  const int blocks = (ntasks + w - 1) / w;
  const int def = c->blocks_per_sm > 0 ? c->blocks_per_sm : (c->use_streams && !c->profiling ? 1 : 4);
  const int bps = c->tuned_bps[cls] > 0 ? c->tuned_bps[cls] : def;
  return std::max(1, std::min(blocks, c->num_sms * bps));
}

// Shard `rank` of `count` of tasks with running cost `prefix` (ntasks + 1
// entries from 0): shard r begins at the first task whose prefix reaches
// r / count of the total, so the shards tile the tasks in order.
static void shard_range(const double *prefix, int64_t ntasks, int rank, int count, int64_t *first, int64_t *n) {
  const double whole = prefix[ntasks];
  auto bound = [&](int r) -> int64_t {
    if (r <= 0) return 0;
    if (r >= count) return ntasks;
    const double target = whole * r / count;
    return std::min<int64_t>(ntasks, std::lower_bound(prefix, prefix + ntasks + 1, target) - prefix);
  };
  const int64_t lo = bound(rank), hi = bound(rank + 1);
  *first = lo;
  *n = std::max<int64_t>(0, hi - lo);
}

// A class launch over all tasks, or with `sharded` over this context's
// shard of them: a contiguous range of the class's tasks whose estimated
// cost (primitive quartets x the class's recursion and Boys flops, plus its
// horizontal recursions per quartet) is 1/shard_count of the class's, so
// shards of uneven task mixes take equal work.
static ClassLaunch base_launch(const hfg_ctx *c, const QuartetClass &q, bool sharded = false) {
  ClassLaunch cl{};
  cl.bra_list = c->pclass[q.bra_pc].d_pairs;
  cl.ket_list = c->pclass[q.ket_pc].d_pairs;
  cl.tasks = q.d_tasks;
  const int total = (int)q.tasks.size();
  cl.task_offset = 0;
  cl.task_stride = 1;
  cl.ntasks = total;
  if (sharded && c->shard_count > 1 && (int)q.cost_prefix.size() == total + 1) {
    int64_t first = 0, count = 0;
    shard_range(q.cost_prefix.data(), total, c->shard_rank, c->shard_count, &first, &count);
    cl.task_offset = (int)first;
    cl.ntasks = (int)count;
  }
  cl.same_class = q.bra_pc == q.ket_pc;
  return cl;
}

// the cost share of a launch in its class (shards report their part of the
// class's quartet and flop counts)
static double launch_share(const QuartetClass &q, const ClassLaunch &cl) {
  if (q.tasks.empty()) return 0.0;
  if ((int)q.cost_prefix.size() != (int)q.tasks.size() + 1 || q.cost_prefix.back() <= 0)
    return (double)cl.ntasks / (double)q.tasks.size();
  return (q.cost_prefix[cl.task_offset + cl.ntasks] - q.cost_prefix[cl.task_offset]) / q.cost_prefix.back();
}

__global__ void finalize_rhf(const double *J, const double *K, double *G, int n) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n * n; x += gridDim.x * blockDim.x) {
    const int i = x / n, j = x - i * n;
    const double jv = J[i * n + j] + J[j * n + i];
    const double kv = K[i * n + j] + K[j * n + i];
    G[x] = jv - 0.5 * kv;
  }
}

__global__ void finalize_uhf(const double *J, const double *Ka, const double *Kb, double *Ga, double *Gb, int n) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n * n; x += gridDim.x * blockDim.x) {
    const int i = x / n, j = x - i * n;
    const double jv = J[i * n + j] + J[j * n + i];
    Ga[x] = jv - (Ka[i * n + j] + Ka[j * n + i]);
    Gb[x] = jv - (Kb[i * n + j] + Kb[j * n + i]);
  }
}

__global__ void add_densities(const double *a, const double *b, double *t, int nn) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < nn; x += gridDim.x * blockDim.x) t[x] = a[x] + b[x];
}

// Incremental builds: dP = P - P_prev (P_prev taken as 0 when `fresh`), then
// P_prev = P.
__global__ void density_difference(const double *P, double *prev, double *dP, int nn, int fresh) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < nn; x += gridDim.x * blockDim.x) {
    const double p = P[x];
    dP[x] = fresh ? p : p - prev[x];
    prev[x] = p;
  }
}

// max |A| (+ |B| when B is given) over each shell block, thread per block
__global__ void shell_block_max(const double *A, const double *B, const int *ao, const int *nf, int ns, int n,
                                float *out) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < ns * ns; x += gridDim.x * blockDim.x) {
    const int sa = x / ns, sb = x - sa * ns;
    const int i0 = ao[sa], j0 = ao[sb], ni = nf[sa], nj = nf[sb];
    double m = 0.0;
    for (int i = i0; i < i0 + ni; ++i)
      for (int j = j0; j < j0 + nj; ++j) {
        const double a = fabs(A[(size_t)i * n + j]) + (B ? fabs(B[(size_t)i * n + j]) : 0.0);
        m = fmax(m, a);
      }
    // round up so that the float bound never undercuts the double one
    out[x] = __double2float_ru(m);
  }
}

// G = (accumulate ? G_prev : 0) + (J + J^T) - (K + K^T)/2, G_prev = G
__global__ void finalize_rhf_incremental(const double *J, const double *K, double *Gprev, double *G, int n,
                                         int accumulate) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n * n; x += gridDim.x * blockDim.x) {
    const int i = x / n, j = x - i * n;
    const double g = (accumulate ? Gprev[x] : 0.0) + (J[i * n + j] + J[j * n + i]) - 0.5 * (K[i * n + j] + K[j * n + i]);
    G[x] = g;
    Gprev[x] = g;
  }
}

__global__ void finalize_uhf_incremental(const double *J, const double *Ka, const double *Kb, double *Gaprev,
                                         double *Gbprev, double *Ga, double *Gb, int n, int accumulate) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n * n; x += gridDim.x * blockDim.x) {
    const int i = x / n, j = x - i * n;
    const double jv = J[i * n + j] + J[j * n + i];
    const double ga = (accumulate ? Gaprev[x] : 0.0) + jv - (Ka[i * n + j] + Ka[j * n + i]);
    const double gb = (accumulate ? Gbprev[x] : 0.0) + jv - (Kb[i * n + j] + Kb[j * n + i]);
    Ga[x] = ga;
    Gb[x] = gb;
    Gaprev[x] = ga;
    Gbprev[x] = gb;
  }
}

static hfg_status ensure(double **p, size_t count) {
  if (*p) return HFG_OK;
  HFG_CUDA(cudaMalloc((void **)p, count * sizeof(double)));
  return HFG_OK;
}

// Launch one class: the fused kernel, or for the large classes the split
// primitive + HRR/digest kernels over chunks of tasks sized to the scratch
// budget.  Counts the kernel launches in *launches.
static int ncomp_range(int lo, int hi) {
  int s = 0;
  for (int L = lo; L <= hi; ++L) s += ncart_h(L);
  return s;
}

// Fork / join of a build's class launches over the build stream and the
// context's auxiliary streams.  Split classes take the auxiliary streams in
// turn, each stream with its own scratch region; fused classes take the
// build stream and the auxiliary streams in turn.  Off (everything on the
// build stream, scratch region 0) while per-class profiling is on.
static void split_chunking(const hfg_ctx *c, int cls, int ntasks, bool ref, size_t *need, int *chunk_tasks);
static int scratch_regions(const hfg_ctx *c);
// the class runs the split (primitive + HRR/digest) kernels over scratch
static bool uses_split(const hfg_ctx *c, int cls) { return kSplit[cls] && !class_on_warp(c, cls); }
static hfg_status grow_scratch(hfg_ctx *c, int slot, size_t need);

struct ClassStreams {
  hfg_ctx *c;
  cudaStream_t s;
  bool on;
  int next = 0, next_split = 0;
  int slot = 0;  // scratch region of the last split pick
  hfg_status fork() {
    if (!on) return HFG_OK;
    HFG_CUDA(cudaEventRecord(c->ev_fork, s));
    for (int i = 0; i < hfg_ctx::kAux; ++i) HFG_CUDA(cudaStreamWaitEvent(c->aux[i], c->ev_fork, 0));
    return HFG_OK;
  }
  cudaStream_t pick(bool split) {
    slot = 0;
    if (!on) return s;
    if (split) {
      slot = next_split++ % hfg_ctx::kAux;
      return c->aux[slot];
    }
    const int k = next++ % (hfg_ctx::kAux + 1);  // 0 = build stream, then aux[0..]
    return k == 0 ? s : c->aux[k - 1];
  }
  // Sizes the scratch region of every split class before anything of the
  // build is launched, following the order pick() will hand out regions in
  // (`ntasks` per quartet class, in class order).
  hfg_status presize(const std::vector<int> &ntasks, bool ref) {
    std::vector<size_t> need(hfg_ctx::kAux, 0);
    int k = 0;
    for (size_t i = 0; i < c->qclasses.size(); ++i) {
      const int cls = c->qclasses[i].cls;
      if (!uses_split(c, cls) || ntasks[i] <= 0) continue;
      size_t nd = 0;
      int chunk = 1;
      split_chunking(c, cls, ntasks[i], ref, &nd, &chunk);
      const int slot_i = on ? k++ % hfg_ctx::kAux : 0;
      need[slot_i] = std::max(need[slot_i], nd);
    }
    for (int i = 0; i < hfg_ctx::kAux; ++i) {
      const hfg_status st = grow_scratch(c, i, need[i]);
      if (st != HFG_OK) return st;
    }
    return HFG_OK;
  }
  hfg_status join() {
    if (!on) return HFG_OK;
    for (int i = 0; i < hfg_ctx::kAux; ++i) {
      HFG_CUDA(cudaEventRecord(c->ev_join[i], c->aux[i]));
      HFG_CUDA(cudaStreamWaitEvent(s, c->ev_join[i], 0));
    }
    return HFG_OK;
  }
};

// `prec`: 0 plain FP64, 1 density-screened FP64, 2 density-screened with
// the per-task FP64/FP32 choice (the precision form).
// Scratch regions in use: one per auxiliary stream with concurrent classes,
// else one.
static int scratch_regions(const hfg_ctx *c) { return c->use_streams && !c->profiling ? hfg_ctx::kAux : 1; }

// Scratch doubles and tasks per chunk of a split class launched over
// `ntasks` tasks: chunks keep one region within its share of the scratch
// budget.
static void split_chunking(const hfg_ctx *c, int cls, int ntasks, bool ref, size_t *need, int *chunk_tasks) {
  const ClassEntry &e = kClasses[cls];
  const size_t acc = (size_t)ncomp_range(e.la, e.la + e.lb) * ncomp_range(e.lc, e.lc + e.ld);
  const bool two = ref && e.la == 2 && e.lb == 2 && e.lc == 2 && e.ld == 2;
  const size_t per_task = 32 * acc * (two ? 2 : 1);
  const int max_tasks =
      (int)std::max<size_t>(1, c->scratch_budget_bytes / scratch_regions(c) / (per_task * sizeof(double)));
  *chunk_tasks = std::min(ntasks, max_tasks);
  *need = (size_t)*chunk_tasks * per_task;
}

// Grows scratch region `slot` to `need` doubles.  The old region may still
// be read by queued split kernels, so the device is drained before it is
// freed (a build sizes its regions before it launches anything, so this
// runs on the first builds only).
static hfg_status grow_scratch(hfg_ctx *c, int slot, size_t need) {
  if (need <= c->scratch_doubles[slot]) return HFG_OK;
  HFG_CUDA(cudaDeviceSynchronize());
  cudaFree(c->d_scratch[slot]);
  c->d_scratch[slot] = nullptr;
  c->scratch_doubles[slot] = 0;
  HFG_CUDA(cudaMalloc((void **)&c->d_scratch[slot], need * sizeof(double)));
  c->scratch_doubles[slot] = need;
  ++c->config_version;  // a captured graph holds the old region
  return HFG_OK;
}

static hfg_status ensure_task_scratch(hfg_ctx *c);
__global__ void compact_screened_tasks(const EngineView v, const ClassLaunch cl, Task *__restrict__ out, int *count);

static hfg_status launch_class(hfg_ctx *c, const QuartetClass &q, const ClassLaunch &cl, int mode, bool ref,
                               int prec, cudaStream_t s, int *launches, int slot = 0) {
  const ClassEntry &e = kClasses[q.cls];
  if (class_on_warp(c, q.cls) && mode != kBlock) {
    kWarp[q.cls](c->view(), cl, mode, ref, prec, 0, s);
    ++*launches;
    return HFG_OK;
  }
  if (!kSplit[q.cls]) {
    e.launch(c->view(), cl, mode, ref, prec, grid_for(c, cl.ntasks, q.cls), s);
    ++*launches;
    return HFG_OK;
  }
  const size_t acc = (size_t)ncomp_range(e.la, e.la + e.lb) * ncomp_range(e.lc, e.lc + e.ld);
  size_t need = 0;
  int chunk_tasks = 1;
  split_chunking(c, q.cls, cl.ntasks, ref, &need, &chunk_tasks);
  hfg_status st = grow_scratch(c, slot, need);
  if (st != HFG_OK) return st;
  for (int t0 = 0; t0 < cl.ntasks; t0 += chunk_tasks) {
    SplitChunk ch{};
    ch.ntasks = std::min(chunk_tasks, cl.ntasks - t0);
    ch.task0 = t0;
    ch.stride = (long long)ch.ntasks * 32;
    ch.scr_fwd = c->d_scratch[slot];
    ch.scr_rev = c->d_scratch[slot] + acc * (size_t)ch.stride;
    kSplit[q.cls](c->view(), cl, ch, mode, ref, prec, s);
    *launches += 2;
  }
  return HFG_OK;
}

// Direct J/K build: all classes on `s`, then G.  The plain form reads the
// full density; the precision form (see hfg_opts) first forms the density
// difference (incremental), the shell-block maxima for the density
// screening, and accumulates G onto the previous one.
static hfg_status direct_build_body(hfg_ctx *c, bool uhf, const double *dPa, const double *dPb, double *dGa,
                                    double *dGb, cudaStream_t s, bool capturing) {
  if (c->batch) return fail(HFG_INVALID_ARG, "batched context: use hfg_fock_rhf/uhf_batch_device");
  const size_t nn = (size_t)c->nbf * c->nbf;
  const int n = c->nbf;
  hfg_status st;
  if ((st = ensure(&c->d_J, nn)) != HFG_OK || (st = ensure(&c->d_Ka, nn)) != HFG_OK) return st;
  if (uhf && ((st = ensure(&c->d_Kb, nn)) != HFG_OK || (st = ensure(&c->d_Pt, nn)) != HFG_OK)) return st;
  const bool precise = c->precision_form();
  const bool incremental = precise && c->opts.incremental;
  const bool fresh = !c->inc_valid || c->inc_uhf != uhf;
  const int eg = std::max(1, std::min(1024, (int)((nn + 255) / 256)));
  int launches = 2;
  const double *Da = dPa, *Db = dPb;
  if (precise) {
    const int ns = c->nshells;
    if (!c->d_shell_dmax) HFG_CUDA(cudaMalloc((void **)&c->d_shell_dmax, (size_t)ns * ns * sizeof(float)));
    if (!c->d_counters) HFG_CUDA(cudaMalloc((void **)&c->d_counters, 2 * sizeof(unsigned long long)));
    HFG_CUDA(cudaMemsetAsync(c->d_counters, 0, 2 * sizeof(unsigned long long), s));
    if (incremental) {
      for (int k = 0; k < (uhf ? 2 : 1); ++k)
        if ((st = ensure(&c->d_prev_P[k], nn)) != HFG_OK || (st = ensure(&c->d_prev_G[k], nn)) != HFG_OK ||
            (st = ensure(&c->d_dP[k], nn)) != HFG_OK)
          return st;
      density_difference<<<eg, 256, 0, s>>>(dPa, c->d_prev_P[0], c->d_dP[0], (int)nn, fresh);
      Da = c->d_dP[0];
      ++launches;
      if (uhf) {
        density_difference<<<eg, 256, 0, s>>>(dPb, c->d_prev_P[1], c->d_dP[1], (int)nn, fresh);
        Db = c->d_dP[1];
        ++launches;
      }
    }
    const int sg = std::max(1, std::min(4096, (ns * ns + 255) / 256));
    shell_block_max<<<sg, 256, 0, s>>>(Da, uhf ? Db : nullptr, c->d_shell_ao, c->d_shell_nf, ns, n, c->d_shell_dmax);
    launches += 2;
  }
  HFG_CUDA(cudaMemsetAsync(c->d_J, 0, nn * sizeof(double), s));
  HFG_CUDA(cudaMemsetAsync(c->d_Ka, 0, nn * sizeof(double), s));
  if (uhf) {
    HFG_CUDA(cudaMemsetAsync(c->d_Kb, 0, nn * sizeof(double), s));
    add_densities<<<256, 256, 0, s>>>(Da, Db, c->d_Pt, (int)nn);
    launches += 2;
  }
  const bool ref = c->opts.eri_convention == HFG_ERI_REFERENCE;
  const size_t nq = c->qclasses.size();
  // density-screened builds first compact each fused / warp class's tasks to
  // those with a quartet above the threshold (late incremental builds keep
  // a small fraction); the class kernels then take them from the queue
  const bool compact = precise && c->use_compaction && nq > 0;
  if ((c->use_queue || compact) && nq > 0) {
    if ((st = ensure_task_scratch(c)) != HFG_OK) return st;
    HFG_CUDA(cudaMemsetAsync(c->d_queue, 0, nq * sizeof(int), s));
    ++launches;
    if (compact) {
      HFG_CUDA(cudaMemsetAsync(c->d_task_counts, 0, nq * sizeof(int), s));
      ++launches;
    }
  }
  ClassStreams cs{c, s, c->use_streams && !c->profiling};
  {
    std::vector<int> nt(c->qclasses.size());
    for (size_t i = 0; i < nt.size(); ++i) nt[i] = base_launch(c, c->qclasses[i], true).ntasks;
    if ((st = cs.presize(nt, ref)) != HFG_OK) return st;
  }
  if (!capturing) HFG_CUDA(cudaEventRecord(c->ev0, s));
  if ((st = cs.fork()) != HFG_OK) return st;
  const int prec = !precise ? 0 : c->mixed_cutoff > 0 ? 2 : 1;
  c->stats = hfg_stats{};
  for (size_t qi = 0; qi < nq; ++qi) {
    QuartetClass &q = c->qclasses[qi];
    ClassLaunch cl = base_launch(c, q, true);
    if (c->profiling) HFG_CUDA(cudaEventRecord(q.ev_a, s));
    cl.Da = Da;
    cl.Db = Db;
    cl.Dt = uhf ? c->d_Pt : Da;
    cl.J = c->d_J;
    cl.Ka = c->d_Ka;
    cl.Kb = c->d_Kb;
    cl.dens_threshold = (float)c->density_threshold();
    cl.mixed_cutoff = (float)c->mixed_cutoff;
    cl.counters = precise ? c->d_counters : nullptr;
    if (cl.ntasks > 0) {
      const cudaStream_t cls_stream = cs.pick(uses_split(c, q.cls));
      ClassLaunch cll = cl;
      if ((c->use_queue || compact) && !uses_split(c, q.cls)) cll.queue = c->d_queue + qi;
      if (compact && !uses_split(c, q.cls)) {
        const int cg = std::max(1, std::min(c->num_sms * 8, (cl.ntasks + 7) / 8));
        compact_screened_tasks<<<cg, 256, 0, cls_stream>>>(c->view(), cl, c->d_task_active + c->task_base[qi],
                                                            c->d_task_counts + qi);
        ++launches;
        cll.tasks = c->d_task_active + c->task_base[qi];
        cll.task_offset = 0;
        cll.task_stride = 1;
        cll.ntasks_dev = c->d_task_counts + qi;  // cll.ntasks stays the bound the grid is sized from
      }
      st = launch_class(c, q, cll, uhf ? kJkUhf : kJkRhf, ref, prec, cls_stream, &launches, cs.slot);
      if (st != HFG_OK) return st;
    }
    if (c->profiling) HFG_CUDA(cudaEventRecord(q.ev_b, s));
    // a shard's share of the class, in proportion to its estimated cost
    const double share = launch_share(q, cl);
    c->stats.shell_quartets += (int64_t)(share * (double)q.shell_quartets + 0.5);
    c->stats.function_quartets += (int64_t)(share * (double)q.function_quartets + 0.5);
    c->stats.primitive_quartets += (int64_t)(share * (double)q.prim_quartets + 0.5);
    c->stats.flops += share * q.flops;
  }
  HFG_CUDA(cudaGetLastError());
  if ((st = cs.join()) != HFG_OK) return st;
  if (!capturing) HFG_CUDA(cudaEventRecord(c->ev1, s));
  const int fg = std::max(1, std::min(1024, (int)((nn + 255) / 256)));
  if (incremental) {
    if (uhf)
      finalize_uhf_incremental<<<fg, 256, 0, s>>>(c->d_J, c->d_Ka, c->d_Kb, c->d_prev_G[0], c->d_prev_G[1], dGa, dGb,
                                                  n, !fresh);
    else
      finalize_rhf_incremental<<<fg, 256, 0, s>>>(c->d_J, c->d_Ka, c->d_prev_G[0], dGa, n, !fresh);
    c->inc_valid = true;
    c->inc_uhf = uhf;
  } else if (uhf) {
    finalize_uhf<<<fg, 256, 0, s>>>(c->d_J, c->d_Ka, c->d_Kb, dGa, dGb, n);
  } else {
    finalize_rhf<<<fg, 256, 0, s>>>(c->d_J, c->d_Ka, dGa, n);
  }
  ++launches;
  HFG_CUDA(cudaGetLastError());
  if (!capturing) HFG_CUDA(cudaEventRecord(c->ev_done, s));
  c->stats.kernel_launches = launches;
  c->stats.shell_pairs = c->npairs;
  c->counted = precise;
  if (!precise) c->stats.fp64_shell_quartets = c->stats.shell_quartets;
  return HFG_OK;
}

// Direct build, through a CUDA graph where it can be: the plain form (no
// profiling, a created stream) with graphs on.  The first build with given
// buffers, stream and settings runs normally (and sizes every buffer); the
// second is captured and instantiated; later ones replay the graph.  Any
// change of buffers, stream or settings starts over.
static hfg_status direct_build(hfg_ctx *c, bool uhf, const double *dPa, const double *dPb, double *dGa, double *dGb,
                               cudaStream_t s) {
  const bool graphable = c->use_graphs && !c->batch && !c->precision_form() && !c->profiling && s != nullptr &&
                         s != cudaStreamLegacy && s != cudaStreamPerThread;
  if (!graphable) return direct_build_body(c, uhf, dPa, dPb, dGa, dGb, s, false);
  hfg_ctx::GraphKey key;
  key.uhf = uhf;
  key.pa = dPa;
  key.pb = dPb;
  key.ga = dGa;
  key.gb = dGb;
  key.s = s;
  key.version = c->config_version;
  if (!(c->graph_exec && c->graph_key == key) && c->graph_seen_valid && c->graph_seen == key) {
    if (c->graph_exec) {
      cudaGraphExecDestroy(c->graph_exec);
      c->graph_exec = nullptr;
    }
    HFG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const hfg_status st = direct_build_body(c, uhf, dPa, dPb, dGa, dGb, s, true);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s, &g);
    if (st == HFG_OK && e == cudaSuccess && g) {
      if (cudaGraphInstantiate(&c->graph_exec, g, 0) != cudaSuccess) c->graph_exec = nullptr;
      c->graph_key = key;
      c->graph_stats = c->stats;
    }
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();  // a failed capture leaves nothing behind: build normally below
    if (st != HFG_OK) return st;
  }
  if (c->graph_exec && c->graph_key == key) {
    HFG_CUDA(cudaEventRecord(c->ev0, s));
    HFG_CUDA(cudaGraphLaunch(c->graph_exec, s));
    HFG_CUDA(cudaEventRecord(c->ev1, s));
    HFG_CUDA(cudaEventRecord(c->ev_done, s));
    c->stats = c->graph_stats;
    return HFG_OK;
  }
  c->graph_seen = key;
  c->graph_seen_valid = true;
  return direct_build_body(c, uhf, dPa, dPb, dGa, dGb, s, false);
}

// Batched contexts: G of every active molecule, blockIdx.y = molecule.
__global__ void finalize_rhf_batch(const double *J, const double *K, double *G, const int *nbf,
                                   const long long *off, const unsigned char *active) {
  const int m = blockIdx.y;
  if (!active[m]) return;
  const int n = nbf[m];
  const long long b = off[m];
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n * n; x += gridDim.x * blockDim.x) {
    const int i = x / n, j = x - i * n;
    G[b + x] = (J[b + i * n + j] + J[b + j * n + i]) - 0.5 * (K[b + i * n + j] + K[b + j * n + i]);
  }
}

__global__ void finalize_uhf_batch(const double *J, const double *Ka, const double *Kb, double *Ga, double *Gb,
                                   const int *nbf, const long long *off, const unsigned char *active) {
  const int m = blockIdx.y;
  if (!active[m]) return;
  const int n = nbf[m];
  const long long b = off[m];
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n * n; x += gridDim.x * blockDim.x) {
    const int i = x / n, j = x - i * n;
    const double jv = J[b + i * n + j] + J[b + j * n + i];
    Ga[b + x] = jv - (Ka[b + i * n + j] + Ka[b + j * n + i]);
    Gb[b + x] = jv - (Kb[b + i * n + j] + Kb[b + j * n + i]);
  }
}

// Tasks of active molecules, in the class's order up to warp-sized groups:
// each warp writes its kept tasks as one contiguous run (ballot + one
// atomic per warp).
// Device lists of compacted tasks (one region per quartet class, as long as
// the class's task list), their counts and work-queue counters; allocated by
// the first build that compacts, freed when the task lists are rebuilt.
static hfg_status ensure_task_scratch(hfg_ctx *c) {
  const size_t nq = c->qclasses.size();
  if (!c->d_task_active) {
    size_t total = 0;
    c->task_base.assign(nq, 0);
    for (size_t i = 0; i < nq; ++i) {
      c->task_base[i] = (int)total;
      total += c->qclasses[i].tasks.size();
    }
    HFG_CUDA(cudaMalloc((void **)&c->d_task_active, std::max<size_t>(1, total) * sizeof(Task)));
    HFG_CUDA(cudaMalloc((void **)&c->d_task_counts, std::max<size_t>(1, nq) * sizeof(int)));
  }
  if (!c->d_queue) HFG_CUDA(cudaMalloc((void **)&c->d_queue, std::max<size_t>(1, nq) * sizeof(int)));
  return HFG_OK;
}

__global__ void compact_active_tasks(const Task *__restrict__ tasks, int ntasks, const int *__restrict__ bra_list,
                                     const int *__restrict__ pair_mol, const unsigned char *__restrict__ active,
                                     Task *__restrict__ out, int *count) {
  const int lane = threadIdx.x & 31;
  for (int base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31; base < ntasks; base += gridDim.x * blockDim.x) {
    const int t = base + lane;
    bool keep = false;
    Task tk{};
    if (t < ntasks) {
      tk = tasks[t];
      keep = active[pair_mol[bra_list[tk.bra_pos]]] != 0;
    }
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    int at = 0;
    if (lane == 0 && m) at = atomicAdd(count, __popc(m));
    at = __shfl_sync(0xffffffffu, at, 0);
    if (keep) out[at + __popc(m & ((1u << lane) - 1))] = tk;
  }
}

// Density-screened builds: the tasks of one class launch (its shard range)
// with at least one quartet whose density-weighted bound reaches the
// threshold -- the test the class kernels apply per lane (screen_task) -- in
// task order within each warp's group, appended to `out`; `count` ends as
// their number.  One warp per task.
__global__ void compact_screened_tasks(const EngineView v, const ClassLaunch cl, Task *__restrict__ out,
                                       int *count) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < cl.ntasks; t += warps) {
    const Task task = launch_task(cl, t);
    const int bp = cl.bra_list[task.bra_pos];
    bool keep = false;
    for (int k = task.ket_start + lane; k < task.ket_end; k += 32)
      keep = keep || density_bound(v, bp, cl.ket_list[k]) >= cl.dens_threshold;
    if (__any_sync(0xffffffffu, keep) && lane == 0) out[atomicAdd(count, 1)] = task;
  }
}

// Direct J/K build of a batched context: one launch per quartet class over
// the tasks of all molecules (inactive molecules' tasks exit at once), then
// G per active molecule.  `active`: host flags per molecule, or null = all.
static hfg_status batch_build(hfg_ctx *c, bool uhf, const double *dPa, const double *dPb, double *dGa, double *dGb,
                              const unsigned char *active, cudaStream_t s) {
  const size_t tot = (size_t)c->batch_elems;
  hfg_status st;
  if ((st = ensure(&c->d_J, tot)) != HFG_OK || (st = ensure(&c->d_Ka, tot)) != HFG_OK) return st;
  if (uhf && ((st = ensure(&c->d_Kb, tot)) != HFG_OK || (st = ensure(&c->d_Pt, tot)) != HFG_OK)) return st;
  const std::vector<unsigned char> all(c->nmol, 1);
  HFG_CUDA(cudaMemcpyAsync(c->d_mol_active, active ? active : all.data(), c->nmol, cudaMemcpyHostToDevice, s));
  HFG_CUDA(cudaMemsetAsync(c->d_J, 0, tot * sizeof(double), s));
  HFG_CUDA(cudaMemsetAsync(c->d_Ka, 0, tot * sizeof(double), s));
  int launches = 2;
  if (uhf) {
    HFG_CUDA(cudaMemsetAsync(c->d_Kb, 0, tot * sizeof(double), s));
    add_densities<<<std::max(1, std::min(1024, (int)((tot + 255) / 256))), 256, 0, s>>>(dPa, dPb, c->d_Pt, (int)tot);
    launches += 2;
  }
  // with converged molecules, launch over the active molecules' tasks only
  // (compacted on the device; one sync for the counts) instead of letting
  // every warp read and skip the others'
  bool compact = false;
  std::vector<int> counts;
  if (active && c->shard_count == 1) {
    int nact = 0;
    for (int m = 0; m < c->nmol; ++m) nact += active[m] != 0;
    compact = nact < c->nmol;
  }
  if (compact) {
    const size_t nq = c->qclasses.size();
    if ((st = ensure_task_scratch(c)) != HFG_OK) return st;
    HFG_CUDA(cudaMemsetAsync(c->d_task_counts, 0, nq * sizeof(int), s));
    for (size_t i = 0; i < nq; ++i) {
      const QuartetClass &q = c->qclasses[i];
      const int nt = (int)q.tasks.size();
      if (nt == 0) continue;
      const int grid = std::max(1, std::min(c->num_sms * 8, (nt + 255) / 256));
      compact_active_tasks<<<grid, 256, 0, s>>>(q.d_tasks, nt, c->pclass[q.bra_pc].d_pairs, c->d_pair_mol,
                                                c->d_mol_active, c->d_task_active + c->task_base[i],
                                                c->d_task_counts + i);
      ++launches;
    }
    counts.assign(nq, 0);
    HFG_CUDA(cudaMemcpyAsync(counts.data(), c->d_task_counts, nq * sizeof(int), cudaMemcpyDeviceToHost, s));
    HFG_CUDA(cudaStreamSynchronize(s));
  }
  const bool ref = c->opts.eri_convention == HFG_ERI_REFERENCE;
  ClassStreams cs{c, s, c->use_streams && !c->profiling};
  {
    std::vector<int> nt(c->qclasses.size());
    for (size_t i = 0; i < nt.size(); ++i) nt[i] = compact ? counts[i] : base_launch(c, c->qclasses[i], true).ntasks;
    if ((st = cs.presize(nt, ref)) != HFG_OK) return st;
  }
  HFG_CUDA(cudaEventRecord(c->ev0, s));
  if ((st = cs.fork()) != HFG_OK) return st;
  c->stats = hfg_stats{};
  for (size_t qi = 0; qi < c->qclasses.size(); ++qi) {
    auto &q = c->qclasses[qi];
    ClassLaunch cl = base_launch(c, q, true);
    if (compact) {
      cl.tasks = c->d_task_active + c->task_base[qi];
      cl.task_offset = 0;
      cl.task_stride = 1;
      cl.ntasks = counts[qi];
    }
    if (c->profiling) HFG_CUDA(cudaEventRecord(q.ev_a, s));
    cl.Da = dPa;
    cl.Db = dPb;
    cl.Dt = uhf ? c->d_Pt : dPa;
    cl.J = c->d_J;
    cl.Ka = c->d_Ka;
    cl.Kb = c->d_Kb;
    if (cl.ntasks > 0) {
      const cudaStream_t cls_stream = cs.pick(uses_split(c, q.cls));
      st = launch_class(c, q, cl, uhf ? kJkUhf : kJkRhf, ref, 0, cls_stream, &launches, cs.slot);
      if (st != HFG_OK) return st;
    }
    if (c->profiling) HFG_CUDA(cudaEventRecord(q.ev_b, s));
    c->stats.shell_quartets += q.shell_quartets;
    c->stats.function_quartets += q.function_quartets;
    c->stats.primitive_quartets += q.prim_quartets;
    c->stats.flops += q.flops;
  }
  HFG_CUDA(cudaGetLastError());
  if ((st = cs.join()) != HFG_OK) return st;
  HFG_CUDA(cudaEventRecord(c->ev1, s));
  int nmax = 0;
  for (int n : c->mol_nbf) nmax = std::max(nmax, n);
  const dim3 fg(std::max(1, std::min(64, (nmax * nmax + 255) / 256)), c->nmol);
  if (uhf)
    finalize_uhf_batch<<<fg, 256, 0, s>>>(c->d_J, c->d_Ka, c->d_Kb, dGa, dGb, c->d_mol_nbf, c->d_mol_off,
                                          c->d_mol_active);
  else
    finalize_rhf_batch<<<fg, 256, 0, s>>>(c->d_J, c->d_Ka, dGa, c->d_mol_nbf, c->d_mol_off, c->d_mol_active);
  ++launches;
  HFG_CUDA(cudaGetLastError());
  HFG_CUDA(cudaEventRecord(c->ev_done, s));
  c->stats.kernel_launches = launches;
  c->stats.shell_pairs = c->npairs;
  c->stats.fp64_shell_quartets = c->stats.shell_quartets;
  c->counted = false;
  return HFG_OK;
}

// Batched build with no host synchronisation (the batched SCF captures it in
// a CUDA graph): the active mask is read from device memory, every class's
// active tasks are compacted on the device and the class kernels take them
// from a device work queue (count and counter in device memory, one fixed
// grid per class), then G per active molecule.  The large classes run the
// warp-cooperative kernels whatever the context's per-class choice (no
// scratch, no host-sized chunks).  Buffers are allocated by the first call.
static hfg_status batch_build_async(hfg_ctx *c, bool uhf, const double *dPa, const double *dPb, double *dGa,
                                    double *dGb, const unsigned char *d_active, cudaStream_t s) {
  const size_t tot = (size_t)c->batch_elems;
  const size_t nq = c->qclasses.size();
  hfg_status st;
  if ((st = ensure(&c->d_J, tot)) != HFG_OK || (st = ensure(&c->d_Ka, tot)) != HFG_OK) return st;
  if (uhf && ((st = ensure(&c->d_Kb, tot)) != HFG_OK || (st = ensure(&c->d_Pt, tot)) != HFG_OK)) return st;
  if ((st = ensure_task_scratch(c)) != HFG_OK) return st;
  HFG_CUDA(cudaMemsetAsync(c->d_J, 0, tot * sizeof(double), s));
  HFG_CUDA(cudaMemsetAsync(c->d_Ka, 0, tot * sizeof(double), s));
  int launches = 2;
  if (uhf) {
    HFG_CUDA(cudaMemsetAsync(c->d_Kb, 0, tot * sizeof(double), s));
    add_densities<<<std::max(1, std::min(1024, (int)((tot + 255) / 256))), 256, 0, s>>>(dPa, dPb, c->d_Pt, (int)tot);
    launches += 2;
  }
  HFG_CUDA(cudaMemsetAsync(c->d_task_counts, 0, nq * sizeof(int), s));
  HFG_CUDA(cudaMemsetAsync(c->d_queue, 0, nq * sizeof(int), s));
  launches += 2;
  for (size_t i = 0; i < nq; ++i) {
    const QuartetClass &q = c->qclasses[i];
    const int nt = (int)q.tasks.size();
    if (nt == 0) continue;
    const int grid = std::max(1, std::min(c->num_sms * 8, (nt + 255) / 256));
    compact_active_tasks<<<grid, 256, 0, s>>>(q.d_tasks, nt, c->pclass[q.bra_pc].d_pairs, c->d_pair_mol, d_active,
                                              c->d_task_active + c->task_base[i], c->d_task_counts + i);
    ++launches;
  }
  EngineView v = c->view();
  v.mol_active = d_active;
  const bool ref = c->opts.eri_convention == HFG_ERI_REFERENCE;
  ClassStreams cs{c, s, c->use_streams && !c->profiling};
  if ((st = cs.fork()) != HFG_OK) return st;
  c->stats = hfg_stats{};
  for (size_t qi = 0; qi < nq; ++qi) {
    auto &q = c->qclasses[qi];
    if (q.tasks.empty()) continue;
    ClassLaunch cl = base_launch(c, q, false);
    cl.tasks = c->d_task_active + c->task_base[qi];
    cl.task_offset = 0;
    cl.task_stride = 1;
    cl.ntasks = (int)q.tasks.size();  // bound: the grid sizes from it
    cl.ntasks_dev = c->d_task_counts + qi;
    cl.queue = c->d_queue + qi;
    cl.Da = dPa;
    cl.Db = dPb;
    cl.Dt = uhf ? c->d_Pt : dPa;
    cl.J = c->d_J;
    cl.Ka = c->d_Ka;
    cl.Kb = c->d_Kb;
    const cudaStream_t cls_stream = cs.pick(false);
    const int mode = uhf ? kJkUhf : kJkRhf;
    if (kWarp[q.cls]) kWarp[q.cls](v, cl, mode, ref, 0, 0, cls_stream);
    else kClasses[q.cls].launch(v, cl, mode, ref, 0, grid_for(c, cl.ntasks, q.cls), cls_stream);
    ++launches;
    c->stats.shell_quartets += q.shell_quartets;
    c->stats.function_quartets += q.function_quartets;
    c->stats.primitive_quartets += q.prim_quartets;
    c->stats.flops += q.flops;
  }
  HFG_CUDA(cudaGetLastError());
  if ((st = cs.join()) != HFG_OK) return st;
  int nmax = 0;
  for (int n : c->mol_nbf) nmax = std::max(nmax, n);
  const dim3 fg(std::max(1, std::min(64, (nmax * nmax + 255) / 256)), c->nmol);
  if (uhf)
    finalize_uhf_batch<<<fg, 256, 0, s>>>(c->d_J, c->d_Ka, c->d_Kb, dGa, dGb, c->d_mol_nbf, c->d_mol_off, d_active);
  else
    finalize_rhf_batch<<<fg, 256, 0, s>>>(c->d_J, c->d_Ka, dGa, c->d_mol_nbf, c->d_mol_off, d_active);
  ++launches;
  HFG_CUDA(cudaGetLastError());
  c->stats.kernel_launches = launches;
  c->stats.shell_pairs = c->npairs;
  c->stats.fp64_shell_quartets = c->stats.shell_quartets;
  c->counted = false;
  return HFG_OK;
}

static hfg_status finish_timing(hfg_ctx *c) {
  HFG_CUDA(cudaEventSynchronize(c->ev1));
  float ms = 0;
  HFG_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->stats.last_build_ms = ms;
  if (c->profiling)
    for (auto &q : c->qclasses) HFG_CUDA(cudaEventElapsedTime(&q.last_ms, q.ev_a, q.ev_b));
  return HFG_OK;
}

static hfg_status stored_build(hfg_ctx *c, double *d_out, int64_t count, cudaStream_t s) {
  if (c->batch) return fail(HFG_INVALID_ARG, "batched context: no stored table");
  HFG_CUDA(cudaMemsetAsync(d_out, 0, (size_t)count * sizeof(double), s));
  HFG_CUDA(cudaEventRecord(c->ev0, s));
  const bool ref = c->opts.eri_convention == HFG_ERI_REFERENCE;
  c->stats = hfg_stats{};
  int launches = 1;
  for (auto &q : c->qclasses) {
    ClassLaunch cl = base_launch(c, q);
    cl.packed = d_out;
    if (c->profiling) HFG_CUDA(cudaEventRecord(q.ev_a, s));
    const hfg_status st = launch_class(c, q, cl, kStorePacked, ref, 0, s, &launches);
    if (st != HFG_OK) return st;
    if (c->profiling) HFG_CUDA(cudaEventRecord(q.ev_b, s));
    c->stats.shell_quartets += q.shell_quartets;
    c->stats.function_quartets += q.function_quartets;
    c->stats.primitive_quartets += q.prim_quartets;
    c->stats.flops += q.flops;
  }
  HFG_CUDA(cudaGetLastError());
  HFG_CUDA(cudaEventRecord(c->ev1, s));
  c->stats.kernel_launches = launches;
  c->stats.shell_pairs = c->npairs;
  c->stats.fp64_shell_quartets = c->stats.shell_quartets;
  c->counted = false;
  return HFG_OK;
}

}  // namespace hfg

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

void hfg_default_opts(hfg_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->schwarz_threshold = 1e-12;
  o->mixed_cutoff = 0.0;
  o->eri_convention = HFG_ERI_REFERENCE;
  o->device = 0;
  o->density_screening = 0;
}

const char *hfg_last_error(void) { return hfg::g_last_error.c_str(); }

int32_t hfg_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

int64_t hfg_packed_size(int32_t n) {
  if (n <= 0) return 0;
  auto tri = [](int64_t a, int64_t b) { return a < b ? b * (b + 1) / 2 + a : a * (a + 1) / 2 + b; };
  return tri(tri(n - 1, n - 1), tri(n - 1, n - 1)) + 1;
}

int32_t hfg_ctx_nbf(const hfg_ctx *c) { return c ? c->nbf : 0; }

}  // extern "C"

// Context over one molecule (shell_mol = nullptr) or over `nmol` molecules
// whose shells `sh` lists one after another (shell_mol[s] = molecule of
// shell s, AO offsets molecule-local, mol_nbf[m] its functions): shell pairs,
// and hence quartets, only within a molecule.
static hfg_status create_context(const hfg_shells *sh, const int *shell_mol, int nmol, const int *mol_nbf,
                                 const hfg_opts *opts, hfg_ctx **out) {
  using namespace hfg;
  if (!out) return fail(HFG_INVALID_ARG, "out is null");
  *out = nullptr;
  if (!sh || sh->nshells <= 0 || !sh->center || !sh->L || !sh->nprim || !sh->prim_offset || !sh->ao_offset ||
      !sh->exponent || !sh->coefficient || (!shell_mol && sh->nbf <= 0))
    return fail(HFG_INVALID_ARG, "incomplete hfg_shells");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(HFG_NO_DEVICE, "no CUDA device");
  auto ctx = std::make_unique<hfg_ctx>();
  if (opts) ctx->opts = *opts;
  else hfg_default_opts(&ctx->opts);
  if (ctx->opts.device < 0 || ctx->opts.device >= ndev) return fail(HFG_INVALID_ARG, "device out of range");
  if (!(ctx->opts.schwarz_threshold >= 0)) return fail(HFG_INVALID_ARG, "negative screening threshold");
  ctx->device = ctx->opts.device;
  HFG_CUDA(cudaSetDevice(ctx->device));
  HFG_CUDA(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->device));
  ctx->use_graphs = ctx->opts.cuda_graphs != 0;
  ctx->use_streams = ctx->opts.concurrent_classes != 0;
  // tuning: HFG_BLOCKS_PER_SM overrides the grid cap (every block stages the
  // class's Boys table once, so fewer, longer-lived blocks stage it less)
  if (const char *e = std::getenv("HFG_BLOCKS_PER_SM")) ctx->blocks_per_sm = std::max(1, std::atoi(e));
  // tuning: HFG_PRIM_TARGET sets the lane-group target (0: one lane per quartet)
  if (const char *e = std::getenv("HFG_PRIM_TARGET")) ctx->prim_target = std::max(0, std::atoi(e));
  // default kernel per large class: the warp-cooperative kernel where one
  // quartet's primitive work fills a warp -- (dd|dd), 1296 Cartesian
  // components -- the split path for the rest; HFG_SPLIT_PATH=1 / HFG_WARP_PATH=1
  // put every large class on one of them
  for (int k = 0; k < kNumClasses; ++k) {
    const ClassEntry &e = kClasses[k];
    ctx->warp_class[k] = kWarp[k] && e.la + e.lb + e.lc + e.ld >= 8 ? 1 : 0;
  }
  if (const char *e = std::getenv("HFG_WORK_QUEUE")) ctx->use_queue = std::atoi(e) != 0;
  if (const char *e = std::getenv("HFG_NO_COMPACT")) ctx->use_compaction = std::atoi(e) == 0;
  // tuning: HFG_SCRATCH_MB bounds the split path's scratch (all regions together)
  if (const char *e = std::getenv("HFG_SCRATCH_MB")) ctx->scratch_budget_bytes = size_t(std::max(16, std::atoi(e))) << 20;
  if (const char *e = std::getenv("HFG_SPLIT_PATH"); e && std::atoi(e) != 0)
    std::fill(std::begin(ctx->warp_class), std::end(ctx->warp_class), int8_t(0));
  if (const char *e = std::getenv("HFG_WARP_PATH"); e && std::atoi(e) != 0)
    std::fill(std::begin(ctx->warp_class), std::end(ctx->warp_class), int8_t(1));
  ctx->batch = shell_mol != nullptr;
  ctx->nmol = ctx->batch ? nmol : 1;
  ctx->nbf = ctx->batch ? 0 : sh->nbf;
  const int ns = sh->nshells;
  ctx->shells.resize(ns);
  std::vector<int64_t> funcs(ctx->nmol, 0);
  for (int s = 0; s < ns; ++s) {
    HostShell &h = ctx->shells[s];
    for (int d = 0; d < 3; ++d) h.c[d] = sh->center[3 * s + d];
    h.L = sh->L[s];
    h.nprim = sh->nprim[s];
    h.prim_off = sh->prim_offset[s];
    h.ao = sh->ao_offset[s];
    const int m = ctx->batch ? shell_mol[s] : 0;
    const int mnbf = ctx->batch ? mol_nbf[m] : sh->nbf;
    if (h.L < 0 || h.L > kMaxL) return fail(HFG_UNSUPPORTED_L, "shell angular momentum above d");
    if (h.nprim <= 0 || h.prim_off < 0) return fail(HFG_INVALID_ARG, "shell without primitives");
    if (h.ao < 0 || h.ao + ncart_h(h.L) > mnbf) return fail(HFG_INVALID_ARG, "AO offset outside nbf");
    funcs[m] += ncart_h(h.L);
  }
  for (int m = 0; m < ctx->nmol; ++m)
    if (funcs[m] != (ctx->batch ? mol_nbf[m] : sh->nbf))
      return fail(HFG_INVALID_ARG, "shell functions do not sum to nbf");
  if (!(ctx->opts.mixed_cutoff >= 0) || !(ctx->opts.mixed_cutoff < 1e300) || !(ctx->opts.density_threshold >= 0))
    return fail(HFG_INVALID_ARG, "mixed cutoff and density threshold must be finite and >= 0");
  ctx->mixed_cutoff = ctx->opts.mixed_cutoff;
  ctx->nshells = ns;
  {
    std::vector<int> sao(ns), snf(ns);
    for (int s = 0; s < ns; ++s) {
      sao[s] = ctx->shells[s].ao;
      snf[s] = ncart_h(ctx->shells[s].L);
    }
    hfg_status st0;
    if ((st0 = upload(&ctx->d_shell_ao, sao)) != HFG_OK || (st0 = upload(&ctx->d_shell_nf, snf)) != HFG_OK) return st0;
  }

  // ---- shell pairs (a >= b, same molecule; one molecule: pair index
  // a*(a+1)/2 + b) and their primitive pairs
  std::vector<std::pair<int, int>> plist;
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b <= a; ++b)
      if (!ctx->batch || shell_mol[a] == shell_mol[b]) plist.emplace_back(a, b);
  const int np = (int)plist.size();
  ctx->npairs = np;
  if (ctx->batch) {
    ctx->pair_mol.resize(np);
    for (int p = 0; p < np; ++p) ctx->pair_mol[p] = shell_mol[plist[p].first];
  }
  std::vector<PrimPair> prim;
  std::vector<int> poff(np), pn(np), psa(np), psb(np), paoa(np), paob(np);
  std::vector<double> pab(3 * (size_t)np);
  ctx->pair_sa.resize(np);
  ctx->pair_sb.resize(np);
  ctx->pair_cls.resize(np);
  const double sqrt2pi54 = std::sqrt(2.0) * std::pow(M_PI, 1.25);
  for (int p = 0; p < np; ++p) {
    {
      const int a = plist[p].first, b = plist[p].second;
      int f = a, g = b;
      if (ctx->shells[b].L > ctx->shells[a].L) std::swap(f, g);  // first = higher L, else higher index
      const HostShell &A = ctx->shells[f], &B = ctx->shells[g];
      psa[p] = f;
      psb[p] = g;
      ctx->pair_sa[p] = f;
      ctx->pair_sb[p] = g;
      paoa[p] = A.ao;
      paob[p] = B.ao;
      ctx->pair_cls[p] = pair_class_index(A.L, B.L);
      double AB[3], ab2 = 0;
      for (int d = 0; d < 3; ++d) {
        AB[d] = A.c[d] - B.c[d];
        pab[3 * (size_t)p + d] = AB[d];
        ab2 += AB[d] * AB[d];
      }
      poff[p] = (int)prim.size();
      for (int i = 0; i < A.nprim; ++i)
        for (int j = 0; j < B.nprim; ++j) {
          const double al = sh->exponent[A.prim_off + i], be = sh->exponent[B.prim_off + j];
          // L-dependent part of GaussianOrbital::getNormalizationFactor
          // (GaussianOrbital.cpp:25-30): (2a/pi)^(3/4) (4a)^(L/2)
          const double na = std::pow(2 * al / M_PI, 0.75) * std::pow(4 * al, A.L / 2.0);
          const double nb = std::pow(2 * be / M_PI, 0.75) * std::pow(4 * be, B.L / 2.0);
          const double ca = sh->coefficient[A.prim_off + i] * na, cb = sh->coefficient[B.prim_off + j] * nb;
          PrimPair pp;
          pp.zeta = al + be;
          pp.inv_zeta = 1.0 / pp.zeta;
          const double P[3] = {(al * A.c[0] + be * B.c[0]) * pp.inv_zeta, (al * A.c[1] + be * B.c[1]) * pp.inv_zeta,
                               (al * A.c[2] + be * B.c[2]) * pp.inv_zeta};
          pp.Px = P[0];
          pp.Py = P[1];
          pp.Pz = P[2];
          pp.PAx = P[0] - A.c[0];
          pp.PAy = P[1] - A.c[1];
          pp.PAz = P[2] - A.c[2];
          pp.bABx = be * AB[0];
          pp.bABy = be * AB[1];
          pp.bABz = be * AB[2];
          pp.K = ca * cb * std::exp(-al * be * pp.inv_zeta * ab2) * sqrt2pi54 * pp.inv_zeta;
          prim.push_back(pp);
        }
      pn[p] = (int)prim.size() - poff[p];
    }
  }
  // Primitive-pair screening: drop primitive pairs whose largest possible
  // quartet contribution, |K_ab| max|K| / sqrt(zeta_ab + min zeta), is below
  // 1e-21 (recursion factors cannot lift that to the 1e-15 level).  Mostly
  // tight-exponent pairs on distant atoms, about 60% of all for water clusters.
  {
    double kmax = 0, zmin = 1e300;
    for (const PrimPair &pp : prim) {
      kmax = std::max(kmax, std::fabs(pp.K));
      zmin = std::min(zmin, pp.zeta);
    }
    std::vector<PrimPair> kept;
    kept.reserve(prim.size());
    for (int p = 0; p < np; ++p) {
      const int o = poff[p], cnt = pn[p];
      poff[p] = (int)kept.size();
      for (int x = o; x < o + cnt; ++x)
        if (std::fabs(prim[x].K) * kmax / std::sqrt(prim[x].zeta + zmin) >= 1e-21) kept.push_back(prim[x]);
      pn[p] = (int)kept.size() - poff[p];
    }
    prim.swap(kept);
    if (prim.empty()) prim.push_back(PrimPair{});  // keep a valid device allocation
  }
  ctx->pair_nprim = pn;
  std::vector<PrimPairF> primf(prim.size());
  for (size_t x = 0; x < prim.size(); ++x) {
    const PrimPair &d = prim[x];
    primf[x] = PrimPairF{(float)d.zeta, (float)d.Px,   (float)d.Py,   (float)d.Pz, (float)d.PAx,     (float)d.PAy,
                         (float)d.PAz,  (float)d.bABx, (float)d.bABy, (float)d.bABz, (float)d.K, (float)d.inv_zeta};
  }
  hfg_status st;
  if ((st = upload(&ctx->d_prim, prim)) != HFG_OK || (st = upload(&ctx->d_primf, primf)) != HFG_OK ||
      (st = upload(&ctx->d_pair_prim_off, poff)) != HFG_OK ||
      (st = upload(&ctx->d_pair_nprim, pn)) != HFG_OK || (st = upload(&ctx->d_pair_sa, psa)) != HFG_OK ||
      (st = upload(&ctx->d_pair_sb, psb)) != HFG_OK || (st = upload(&ctx->d_pair_ao_a, paoa)) != HFG_OK ||
      (st = upload(&ctx->d_pair_ao_b, paob)) != HFG_OK || (st = upload(&ctx->d_pair_AB, pab)) != HFG_OK ||
      (st = upload(&ctx->d_boys, boys_table_host())) != HFG_OK)
    return st;
  HFG_CUDA(cudaMalloc((void **)&ctx->d_pair_Q, (size_t)np * sizeof(double)));
  HFG_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  HFG_CUDA(cudaEventCreate(&ctx->ev0));
  HFG_CUDA(cudaEventCreate(&ctx->ev1));
  HFG_CUDA(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
  HFG_CUDA(cudaEventCreateWithFlags(&ctx->ev_done, cudaEventDisableTiming));
  for (int i = 0; i < hfg_ctx::kAux; ++i) {
    HFG_CUDA(cudaStreamCreateWithFlags(&ctx->aux[i], cudaStreamNonBlocking));
    HFG_CUDA(cudaEventCreateWithFlags(&ctx->ev_join[i], cudaEventDisableTiming));
  }

  // ---- Schwarz bounds per pair class
  std::vector<std::vector<int>> by_class(kNumPairClasses);
  for (int p = 0; p < np; ++p) by_class[ctx->pair_cls[p]].push_back(p);
  const EngineView v0 = ctx->view();
  std::vector<int *> tmp_lists;
  for (int pc = 0; pc < kNumPairClasses; ++pc) {
    if (by_class[pc].empty()) continue;
    int *d_list = nullptr;
    if ((st = upload(&d_list, by_class[pc])) != HFG_OK) return st;
    tmp_lists.push_back(d_list);
    launch_schwarz(kPairClasses[pc][0], kPairClasses[pc][1], v0, d_list, (int)by_class[pc].size(), ctx->d_pair_Q,
                   ctx->stream);
  }
  HFG_CUDA(cudaGetLastError());
  HFG_CUDA(cudaStreamSynchronize(ctx->stream));
  for (int *l : tmp_lists) cudaFree(l);
  ctx->pair_Q.resize(np);
  HFG_CUDA(cudaMemcpy(ctx->pair_Q.data(), ctx->d_pair_Q, (size_t)np * sizeof(double), cudaMemcpyDeviceToHost));

  // ---- class lists: per molecule, primitive-count buckets, each sorted by
  // Q descending
  const int nmols = ctx->nmol;
  for (int pc = 0; pc < kNumPairClasses; ++pc) {
    PairClassList &L = ctx->pclass[pc];
    L.pairs.clear();
    L.seg_start.assign((size_t)nmols * kBuckets + 1, 0);
    std::vector<std::vector<int>> seg((size_t)nmols * kBuckets);
    for (int p : by_class[pc]) {
      const int m = ctx->pair_mol.empty() ? 0 : ctx->pair_mol[p];
      seg[(size_t)m * kBuckets + prim_bucket(pn[p])].push_back(p);
    }
    for (size_t x = 0; x < seg.size(); ++x) {
      L.seg_start[x] = (int)L.pairs.size();
      std::stable_sort(seg[x].begin(), seg[x].end(),
                       [&](int a, int b) { return ctx->pair_Q[a] > ctx->pair_Q[b]; });
      L.pairs.insert(L.pairs.end(), seg[x].begin(), seg[x].end());
    }
    L.seg_start[seg.size()] = (int)L.pairs.size();
    if ((st = upload(&L.d_pairs, L.pairs)) != HFG_OK) return st;
  }
  build_quartet_classes(ctx.get(), ctx->opts.schwarz_threshold);
  if ((st = upload_classes(ctx.get())) != HFG_OK) return st;
  if (ctx->batch) {
    ctx->mol_nbf.assign(mol_nbf, mol_nbf + nmol);
    ctx->mol_off.resize(nmol);
    long long off = 0;
    for (int m = 0; m < nmol; ++m) {
      ctx->mol_off[m] = off;
      off += (long long)mol_nbf[m] * mol_nbf[m];
    }
    ctx->batch_elems = off;
    const std::vector<unsigned char> all_active(nmol, 1);
    if ((st = upload(&ctx->d_pair_mol, ctx->pair_mol)) != HFG_OK ||
        (st = upload(&ctx->d_mol_nbf, ctx->mol_nbf)) != HFG_OK ||
        (st = upload(&ctx->d_mol_off, ctx->mol_off)) != HFG_OK ||
        (st = upload(&ctx->d_mol_active, all_active)) != HFG_OK)
      return st;
  }
  *out = ctx.release();
  return HFG_OK;
}

extern "C" {

hfg_status hfg_ctx_create(const hfg_shells *sh, const hfg_opts *opts, hfg_ctx **out) {
  return create_context(sh, nullptr, 1, nullptr, opts, out);
}

hfg_status hfg_batch_create(const hfg_shells *mols, int32_t nmol, const hfg_opts *opts, hfg_ctx **out) {
  using namespace hfg;
  if (!out) return fail(HFG_INVALID_ARG, "out is null");
  *out = nullptr;
  if (!mols || nmol <= 0) return fail(HFG_INVALID_ARG, "no molecules");
  hfg_opts o;
  if (opts) o = *opts;
  else hfg_default_opts(&o);
  if (o.density_screening || o.incremental || o.mixed_cutoff > 0)
    return fail(HFG_INVALID_ARG, "batched contexts run the plain FP64 form");
  // one shell list: molecule after molecule, primitives concatenated
  std::vector<double> center, expo, coef;
  std::vector<int32_t> L, nprim, poff, aoff;
  std::vector<int> shell_mol, nbf(nmol);
  for (int m = 0; m < nmol; ++m) {
    const hfg_shells &s = mols[m];
    if (s.nshells <= 0 || !s.center || !s.L || !s.nprim || !s.prim_offset || !s.ao_offset || !s.exponent ||
        !s.coefficient || s.nbf <= 0)
      return fail(HFG_INVALID_ARG, "incomplete hfg_shells of molecule " + std::to_string(m));
    nbf[m] = s.nbf;
    for (int x = 0; x < s.nshells; ++x) {
      if (s.nprim[x] <= 0 || s.prim_offset[x] < 0) return fail(HFG_INVALID_ARG, "shell without primitives");
      center.insert(center.end(), s.center + 3 * x, s.center + 3 * x + 3);
      L.push_back(s.L[x]);
      nprim.push_back(s.nprim[x]);
      poff.push_back((int32_t)expo.size());
      aoff.push_back(s.ao_offset[x]);
      expo.insert(expo.end(), s.exponent + s.prim_offset[x], s.exponent + s.prim_offset[x] + s.nprim[x]);
      coef.insert(coef.end(), s.coefficient + s.prim_offset[x], s.coefficient + s.prim_offset[x] + s.nprim[x]);
      shell_mol.push_back(m);
    }
  }
  const hfg_shells all{(int32_t)L.size(), center.data(), L.data(), nprim.data(), poff.data(), aoff.data(),
                       expo.data(), coef.data(), 0};
  return create_context(&all, shell_mol.data(), nmol, nbf.data(), &o, out);
}

int32_t hfg_batch_size(const hfg_ctx *c) { return c && c->batch ? c->nmol : 0; }

hfg_status hfg_batch_layout(const hfg_ctx *c, int32_t *nbf, int64_t *offset, int64_t *total) {
  if (!c || !c->batch) return hfg::fail(HFG_INVALID_ARG, "not a batched context");
  for (int m = 0; m < c->nmol; ++m) {
    if (nbf) nbf[m] = c->mol_nbf[m];
    if (offset) offset[m] = c->mol_off[m];
  }
  if (total) *total = c->batch_elems;
  return HFG_OK;
}

void hfg_ctx_destroy(hfg_ctx *c) { delete c; }

hfg_status hfg_eri_packed_device(hfg_ctx *c, double *dev_out, int64_t count, void *stream) {
  if (!c || !dev_out) return fail(HFG_INVALID_ARG, "null argument");
  if (count != hfg_packed_size(c->nbf)) return fail(HFG_INVALID_ARG, "count != hfg_packed_size(nbf)");
  HFG_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  hfg_status st = stored_build(c, dev_out, count, s);
  if (st != HFG_OK) return st;
  return finish_timing(c);
}

hfg_status hfg_eri_packed(hfg_ctx *c, double *host_out, int64_t count) {
  if (!c || !host_out) return fail(HFG_INVALID_ARG, "null argument");
  if (count != hfg_packed_size(c->nbf)) return fail(HFG_INVALID_ARG, "count != hfg_packed_size(nbf)");
  HFG_CUDA(cudaSetDevice(c->device));
  double *d = nullptr;
  HFG_CUDA(cudaMalloc((void **)&d, (size_t)count * sizeof(double)));
  hfg_status st = stored_build(c, d, count, c->stream);
  if (st == HFG_OK) st = finish_timing(c);
  if (st == HFG_OK) {
    cudaError_t e = cudaMemcpyAsync(host_out, d, (size_t)count * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) st = fail(HFG_DEVICE_ERROR, cudaGetErrorString(e));
  }
  cudaFree(d);
  return st;
}

hfg_status hfg_fock_rhf_device(hfg_ctx *c, const double *dP, double *dG, void *stream) {
  if (!c || !dP || !dG) return fail(HFG_INVALID_ARG, "null argument");
  HFG_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  hfg_status st = direct_build(c, false, dP, nullptr, dG, nullptr, s);
  if (st != HFG_OK) return st;
  return finish_timing(c);
}

hfg_status hfg_fock_uhf_device(hfg_ctx *c, const double *dPa, const double *dPb, double *dGa, double *dGb,
                               void *stream) {
  if (!c || !dPa || !dPb || !dGa || !dGb) return fail(HFG_INVALID_ARG, "null argument");
  HFG_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  hfg_status st = direct_build(c, true, dPa, dPb, dGa, dGb, s);
  if (st != HFG_OK) return st;
  return finish_timing(c);
}

hfg_status hfg_fock_rhf_batch_device(hfg_ctx *c, const double *dP, double *dG, const uint8_t *active,
                                     void *stream) {
  if (!c || !dP || !dG) return fail(HFG_INVALID_ARG, "null argument");
  if (!c->batch) return fail(HFG_INVALID_ARG, "not a batched context");
  HFG_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  hfg_status st = batch_build(c, false, dP, nullptr, dG, nullptr, active, s);
  if (st != HFG_OK) return st;
  return finish_timing(c);
}

hfg_status hfg_fock_uhf_batch_device(hfg_ctx *c, const double *dPa, const double *dPb, double *dGa, double *dGb,
                                     const uint8_t *active, void *stream) {
  if (!c || !dPa || !dPb || !dGa || !dGb) return fail(HFG_INVALID_ARG, "null argument");
  if (!c->batch) return fail(HFG_INVALID_ARG, "not a batched context");
  HFG_CUDA(cudaSetDevice(c->device));
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  hfg_status st = batch_build(c, true, dPa, dPb, dGa, dGb, active, s);
  if (st != HFG_OK) return st;
  return finish_timing(c);
}

hfg_status hfg_fock_rhf_batch_async(hfg_ctx *c, const double *dP, double *dG, const uint8_t *d_active,
                                    void *stream) {
  if (!c || !dP || !dG || !d_active) return fail(HFG_INVALID_ARG, "null argument");
  if (!c->batch) return fail(HFG_INVALID_ARG, "not a batched context");
  HFG_CUDA(cudaSetDevice(c->device));
  return batch_build_async(c, false, dP, nullptr, dG, nullptr, d_active, stream ? (cudaStream_t)stream : c->stream);
}

hfg_status hfg_fock_uhf_batch_async(hfg_ctx *c, const double *dPa, const double *dPb, double *dGa, double *dGb,
                                    const uint8_t *d_active, void *stream) {
  if (!c || !dPa || !dPb || !dGa || !dGb || !d_active) return fail(HFG_INVALID_ARG, "null argument");
  if (!c->batch) return fail(HFG_INVALID_ARG, "not a batched context");
  HFG_CUDA(cudaSetDevice(c->device));
  return batch_build_async(c, true, dPa, dPb, dGa, dGb, d_active, stream ? (cudaStream_t)stream : c->stream);
}

hfg_status hfg_fock_rhf(hfg_ctx *c, const double *P, double *G) {
  if (!c || !P || !G) return fail(HFG_INVALID_ARG, "null argument");
  HFG_CUDA(cudaSetDevice(c->device));
  const size_t nn = (size_t)c->nbf * c->nbf;
  hfg_status st;
  if ((st = ensure(&c->d_P, nn)) != HFG_OK || (st = ensure(&c->d_G, nn)) != HFG_OK) return st;
  HFG_CUDA(cudaMemcpyAsync(c->d_P, P, nn * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if ((st = direct_build(c, false, c->d_P, nullptr, c->d_G, nullptr, c->stream)) != HFG_OK) return st;
  HFG_CUDA(cudaMemcpyAsync(G, c->d_G, nn * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HFG_CUDA(cudaStreamSynchronize(c->stream));
  return finish_timing(c);
}

hfg_status hfg_fock_uhf(hfg_ctx *c, const double *Pa, const double *Pb, double *Ga, double *Gb) {
  if (!c || !Pa || !Pb || !Ga || !Gb) return fail(HFG_INVALID_ARG, "null argument");
  HFG_CUDA(cudaSetDevice(c->device));
  const size_t nn = (size_t)c->nbf * c->nbf;
  hfg_status st;
  if ((st = ensure(&c->d_P, nn)) != HFG_OK || (st = ensure(&c->d_Pb, nn)) != HFG_OK ||
      (st = ensure(&c->d_G, nn)) != HFG_OK || (st = ensure(&c->d_Gb, nn)) != HFG_OK)
    return st;
  HFG_CUDA(cudaMemcpyAsync(c->d_P, Pa, nn * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  HFG_CUDA(cudaMemcpyAsync(c->d_Pb, Pb, nn * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if ((st = direct_build(c, true, c->d_P, c->d_Pb, c->d_G, c->d_Gb, c->stream)) != HFG_OK) return st;
  HFG_CUDA(cudaMemcpyAsync(Ga, c->d_G, nn * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HFG_CUDA(cudaMemcpyAsync(Gb, c->d_Gb, nn * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  HFG_CUDA(cudaStreamSynchronize(c->stream));
  return finish_timing(c);
}

hfg_status hfg_schwarz(hfg_ctx *c, double *host_out, int64_t count) {
  if (!c || !host_out) return fail(HFG_INVALID_ARG, "null argument");
  if (count != c->npairs) return fail(HFG_INVALID_ARG, "count != nshells*(nshells+1)/2");
  std::memcpy(host_out, c->pair_Q.data(), (size_t)count * sizeof(double));
  return HFG_OK;
}

hfg_status hfg_eri_quartet(hfg_ctx *c, int32_t i, int32_t j, int32_t k, int32_t l, double *out) {
  using namespace hfg;
  if (!c || !out) return fail(HFG_INVALID_ARG, "null argument");
  const int n = c->nbf;
  if (i < 0 || j < 0 || k < 0 || l < 0 || i >= n || j >= n || k >= n || l >= n)
    return fail(HFG_INVALID_ARG, "function index out of range");
  HFG_CUDA(cudaSetDevice(c->device));
  auto shell_of = [&](int ao) {
    for (size_t s = 0; s < c->shells.size(); ++s)
      if (ao >= c->shells[s].ao && ao < c->shells[s].ao + ncart_h(c->shells[s].L)) return (int)s;
    return -1;
  };
  auto pair_of = [](int a, int b) { return a >= b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a; };
  int sI = shell_of(i), sJ = shell_of(j), sK = shell_of(k), sL = shell_of(l);
  int p1 = pair_of(sI, sJ), p2 = pair_of(sK, sL);
  int bra = p1, ket = p2;
  const int c1 = c->pair_cls[p1], c2 = c->pair_cls[p2];
  // bra class must not precede the ket class in pair-class order
  if (c1 < c2 || (c1 == c2 && c->pair_Q[p1] < c->pair_Q[p2])) std::swap(bra, ket);
  const int cb = c->pair_cls[bra], ck = c->pair_cls[ket];
  const int cls = class_index(kPairClasses[cb][0], kPairClasses[cb][1], kPairClasses[ck][0], kPairClasses[ck][1]);
  if (cls < 0) return fail(HFG_INVALID_ARG, "no class for quartet");
  // one-task launch over two one-element lists
  std::vector<int> bl{bra}, kl{ket};
  std::vector<Task> tk{Task{0, 0, 1}};
  int *d_bl = nullptr, *d_kl = nullptr;
  Task *d_tk = nullptr;
  hfg_status st;
  if ((st = upload(&d_bl, bl)) != HFG_OK || (st = upload(&d_kl, kl)) != HFG_OK || (st = upload(&d_tk, tk)) != HFG_OK ||
      (st = ensure(&c->d_block, 1296)) != HFG_OK) {
    cudaFree(d_bl); cudaFree(d_kl); cudaFree(d_tk);
    return st;
  }
  ClassLaunch cl{};
  cl.bra_list = d_bl;
  cl.ket_list = d_kl;
  cl.tasks = d_tk;
  cl.ntasks = 1;
  cl.packed = c->d_block;
  kClasses[cls].launch(c->view(), cl, kBlock, c->opts.eri_convention == HFG_ERI_REFERENCE, 0, 1, c->stream);
  double blk[1296];
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(blk, c->d_block, sizeof blk, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d_bl); cudaFree(d_kl); cudaFree(d_tk);
  if (e != cudaSuccess) return fail(HFG_DEVICE_ERROR, cudaGetErrorString(e));
  // locate (i j | k l) in the (first second | first second) block
  const int fa = c->pair_sa[bra], fb = c->pair_sb[bra], fc = c->pair_sa[ket], fd = c->pair_sb[ket];
  const int NB = ncart_h(c->shells[fb].L), NC = ncart_h(c->shells[fc].L), ND = ncart_h(c->shells[fd].L);
  int x[4] = {i, j, k, l};
  // orient the requested indices to the block's shells
  if (bra != p1) { std::swap(x[0], x[2]); std::swap(x[1], x[3]); }
  if (shell_of(x[0]) != fa) std::swap(x[0], x[1]);
  if (shell_of(x[2]) != fc) std::swap(x[2], x[3]);
  const int a = x[0] - c->shells[fa].ao, b = x[1] - c->shells[fb].ao, cc = x[2] - c->shells[fc].ao,
            d = x[3] - c->shells[fd].ao;
  *out = blk[((a * NB + b) * NC + cc) * ND + d];
  return HFG_OK;
}

hfg_status hfg_set_profiling(hfg_ctx *c, int32_t on) {
  if (!c) return hfg::fail(HFG_INVALID_ARG, "null context");
  HFG_CUDA(cudaSetDevice(c->device));
  for (auto &q : c->qclasses) {
    if (!q.ev_a) HFG_CUDA(cudaEventCreate(&q.ev_a));
    if (!q.ev_b) HFG_CUDA(cudaEventCreate(&q.ev_b));
  }
  c->profiling = on != 0;
  ++c->config_version;
  return HFG_OK;
}

hfg_status hfg_class_profile(const hfg_ctx *c, hfg_class_time *out, int32_t cap, int32_t *count) {
  using namespace hfg;
  if (!c || !out || !count) return fail(HFG_INVALID_ARG, "null argument");
  int n = 0;
  for (const auto &q : c->qclasses) {
    if (n >= cap) break;
    const ClassEntry &e = kClasses[q.cls];
    out[n] = hfg_class_time{e.la,    e.lb,    e.lc,         e.ld, q.shell_quartets, q.function_quartets, q.prim_quartets,
                            q.flops, (double)q.last_ms, (int64_t)q.tasks.size(),
                            q.warp_work > 0 ? q.lane_work / q.warp_work : 0.0, class_on_warp(c, q.cls) ? 1 : 0, 0};
    ++n;
  }
  *count = n;
  return HFG_OK;
}

hfg_status hfg_ctx_stats(const hfg_ctx *c, hfg_stats *out) {
  if (!c || !out) return hfg::fail(HFG_INVALID_ARG, "null argument");
  *out = c->stats;
  if (c->counted) {
    // quartets the density screening kept, per precision (waits for the build)
    unsigned long long cnt[2] = {0, 0};
    HFG_CUDA(cudaSetDevice(c->device));
    HFG_CUDA(cudaMemcpy(cnt, c->d_counters, sizeof cnt, cudaMemcpyDeviceToHost));
    out->fp64_shell_quartets = (int64_t)cnt[0];
    out->fp32_shell_quartets = (int64_t)cnt[1];
  }
  return HFG_OK;
}

hfg_status hfg_fock_reset(hfg_ctx *c) {
  if (!c) return hfg::fail(HFG_INVALID_ARG, "null context");
  c->inc_valid = false;
  ++c->config_version;
  return HFG_OK;
}

hfg_status hfg_set_mixed_cutoff(hfg_ctx *c, double cutoff) {
  if (!c) return hfg::fail(HFG_INVALID_ARG, "null context");
  if (!(cutoff >= 0) || !(cutoff < 1e300)) return hfg::fail(HFG_INVALID_ARG, "mixed cutoff must be finite and >= 0");
  c->mixed_cutoff = cutoff;
  ++c->config_version;
  return HFG_OK;
}

// Grid autotuner: for every fused class with tasks, time the class's J/K
// kernel at 1, 2, 4, 8 and 16 blocks per SM on the caller's density (one
// warm-up and two timed launches each, CUDA events on the build stream) and
// keep the fastest for the context's later builds.  Split classes keep
// their fixed chunked launch.  The J/K scratch it writes is cleared by the
// next build.
// Median of five timed direct builds after an untimed one, for the
// whole-build autotuner (single concurrent builds vary by a few per cent).
static hfg_status median_build_ms(hfg_ctx *c, const double *dP, cudaStream_t s, float *out) {
  float t[5];
  hfg_status st;
  for (int r = 0; r < 6; ++r) {
    if ((st = direct_build(c, false, dP, nullptr, c->d_G, nullptr, s)) != HFG_OK) return st;
    if ((st = finish_timing(c)) != HFG_OK) return st;
    if (r > 0) t[r - 1] = c->stats.last_build_ms;
  }
  std::sort(t, t + 5);
  *out = t[2];
  return HFG_OK;
}

hfg_status hfg_autotune(hfg_ctx *c, const double *dP, int32_t *chosen, int32_t cap, int32_t *count, void *stream) {
  if (!c || !dP) return hfg::fail(HFG_INVALID_ARG, "null context or density");
  using namespace hfg;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  const size_t tot = c->batch ? (size_t)c->batch_elems : (size_t)c->nbf * c->nbf;
  hfg_status st;
  if ((st = ensure(&c->d_J, tot)) != HFG_OK || (st = ensure(&c->d_Ka, tot)) != HFG_OK) return st;
  if (c->batch) {
    const std::vector<unsigned char> all(c->nmol, 1);
    HFG_CUDA(cudaMemcpyAsync(c->d_mol_active, all.data(), c->nmol, cudaMemcpyHostToDevice, s));
  }
  const bool ref = c->opts.eri_convention == HFG_ERI_REFERENCE;
  const int cand[] = {1, 2, 4, 8, 16};
  int written = 0;
  if (c->use_streams && !c->batch && !c->precision_form()) {
    // classes share the SMs: one cap for all, timed on whole builds, then
    // a higher one for the classes without shared memory
    const size_t nn = (size_t)c->nbf * c->nbf;
    if ((st = ensure(&c->d_G, nn)) != HFG_OK) return st;
    float best = 1e30f;
    int best_bps = 1;
    for (int b : {1, 2, 4}) {
      for (int k = 0; k < kNumClasses; ++k) c->tuned_bps[k] = b;
      ++c->config_version;
      float ms_sum = 0;
      if ((st = median_build_ms(c, dP, s, &ms_sum)) != HFG_OK) return st;
      if (ms_sum < best) {
        best = ms_sum;
        best_bps = b;
      }
    }
    for (int k = 0; k < kNumClasses; ++k) c->tuned_bps[k] = best_bps;
    // the fused classes that read their Boys rows from global memory hold no
    // shared memory: a higher cap for them alone, timed the same way
    auto no_smem = [](int k) {
      const ClassEntry &e = kClasses[k];
      return !kSplit[k] && !kWarp[k] && boys_from_global(e.la, e.lb, e.lc, e.ld);
    };
    int best_free = best_bps;
    for (int b : {2 * best_bps, 4 * best_bps}) {
      for (int k = 0; k < kNumClasses; ++k)
        if (no_smem(k)) c->tuned_bps[k] = b;
      ++c->config_version;
      float ms_sum = 0;
      if ((st = median_build_ms(c, dP, s, &ms_sum)) != HFG_OK) return st;
      if (ms_sum < best) {
        best = ms_sum;
        best_free = b;
      }
    }
    for (int k = 0; k < kNumClasses; ++k)
      if (no_smem(k)) c->tuned_bps[k] = best_free;
    if (chosen && cap >= 5) {
      const int rec[5] = {-1, -1, -1, -1, best_bps};  // all classes
      std::copy(rec, rec + 5, chosen);
      written = 5;
    }
    for (int k = 0; k < kNumClasses && best_free != best_bps; ++k) {
      if (!chosen || !no_smem(k) || written + 5 > cap) continue;
      const ClassEntry &e = kClasses[k];
      const int rec[5] = {e.la, e.lb, e.lc, e.ld, best_free};
      std::copy(rec, rec + 5, chosen + written);
      written += 5;
    }
    if (count) *count = written / 5;
    ++c->config_version;
    return HFG_OK;
  }
  for (auto &q : c->qclasses) {
    if (kSplit[q.cls] || kWarp[q.cls] || q.tasks.empty()) continue;
    ClassLaunch cl = base_launch(c, q, true);
    if (cl.ntasks == 0) continue;
    cl.Da = dP;
    cl.Dt = dP;
    cl.J = c->d_J;
    cl.Ka = c->d_Ka;
    float best = 1e30f;
    int best_bps = 4;
    for (int b : cand) {
      c->tuned_bps[q.cls] = b;
      const int grid = grid_for(c, cl.ntasks, q.cls);
      kClasses[q.cls].launch(c->view(), cl, kJkRhf, ref, 0, grid, s);
      HFG_CUDA(cudaEventRecord(c->ev0, s));
      for (int r = 0; r < 2; ++r) kClasses[q.cls].launch(c->view(), cl, kJkRhf, ref, 0, grid, s);
      HFG_CUDA(cudaEventRecord(c->ev1, s));
      HFG_CUDA(cudaEventSynchronize(c->ev1));
      HFG_CUDA(cudaGetLastError());
      float ms = 0;
      HFG_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
      if (ms < best) {
        best = ms;
        best_bps = b;
      }
    }
    c->tuned_bps[q.cls] = best_bps;
    if (chosen && written + 5 <= cap) {
      const ClassEntry &e = kClasses[q.cls];
      const int rec[5] = {e.la, e.lb, e.lc, e.ld, best_bps};
      std::copy(rec, rec + 5, chosen + written);
      written += 5;
    }
  }
  if (count) *count = written / 5;
  ++c->config_version;
  return HFG_OK;
}

}  // extern "C"

namespace hfg {
// Rebuilds every class's task list (after a change of the lane-group
// target): host lists, device copies, and the batched builds' compaction
// buffers, which are sized from the lists.
static hfg_status rebuild_tasks(hfg_ctx *c) {
  HFG_CUDA(cudaDeviceSynchronize());  // queued builds may still read the old lists
  for (auto &q : c->qclasses) {
    cudaFree(q.d_tasks);
    if (q.ev_a) cudaEventDestroy(q.ev_a);
    if (q.ev_b) cudaEventDestroy(q.ev_b);
  }
  build_quartet_classes(c, c->opts.schwarz_threshold);
  hfg_status st = upload_classes(c);
  if (st != HFG_OK) return st;
  if (c->profiling)
    for (auto &q : c->qclasses) {
      HFG_CUDA(cudaEventCreate(&q.ev_a));
      HFG_CUDA(cudaEventCreate(&q.ev_b));
    }
  cudaFree(c->d_task_active);
  cudaFree(c->d_task_counts);
  cudaFree(c->d_queue);
  c->d_task_active = nullptr;
  c->d_task_counts = nullptr;
  c->d_queue = nullptr;
  c->task_base.clear();
  ++c->config_version;
  return HFG_OK;
}
}  // namespace hfg

extern "C" {

hfg_status hfg_set_prim_target(hfg_ctx *c, int32_t target) {
  if (!c || target < 0) return hfg::fail(HFG_INVALID_ARG, "null context or negative target");
  c->prim_target = target;
  std::fill(std::begin(c->class_prim_target), std::end(c->class_prim_target), 0);
  return hfg::rebuild_tasks(c);
}

// Task-shape autotuner: for every thread-per-quartet class, the primitive
// quartets per lane that the task builder aims for when it spreads a quartet
// over a lane group (0: one lane per quartet, then 48, 96, 192, 384),
// each timed on the class's J/K kernel alone (one warm-up, two timed
// launches, CUDA events) with the caller's density; the fastest is kept.
hfg_status hfg_autotune_tasks(hfg_ctx *c, const double *dP, int32_t *chosen, int32_t cap, int32_t *count,
                              void *stream) {
  using namespace hfg;
  if (!c || !dP) return fail(HFG_INVALID_ARG, "null context or density");
  if (c->batch) return fail(HFG_INVALID_ARG, "hfg_autotune_tasks: single-molecule contexts");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  const size_t nn = (size_t)c->nbf * c->nbf;
  hfg_status st;
  if ((st = ensure(&c->d_J, nn)) != HFG_OK || (st = ensure(&c->d_Ka, nn)) != HFG_OK) return st;
  const bool ref = c->opts.eri_convention == HFG_ERI_REFERENCE;
  const int cand[] = {0, 48, 96, 192, 384};
  std::vector<float> best(kNumClasses, 1e30f);
  std::vector<int> best_t(kNumClasses, c->prim_target);
  for (int t : cand) {
    c->prim_target = t;
    std::fill(std::begin(c->class_prim_target), std::end(c->class_prim_target), 0);
    if ((st = rebuild_tasks(c)) != HFG_OK) return st;
    for (auto &q : c->qclasses) {
      if (kWarp[q.cls] || kSplit[q.cls]) continue;  // one warp per quartet: no lane groups
      ClassLaunch cl = base_launch(c, q, true);
      if (cl.ntasks == 0) continue;
      cl.Da = dP;
      cl.Dt = dP;
      cl.J = c->d_J;
      cl.Ka = c->d_Ka;
      const int grid = grid_for(c, cl.ntasks, q.cls);
      kClasses[q.cls].launch(c->view(), cl, kJkRhf, ref, 0, grid, s);
      HFG_CUDA(cudaEventRecord(c->ev0, s));
      for (int r = 0; r < 2; ++r) kClasses[q.cls].launch(c->view(), cl, kJkRhf, ref, 0, grid, s);
      HFG_CUDA(cudaEventRecord(c->ev1, s));
      HFG_CUDA(cudaEventSynchronize(c->ev1));
      HFG_CUDA(cudaGetLastError());
      float ms = 0;
      HFG_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
      if (ms < best[q.cls]) {
        best[q.cls] = ms;
        best_t[q.cls] = t;
      }
    }
  }
  c->prim_target = 96;
  int written = 0;
  for (int k = 0; k < kNumClasses; ++k) {
    // class_prim_target: > 0 a target, -1 one lane per quartet, 0 the default
    c->class_prim_target[k] = best[k] < 1e30f ? (best_t[k] > 0 ? best_t[k] : -1) : 0;
    if (best[k] < 1e30f && chosen && written + 5 <= cap) {
      const ClassEntry &e = kClasses[k];
      const int rec[5] = {e.la, e.lb, e.lc, e.ld, best_t[k]};
      std::copy(rec, rec + 5, chosen + written);
      written += 5;
    }
  }
  if (count) *count = written / 5;
  return rebuild_tasks(c);
}

hfg_status hfg_set_class_path(hfg_ctx *c, int32_t la, int32_t lb, int32_t lc, int32_t ld, int32_t path) {
  if (!c) return hfg::fail(HFG_INVALID_ARG, "null context");
  for (int k = 0; k < kNumClasses; ++k) {
    const ClassEntry &e = kClasses[k];
    if (e.la != la || e.lb != lb || e.lc != lc || e.ld != ld) continue;
    if (!kWarp[k] || !kSplit[k]) return hfg::fail(HFG_INVALID_ARG, "hfg_set_class_path: class without both kernels");
    c->warp_class[k] = path != 0 ? 1 : 0;
    ++c->config_version;
    return HFG_OK;
  }
  return hfg::fail(HFG_INVALID_ARG, "hfg_set_class_path: no such canonical quartet class");
}

// Kernel autotuner for the classes with both kernels: each timed on the
// class's J/K build alone (one warm-up, two timed launches, CUDA events)
// with the caller's density, warp kernel against split path; the faster is
// kept.
hfg_status hfg_autotune_paths(hfg_ctx *c, const double *dP, int32_t *chosen, int32_t cap, int32_t *count,
                              void *stream) {
  using namespace hfg;
  if (!c || !dP) return fail(HFG_INVALID_ARG, "null context or density");
  if (c->batch) return fail(HFG_INVALID_ARG, "hfg_autotune_paths: single-molecule contexts");
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  const size_t nn = (size_t)c->nbf * c->nbf;
  hfg_status st;
  if ((st = ensure(&c->d_J, nn)) != HFG_OK || (st = ensure(&c->d_Ka, nn)) != HFG_OK) return st;
  const bool ref = c->opts.eri_convention == HFG_ERI_REFERENCE;
  int written = 0;
  for (auto &q : c->qclasses) {
    if (!kWarp[q.cls] || !kSplit[q.cls] || q.tasks.empty()) continue;
    ClassLaunch cl = base_launch(c, q, true);
    if (cl.ntasks == 0) continue;
    cl.Da = dP;
    cl.Dt = dP;
    cl.J = c->d_J;
    cl.Ka = c->d_Ka;
    float ms[2] = {0, 0};
    for (int path = 0; path < 2; ++path) {
      c->warp_class[q.cls] = (int8_t)path;
      int launches = 0;
      if ((st = launch_class(c, q, cl, kJkRhf, ref, 0, s, &launches)) != HFG_OK) return st;
      HFG_CUDA(cudaEventRecord(c->ev0, s));
      for (int r = 0; r < 2; ++r)
        if ((st = launch_class(c, q, cl, kJkRhf, ref, 0, s, &launches)) != HFG_OK) return st;
      HFG_CUDA(cudaEventRecord(c->ev1, s));
      HFG_CUDA(cudaEventSynchronize(c->ev1));
      HFG_CUDA(cudaGetLastError());
      HFG_CUDA(cudaEventElapsedTime(&ms[path], c->ev0, c->ev1));
    }
    const int pick = ms[1] < ms[0] ? 1 : 0;
    c->warp_class[q.cls] = (int8_t)pick;
    if (chosen && written + 5 <= cap) {
      const ClassEntry &e = kClasses[q.cls];
      const int rec[5] = {e.la, e.lb, e.lc, e.ld, pick};
      std::copy(rec, rec + 5, chosen + written);
      written += 5;
    }
  }
  if (count) *count = written / 5;
  ++c->config_version;
  return HFG_OK;
}

hfg_status hfg_set_streams(hfg_ctx *c, int32_t on) {
  if (!c) return hfg::fail(HFG_INVALID_ARG, "null context");
  c->use_streams = on != 0;
  ++c->config_version;
  return HFG_OK;
}

hfg_status hfg_set_graphs(hfg_ctx *c, int32_t on) {
  if (!c) return hfg::fail(HFG_INVALID_ARG, "null context");
  c->use_graphs = on != 0;
  ++c->config_version;
  return HFG_OK;
}

hfg_status hfg_set_shard(hfg_ctx *c, int32_t rank, int32_t count) {
  if (!c) return hfg::fail(HFG_INVALID_ARG, "null context");
  if (count < 1 || rank < 0 || rank >= count) return hfg::fail(HFG_INVALID_ARG, "shard rank outside [0, count)");
  c->shard_rank = rank;
  c->shard_count = count;
  ++c->config_version;
  c->inc_valid = false;  // an incremental history belongs to one shard
  return HFG_OK;
}

hfg_status hfg_shard_range(const double *cost_prefix, int64_t ntasks, int32_t rank, int32_t count, int64_t *first,
                           int64_t *ntasks_out) {
  if (!cost_prefix || !first || !ntasks_out || ntasks < 0) return hfg::fail(HFG_INVALID_ARG, "hfg_shard_range: arguments");
  if (count < 1 || rank < 0 || rank >= count) return hfg::fail(HFG_INVALID_ARG, "shard rank outside [0, count)");
  shard_range(cost_prefix, ntasks, rank, count, first, ntasks_out);
  return HFG_OK;
}

hfg_status hfg_copy_device(void *dst, const void *src, int64_t bytes, void *stream) {
  if (!dst || !src || bytes < 0) return hfg::fail(HFG_INVALID_ARG, "hfg_copy_device: arguments");
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  HFG_CUDA(cudaMemcpyAsync(dst, src, (size_t)bytes, cudaMemcpyDeviceToDevice, s));
  HFG_CUDA(cudaStreamSynchronize(s));
  return HFG_OK;
}

hfg_status hfg_set_incremental(hfg_ctx *c, int32_t on) {
  if (!c) return hfg::fail(HFG_INVALID_ARG, "null context");
  c->opts.incremental = on != 0;
  c->inc_valid = false;
  ++c->config_version;
  return HFG_OK;
}

}  // extern "C"

// ===========================================================================
// Allocation-free direct RHF build (hfg_fock_rhf_noalloc)
// ===========================================================================
// Serving loops and other callers that must not allocate device memory once
// they are running (a fixed HBM budget, no allocator on the hot path, no
// implicit synchronisation from cudaMalloc/cudaFree) get this variant of the
// direct build: its J and K accumulators live in a file-scope device array
// instead of context buffers.  The array exists once per GPU that loads the
// library and stays resident until the process exits.
namespace hfg {

constexpr int kNoAllocMaxNbf = 1024;
// J then K, each nbf x nbf: 2 * 1024 * 1024 doubles = 16 MiB
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxNbf * kNoAllocMaxNbf];

constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static double *g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on `device` (current).  The host-side
// name g_noalloc_scratch is only a stand-in, so the address is looked up once
// per device with that device current, and cached.
static hfg_status noalloc_scratch(int device, double **out) {
  if (device < 0 || device >= kNoAllocMaxDevices) return fail(HFG_INVALID_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(HFG_DEVICE_ERROR, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
    g_noalloc_ptr[device] = static_cast<double *>(p);
  }
  *out = g_noalloc_ptr[device];
  return HFG_OK;
}

}  // namespace hfg

extern "C" hfg_status hfg_fock_rhf_noalloc(hfg_ctx *c, const double *dP, double *dG, void *stream) {
  using namespace hfg;
  if (!c || !dP || !dG) return fail(HFG_INVALID_ARG, "null argument");
  if (c->batch) return fail(HFG_INVALID_ARG, "batched context: use hfg_fock_rhf_batch_device");
  if (c->precision_form())
    return fail(HFG_INVALID_ARG, "hfg_fock_rhf_noalloc: the context has precision-form settings (density screening, "
                                 "FP32 cutoff or incremental builds); this entry point does plain full FP64 builds only");
  if (c->nbf > kNoAllocMaxNbf)
    return fail(HFG_INVALID_ARG, "hfg_fock_rhf_noalloc: " + std::to_string(c->nbf) +
                                     " basis functions exceed its fixed scratch of " +
                                     std::to_string(kNoAllocMaxNbf) + " (use hfg_fock_rhf_device)");
  HFG_CUDA(cudaSetDevice(c->device));
  double *scratch = nullptr;
  hfg_status st = noalloc_scratch(c->device, &scratch);
  if (st != HFG_OK) return st;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  const int n = c->nbf;
  const size_t nn = (size_t)n * n;
  double *J = scratch, *K = scratch + nn;
  // the array keeps the previous call's sums: clear both accumulators
  HFG_CUDA(cudaMemsetAsync(J, 0, 2 * nn * sizeof(double), s));
  const EngineView v = c->view();
  const bool ref = c->opts.eri_convention == HFG_ERI_REFERENCE;
  for (const auto &q : c->qclasses) {
    ClassLaunch cl = base_launch(c, q);
    cl.Da = dP;
    cl.Dt = dP;
    cl.J = J;
    cl.Ka = K;
    // the large classes run warp-cooperatively: shared memory only, no scratch
    if (kWarp[q.cls]) kWarp[q.cls](v, cl, kJkRhf, ref, 0, 0, s);
    else kClasses[q.cls].launch(v, cl, kJkRhf, ref, 0, grid_for(c, cl.ntasks, q.cls), s);
  }
  const int fg = std::max(1, std::min(1024, (int)((nn + 255) / 256)));
  finalize_rhf<<<fg, 256, 0, s>>>(J, K, dG, n);
  HFG_CUDA(cudaGetLastError());
  return HFG_OK;
}
