#!/usr/bin/env python3
"""Generate straight-line CUDA for every shell-quartet class (La Lb|Lc Ld).

Per primitive quartet: Obara-Saika vertical recursion [e0|00]^(m), then the
Head-Gordon-Pople electron transfer [e0|f0]; after the primitive loops the
two horizontal recursions (ab|f0) and (ab|cd) run once per contracted
quartet.  Each recursion steps along the Cartesian direction the reference
steps along (x if the l exponent is the largest, else y if m is, else z;
GaussianTwoElectrons.h:40-107), and only the intermediates a target actually
depends on are emitted.

`reference` variants reproduce the reference's electron-transfer row range:
for ket column f it computes rows with L(e) >= L(f) - 1 only and the other
rows stay zero (GaussianTwoElectrons.cpp:162).  For L <= 2 that changes only
(dd|dd) with a two-centre bra; `exact` variants compute every row.

Output: eri_gen.cuh with, per class and variant,
  template <class R> __device__ void eri_prim_<tag>(...)   -> accumulates [e0|f0]
  template <class R> __device__ void eri_hrr_<tag>(...)    -> (ab|cd) block
"""
from __future__ import annotations

import os
import sys

MAX_L = 2  # shells up to d (6-31G*, 6-31+G**)


def comps(L):
    """Cartesian components of total L in the reference's canonical order
    (CanonicalIncrement, QuantumNumbers.h:60-80)."""
    out = []
    l, m, n = L, 0, 0
    while True:
        out.append((l, m, n))
        if n == L:
            break
        if m > 0:
            m, n = m - 1, n + 1
        elif l > 0:
            l, m, n = l - 1, L - (l - 1), 0
    return out


def comps_range(lo, hi):
    out = []
    for L in range(lo, hi + 1):
        out += comps(L)
    return out


def tot(c):
    return c[0] + c[1] + c[2]


def direction(c):
    mx = max(c)
    if c[0] == mx:
        return 0
    if c[1] == mx:
        return 1
    return 2


def add(c, i, d):
    c = list(c)
    c[i] += d
    return tuple(c)


def nm(c):
    return f"{c[0]}{c[1]}{c[2]}"


class ClassGen:
    def __init__(self, la, lb, lc, ld, reference):
        self.la, self.lb, self.lc, self.ld = la, lb, lc, ld
        self.ltot = la + lb + lc + ld
        self.reference = reference
        self.lines = []
        self.vrr_done = {}
        self.et_done = {}
        self.flops = 0

    # ---- vertical recursion [e0|00]^(m) ----------------------------------
    def vrr(self, e, m):
        key = (e, m)
        if key in self.vrr_done:
            return self.vrr_done[key]
        if tot(e) == 0:
            name = f"F[{m}]"
            self.vrr_done[key] = name
            return name
        i = direction(e)
        e1 = add(e, i, -1)
        a = self.vrr(e1, m)
        b = self.vrr(e1, m + 1)
        expr = f"PA{i} * {a} + WP{i} * {b}"
        self.flops += 3
        if e1[i] > 0:
            e2 = add(e, i, -2)
            c = self.vrr(e2, m)
            d = self.vrr(e2, m + 1)
            expr += f" + R({e1[i]}) * oo2z * ({c} - roz * {d})"
            self.flops += 5
        name = f"v{nm(e)}_{m}"
        self.lines.append(f"const R {name} = {expr};")
        self.vrr_done[key] = name
        return name

    # ---- electron transfer [e0|f0] ---------------------------------------
    def et(self, e, f):
        key = (e, f)
        if key in self.et_done:
            return self.et_done[key]
        if tot(f) == 0:
            name = self.vrr(e, 0)
            self.et_done[key] = name
            return name
        if self.reference and tot(e) < tot(f) - 1:
            self.et_done[key] = None  # never computed by the reference: zero
            return None
        i = direction(f)
        f1 = add(f, i, -1)
        terms = []
        t = self.et(e, f1)
        if t is not None:
            terms.append(f"delta{i} * {t}")
        t = self.et(add(e, i, 1), f1)
        if t is not None:
            terms.append(f"- zoe * {t}")
        if e[i] > 0:
            t = self.et(add(e, i, -1), f1)
            if t is not None:
                terms.append(f"+ R({e[i]}) * oo2e * {t}")
        if f1[i] > 0:
            t = self.et(e, add(f, i, -2))
            if t is not None:
                terms.append(f"+ R({f1[i]}) * oo2e * {t}")
        self.flops += 2 * len(terms)
        if not terms:
            self.et_done[key] = None
            return None
        expr = " ".join(terms)
        if expr.startswith("- "):
            expr = "-" + expr[2:]
        elif expr.startswith("+ "):
            expr = expr[2:]
        name = f"t{nm(e)}_{nm(f)}"
        self.lines.append(f"const R {name} = {expr};")
        self.et_done[key] = name
        return name

    def prim_body(self):
        """Accumulate every [e0|f0], e in [La, La+Lb], f in [Lc, Lc+Ld]."""
        E = comps_range(self.la, self.la + self.lb)
        Fc = comps_range(self.lc, self.lc + self.ld)
        acc = []
        for ie, e in enumerate(E):
            for jf, f in enumerate(Fc):
                v = self.et(e, f)
                idx = ie * len(Fc) + jf
                if v is not None:
                    acc.append(f"acc[{idx}] += {v};")
                    self.flops += 1
        return self.lines + acc, len(E), len(Fc)


def hrr_code(la, lb, lc, ld):
    """(e0|f0) -> (ab|f0) -> (ab|cd) on the contracted block `acc`
    (HorizontalRecursion1/2, GaussianTwoElectrons.cpp:198-359)."""
    E = comps_range(la, la + lb)
    Fc = comps_range(lc, lc + ld)
    eidx = {c: i for i, c in enumerate(E)}
    fidx = {c: i for i, c in enumerate(Fc)}
    lines = []
    flops = [0]
    memo1 = {}

    def h1(a, b, f):  # (a b | f 0)
        key = (a, b, f)
        if key in memo1:
            return memo1[key]
        if tot(b) == 0:
            name = f"acc[{eidx[a] * len(Fc) + fidx[f]}]"
            memo1[key] = name
            return name
        i = direction(b)
        b1 = add(b, i, -1)
        x = h1(add(a, i, 1), b1, f)
        y = h1(a, b1, f)
        name = f"h{nm(a)}_{nm(b)}_{nm(f)}"
        lines.append(f"const R {name} = {x} + AB{i} * {y};")
        flops[0] += 2
        memo1[key] = name
        return name

    memo2 = {}

    def h2(a, b, c, d):  # (a b | c d)
        key = (a, b, c, d)
        if key in memo2:
            return memo2[key]
        if tot(d) == 0:
            name = h1(a, b, c)
            memo2[key] = name
            return name
        i = direction(d)
        d1 = add(d, i, -1)
        x = h2(a, b, add(c, i, 1), d1)
        y = h2(a, b, c, d1)
        name = f"o{nm(a)}_{nm(b)}_{nm(c)}_{nm(d)}"
        lines.append(f"const R {name} = {x} + CD{i} * {y};")
        flops[0] += 2
        memo2[key] = name
        return name

    outs = []
    A, B, C, D = comps(la), comps(lb), comps(lc), comps(ld)
    k = 0
    for a in A:
        for b in B:
            for c in C:
                for d in D:
                    outs.append(f"out[{k}] = {h2(a, b, c, d)};")
                    k += 1
    return lines + outs, flops[0]


def canonical_classes():
    """Pair classes (La >= Lb) and quartet classes with the bra class >= ket
    class in pair-class order (so La+Lb >= Lc+Ld)."""
    pairs = [(a, b) for a in range(MAX_L + 1) for b in range(a + 1)]
    pairs.sort(key=lambda p: (p[0] + p[1], p[0]))
    quartets = []
    for i, p in enumerate(pairs):
        for q in pairs[: i + 1]:
            quartets.append((p[0], p[1], q[0], q[1]))
    return pairs, quartets


def main(out_path):
    pairs, quartets = canonical_classes()
    hdr = ["// Generated by gen_eri.py -- do not edit.",
           "#pragma once",
           ""]
    table = []
    for (la, lb, lc, ld) in quartets:
        for variant in ("exact", "reference"):
            ref = variant == "reference"
            if ref and not (lc + ld >= la + 2):
                continue  # identical to exact: the truncated rows are never needed
            g = ClassGen(la, lb, lc, ld, ref)
            body, ne, nf = g.prim_body()
            tag = f"{la}{lb}{lc}{ld}" + ("r" if ref else "")
            hdr.append(f"// ({la}{lb}|{lc}{ld}) {variant}: [e0|f0] block {ne}x{nf}, ~{g.flops} flops per primitive quartet")
            hdr.append(f"template <class R> __device__ __forceinline__ void eri_prim_{tag}(R* __restrict__ acc, const R* __restrict__ F,")
            hdr.append("    R PA0, R PA1, R PA2, R WP0, R WP1, R WP2, R oo2z, R roz,")
            hdr.append("    R delta0, R delta1, R delta2, R zoe, R oo2e) {")
            hdr += ["  " + l for l in body]
            hdr.append("}")
            table.append((tag, g.flops))
        lines, hfl = hrr_code(la, lb, lc, ld)
        tag = f"{la}{lb}{lc}{ld}"
        hdr.append(f"// ({la}{lb}|{lc}{ld}) horizontal recursions, {hfl} flops per contracted quartet")
        hdr.append(f"template <class R> __device__ __forceinline__ void eri_hrr_{tag}(R* __restrict__ out, const R* __restrict__ acc,")
        hdr.append("    R AB0, R AB1, R AB2, R CD0, R CD1, R CD2) {")
        hdr += ["  " + l for l in lines]
        hdr.append("}")
        hdr.append("")
    # class traits: EriClass<LA,LB,LC,LD,REF>::prim / ::hrr
    hdr.append("template <int LA, int LB, int LC, int LD, bool REF> struct EriClass;")
    tags = dict(table)
    for (la, lb, lc, ld) in quartets:
        base = f"{la}{lb}{lc}{ld}"
        for ref in (False, True):
            ptag = base + "r" if (ref and (base + "r") in tags) else base
            hdr.append(f"template <> struct EriClass<{la}, {lb}, {lc}, {ld}, {'true' if ref else 'false'}> {{")
            hdr.append("  template <class R> static __device__ __forceinline__ void prim(R* acc, const R* F, R PA0, R PA1, R PA2,")
            hdr.append("      R WP0, R WP1, R WP2, R oo2z, R roz, R delta0, R delta1, R delta2, R zoe, R oo2e) {")
            hdr.append(f"    eri_prim_{ptag}<R>(acc, F, PA0, PA1, PA2, WP0, WP1, WP2, oo2z, roz, delta0, delta1, delta2, zoe, oo2e);")
            hdr.append("  }")
            hdr.append("  template <class R> static __device__ __forceinline__ void hrr(R* out, const R* acc, R AB0, R AB1, R AB2,")
            hdr.append("      R CD0, R CD1, R CD2) {")
            hdr.append(f"    eri_hrr_{base}<R>(out, acc, AB0, AB1, AB2, CD0, CD1, CD2);")
            hdr.append("  }")
            ne = sum((L + 1) * (L + 2) // 2 for L in range(la, la + lb + 1))
            nf = sum((L + 1) * (L + 2) // 2 for L in range(lc, lc + ld + 1))
            hdr.append(f"  static constexpr int kAcc = {ne * nf};")
            hdr.append("};")
    hdr.append("")
    # flop table used by the roofline accounting
    hdr.append("// primitive-quartet flop counts of the generated recursions")
    hdr.append("struct EriClassFlops { int la, lb, lc, ld, prim_exact, prim_reference, hrr; };")
    hdr.append("static const EriClassFlops kEriClassFlops[] = {")
    for (la, lb, lc, ld) in quartets:
        ex = dict(table)[f"{la}{lb}{lc}{ld}"]
        rf = dict(table).get(f"{la}{lb}{lc}{ld}r", ex)
        _, hfl = hrr_code(la, lb, lc, ld)
        hdr.append(f"  {{{la}, {lb}, {lc}, {ld}, {ex}, {rf}, {hfl}}},")
    hdr.append("};")
    with open(out_path, "w") as fh:
        fh.write("\n".join(hdr) + "\n")


def emit_launchers(out_dir):
    """One translation unit per quartet class (they compile in parallel), the
    Schwarz launcher and the dispatch table."""
    pairs, quartets = canonical_classes()
    modes = ("kStorePacked", "kJkRhf", "kJkUhf", "kBlock")
    for (a, b, c, d) in quartets:
        ref = (c + d) >= a + 2  # classes whose reference variant differs
        lines = [f"// Generated by gen_eri.py: launcher for the ({a}{b}|{c}{d}) class kernels.",
                 '#include "eri_dispatch.cuh"', "", "namespace hfg {", "",
                 f"void launch_class_{a}{b}{c}{d}(const EngineView &v, const ClassLaunch &cl, int mode, bool ref, int grid,",
                 "                       cudaStream_t s) {",
                 "  switch (mode) {"]
        for mode in modes:
            lines.append(f"    case {mode}:")
            k = f"eri_class_kernel<{a}, {b}, {c}, {d}, {mode}"
            if ref:
                lines.append(f"      if (ref) {k}, true><<<grid, kThreads, 0, s>>>(v, cl);")
                lines.append(f"      else {k}, false><<<grid, kThreads, 0, s>>>(v, cl);")
            else:
                lines.append(f"      {k}, false><<<grid, kThreads, 0, s>>>(v, cl);")
            lines.append("      break;")
        lines += ["    default:", "      break;", "  }"]
        if not ref:
            lines.append("  (void)ref;")
        lines += ["}", "", "}  // namespace hfg", ""]
        with open(os.path.join(out_dir, f"eri_class_{a}{b}{c}{d}.cu"), "w") as fh:
            fh.write("\n".join(lines))
    lines = ["// Generated by gen_eri.py: Schwarz-bound kernels, one per pair class.", '#include "eri_dispatch.cuh"', "",
             "namespace hfg {", "",
             "void launch_schwarz(int la, int lb, const EngineView &v, const int *pairs, int npairs, double *Q, cudaStream_t s) {",
             "  const int grid = (npairs + kThreads - 1) / kThreads;",
             "  if (grid == 0) return;"]
    for (a, b) in pairs:
        lines.append(f"  if (la == {a} && lb == {b}) schwarz_kernel<{a}, {b}><<<grid, kThreads, 0, s>>>(v, pairs, npairs, Q);")
    lines += ["}", "", "}  // namespace hfg", ""]
    with open(os.path.join(out_dir, "eri_schwarz.cu"), "w") as fh:
        fh.write("\n".join(lines))
    lines = ["// Generated by gen_eri.py: launch wrappers for the class kernels.", "#pragma once",
             '#include "eri_kernels.cuh"', "", "namespace hfg {", "",
             "using ClassLauncher = void (*)(const EngineView &, const ClassLaunch &, int, bool, int, cudaStream_t);"]
    for (a, b, c, d) in quartets:
        lines.append(f"void launch_class_{a}{b}{c}{d}(const EngineView &v, const ClassLaunch &cl, int mode, bool ref, int grid, cudaStream_t s);")
    lines += ["void launch_schwarz(int la, int lb, const EngineView &v, const int *pairs, int npairs, double *Q, cudaStream_t s);",
              "", "struct ClassEntry {", "  int la, lb, lc, ld;", "  ClassLauncher launch;", "};",
              "static const ClassEntry kClasses[] = {"]
    for (a, b, c, d) in quartets:
        lines.append(f"    {{{a}, {b}, {c}, {d}, launch_class_{a}{b}{c}{d}}},")
    lines += ["};", f"constexpr int kNumClasses = {len(quartets)};",
              "static const int kPairClasses[][2] = {" + ", ".join("{%d, %d}" % p for p in pairs) + "};",
              f"constexpr int kNumPairClasses = {len(pairs)};", "", "}  // namespace hfg", ""]
    with open(os.path.join(out_dir, "eri_dispatch.cuh"), "w") as fh:
        fh.write("\n".join(lines))


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    out_dir = sys.argv[1] if len(sys.argv) > 1 else here
    main(os.path.join(out_dir, "eri_gen.cuh"))
    emit_launchers(out_dir)
