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
        """Accumulate every [e0|f0], e in [La, La+Lb], f in [Lc, Lc+Ld].  Each
        element is added to its accumulator right after the statements that
        compute it, so a target value need not stay live to the end."""
        E = comps_range(self.la, self.la + self.lb)
        Fc = comps_range(self.lc, self.lc + self.ld)
        for ie, e in enumerate(E):
            for jf, f in enumerate(Fc):
                v = self.et(e, f)
                idx = ie * len(Fc) + jf
                if v is not None:
                    self.lines.append(f"acc[{idx}] += {v};")
                    self.flops += 1
        return self.lines, len(E), len(Fc)


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
            hdr.append(f"template <class R, class A> __device__ __forceinline__ void eri_prim_{tag}(A acc, const R* __restrict__ F,")
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
            hdr.append("  // acc: the accumulator block, a register array (R*) or any type with")
            hdr.append("  // operator[] returning an assignable element")
            hdr.append("  template <class R, class A> static __device__ __forceinline__ void prim(A acc, const R* F, R PA0, R PA1,")
            hdr.append("      R PA2, R WP0, R WP1, R WP2, R oo2z, R roz, R delta0, R delta1, R delta2, R zoe, R oo2e) {")
            hdr.append(f"    eri_prim_{ptag}<R, A>(acc, F, PA0, PA1, PA2, WP0, WP1, WP2, oo2z, roz, delta0, delta1, delta2, zoe, oo2e);")
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
    """One translation unit per quartet class (they compile in parallel), a
    second one with the density-screened FP64/FP32 J/K kernels of the fused
    classes, the Schwarz launcher and the dispatch table.  `prec` of a
    launcher: 0 plain FP64, 1 screened FP64, 2 screened with the per-task
    FP64/FP32 choice."""
    pairs, quartets = canonical_classes()
    modes = ("kStorePacked", "kJkRhf", "kJkUhf", "kBlock")

    def launch(lines, ind, k, ref, tail="(v, cl, grid, s);"):
        if ref:
            lines.append(f"{ind}if (ref) {k.format(r='true')}{tail}")
            lines.append(f"{ind}else {k.format(r='false')}{tail}")
        else:
            lines.append(f"{ind}{k.format(r='false')}{tail}")

    for (a, b, c, d) in quartets:
        ref = (c + d) >= a + 2  # classes whose reference variant differs
        split = is_split_class(a, b, c, d)
        tag = f"{a}{b}{c}{d}"
        lines = [f"// Generated by gen_eri.py: launcher for the ({a}{b}|{c}{d}) class kernels.",
                 '#include "eri_dispatch.cuh"', "", "namespace hfg {", "",
                 f"void launch_class_{tag}(const EngineView &v, const ClassLaunch &cl, int mode, bool ref, int prec,",
                 "                       int grid, cudaStream_t s) {"]
        if not split:
            lines += ["  if (prec != 0 && (mode == kJkRhf || mode == kJkUhf)) {",
                      f"    launch_class_{tag}_scr(v, cl, mode, ref, prec, grid, s);",
                      "    return;", "  }"]
        lines.append("  switch (mode) {")
        for mode in modes:
            lines.append(f"    case {mode}:")
            launch(lines, "      ", f"launch_fused<{a}, {b}, {c}, {d}, {mode}, {{r}}>", ref)
            lines.append("      break;")
        lines += ["    default:", "      break;", "  }"]
        if not ref:
            lines.append("  (void)ref;")
        if split:
            lines.append("  (void)prec;")
        lines += ["}", "", "}  // namespace hfg", ""]
        with open(os.path.join(out_dir, f"eri_class_{tag}.cu"), "w") as fh:
            fh.write("\n".join(lines))
        if split:
            continue
        lines = [f"// Generated by gen_eri.py: density-screened J/K kernels of the ({a}{b}|{c}{d}) class.",
                 '#include "eri_dispatch.cuh"', "", "namespace hfg {", "",
                 f"void launch_class_{tag}_scr(const EngineView &v, const ClassLaunch &cl, int mode, bool ref, int prec,",
                 "                           int grid, cudaStream_t s) {",
                 "  switch (mode) {"]
        for mode in ("kJkRhf", "kJkUhf"):
            lines.append(f"    case {mode}:")
            lines.append("      if (prec == 2) {")
            launch(lines, "        ", f"launch_fused<{a}, {b}, {c}, {d}, {mode}, {{r}}, kScreenMixed>", ref)
            lines.append("      } else {")
            launch(lines, "        ", f"launch_fused<{a}, {b}, {c}, {d}, {mode}, {{r}}, kScreenFp64>", ref)
            lines.append("      }")
            lines.append("      break;")
        lines += ["    default:", "      break;", "  }"]
        if not ref:
            lines.append("  (void)ref;")
        lines += ["}", "", "}  // namespace hfg", ""]
        with open(os.path.join(out_dir, f"eri_class_{tag}_scr.cu"), "w") as fh:
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
             "using ClassLauncher = void (*)(const EngineView &, const ClassLaunch &, int, bool, int, int, cudaStream_t);"]
    for (a, b, c, d) in quartets:
        lines.append(f"void launch_class_{a}{b}{c}{d}(const EngineView &v, const ClassLaunch &cl, int mode, bool ref, int prec, int grid, cudaStream_t s);")
        if not is_split_class(a, b, c, d):
            lines.append(f"void launch_class_{a}{b}{c}{d}_scr(const EngineView &v, const ClassLaunch &cl, int mode, bool ref, int prec, int grid, cudaStream_t s);")
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


# ---------------------------------------------------------------------------
# Row-wise horizontal recursion for the split (primitive kernel + HRR/digest
# kernel) path of the large classes.  The HRR is linear, so (a b| expands to
# a short sum over (e| with polynomial coefficients in A-B:
#   (a, b) = (a + 1_i, b - 1_i) + AB_i (a, b - 1_i)
# For one bra row (a, b) this gives <= 4 terms per ket column f; the ket
# recursion expands the same way in C-D.
# ---------------------------------------------------------------------------
def poly_mul_x(p, i):
    out = {}
    for mono, c in p.items():
        m = list(mono)
        m[i] += 1
        out[tuple(m)] = out.get(tuple(m), 0) + c
    return out


def poly_add(p, q):
    out = dict(p)
    for mono, c in q.items():
        out[mono] = out.get(mono, 0) + c
    return {m: c for m, c in out.items() if c != 0}


def hrr_expansion(a, b, memo=None):
    """{e: poly} with (a b| = sum_e poly(X) (e 0|, e on the first centre."""
    if memo is None:
        memo = {}
    key = (a, b)
    if key in memo:
        return memo[key]
    if tot(b) == 0:
        r = {a: {(0, 0, 0): 1}}
    else:
        i = direction(b)
        b1 = add(b, i, -1)
        r = {}
        for e, p in hrr_expansion(add(a, i, 1), b1, memo).items():
            r[e] = poly_add(r.get(e, {}), p)
        for e, p in hrr_expansion(a, b1, memo).items():
            r[e] = poly_add(r.get(e, {}), poly_mul_x(p, i))
    memo[key] = r
    return r


def poly_expr(p, var):
    """C expression of a polynomial in var0..var2 (monomials precomputed as
    {var}_{k0}{k1}{k2})."""
    terms = []
    for mono, c in sorted(p.items()):
        name = None if mono == (0, 0, 0) else f"{var}_{mono[0]}{mono[1]}{mono[2]}"
        if name is None:
            terms.append(f"R({c})")
        elif c == 1:
            terms.append(name)
        else:
            terms.append(f"R({c}) * {name}")
    return " + ".join(terms) if terms else "R(0)"


def monomials(maxdeg):
    out = []
    for d in range(1, maxdeg + 1):
        for k0 in range(d, -1, -1):
            for k1 in range(d - k0, -1, -1):
                out.append((k0, k1, d - k0 - k1))
    return out


def emit_monomials(var, maxdeg):
    lines = []
    for m in monomials(maxdeg):
        name = f"{var}_{m[0]}{m[1]}{m[2]}"
        i = 0 if m[0] else (1 if m[1] else 2)
        lower = list(m)
        lower[i] -= 1
        if sum(lower) == 0:
            lines.append(f"const R {name} = {var}{i};")
        else:
            lines.append(f"const R {name} = {var}_{lower[0]}{lower[1]}{lower[2]} * {var}{i};")
    return lines


def hrr_row_code(la, lb, lc, ld):
    """One bra row (a b | c d), all c d, from the contracted [e0|f0] block
    stored column-major in scratch: acc(e, f) = scr[(e * NF + f) * stride]."""
    E = comps_range(la, la + lb)
    Fc = comps_range(lc, lc + ld)
    eidx = {c: i for i, c in enumerate(E)}
    fidx = {c: i for i, c in enumerate(Fc)}
    NF = len(Fc)
    A, B, C, D = comps(la), comps(lb), comps(lc), comps(ld)
    lines = emit_monomials("X", lb) + emit_monomials("Y", ld)
    lines.append("R vf[%d];" % NF)
    lines.append("switch (ab) {")
    memo = {}
    for ia, a in enumerate(A):
        for ib, b in enumerate(B):
            lines.append(f"  case {ia * len(B) + ib}: {{")
            ex = hrr_expansion(a, b, memo)
            for jf in range(NF):
                terms = [f"({poly_expr(p, 'X')}) * R(scr[({eidx[e]} * {NF} + {jf}) * stride])"
                         for e, p in sorted(ex.items(), key=lambda kv: eidx[kv[0]])]
                lines.append(f"    vf[{jf}] = " + " + ".join(terms) + ";")
            lines.append("  } break;")
    lines.append("  default: break;")
    lines.append("}")
    memo2 = {}
    k = 0
    for c in C:
        for d in D:
            ex = hrr_expansion(c, d, memo2)
            terms = [f"({poly_expr(p, 'Y')}) * vf[{fidx[f]}]" for f, p in sorted(ex.items(), key=lambda kv: fidx[kv[0]])]
            lines.append(f"out[{k}] = " + " + ".join(terms) + ";")
            k += 1
    return lines


def hrr_col_code(la, lb, lc, ld):
    """One ket column (c d | a b), all c d, of a block stored with bra (c d)
    (components C, D, HRR variable X) and ket (a b) (variable Y); `ab`
    selects the ket pair.  Used for the reference convention's swapped
    (dd|dd) orientation."""
    E = comps_range(la, la + lb)
    Fc = comps_range(lc, lc + ld)
    eidx = {c: i for i, c in enumerate(E)}
    fidx = {c: i for i, c in enumerate(Fc)}
    NF = len(Fc)
    A, B, C, D = comps(la), comps(lb), comps(lc), comps(ld)
    lines = emit_monomials("X", lb) + emit_monomials("Y", ld)
    lines.append("R we[%d];" % len(E))
    lines.append("switch (ab) {")
    memo = {}
    for ic, c in enumerate(C):
        for id_, d in enumerate(D):
            lines.append(f"  case {ic * len(D) + id_}: {{")
            ex = hrr_expansion(c, d, memo)
            for ie in range(len(E)):
                terms = [f"({poly_expr(p, 'Y')}) * R(scr[({ie} * {NF} + {fidx[f]}) * stride])"
                         for f, p in sorted(ex.items(), key=lambda kv: fidx[kv[0]])]
                lines.append(f"    we[{ie}] = " + " + ".join(terms) + ";")
            lines.append("  } break;")
    lines.append("  default: break;")
    lines.append("}")
    memo2 = {}
    k = 0
    for a in A:
        for b in B:
            ex = hrr_expansion(a, b, memo2)
            terms = [f"({poly_expr(p, 'X')}) * we[{eidx[e]}]" for e, p in sorted(ex.items(), key=lambda kv: eidx[kv[0]])]
            lines.append(f"out[{k}] = " + " + ".join(terms) + ";")
            k += 1
    return lines


def is_split_class(la, lb, lc, ld):
    """Classes whose fused kernel spills: more than 100 integrals per shell
    quartet.  (dp|ds) and (dd|ps) (108) spill too (255 registers, local
    memory traffic reaching DRAM in their fused kernel); split, (dp|ds) went
    from ~0.9 to 0.65 ms per (H2O)16 build."""
    n = lambda L: (L + 1) * (L + 2) // 2
    return n(la) * n(lb) * n(lc) * n(ld) > 100


def emit_split(out_dir):
    """eri_split_gen.cuh (row/column HRR functions of the split classes),
    one launcher TU per split class, and the split dispatch table."""
    pairs, quartets = canonical_classes()
    hdr = ["// Generated by gen_eri.py -- do not edit.", "#pragma once", ""]
    for (la, lb, lc, ld) in quartets:
        if not is_split_class(la, lb, lc, ld):
            continue
        tag = f"{la}{lb}{lc}{ld}"
        hdr.append(f"// ({la}{lb}|{lc}{ld}): bra row `ab` of the block, all ket (c d)")
        hdr.append(f"template <class R, class S> __device__ __forceinline__ void eri_hrr_row_{tag}(R* __restrict__ out, int ab,")
        hdr.append("    const S* __restrict__ scr, long long stride, R X0, R X1, R X2, R Y0, R Y1, R Y2) {")
        hdr += ["  " + l for l in hrr_row_code(la, lb, lc, ld)]
        hdr.append("}")
        if (la, lb, lc, ld) == (2, 2, 2, 2):
            hdr.append(f"// ({la}{lb}|{lc}{ld}): ket column `ab` of a block stored with bra/ket exchanged")
            hdr.append(f"template <class R, class S> __device__ __forceinline__ void eri_hrr_col_{tag}(R* __restrict__ out, int ab,")
            hdr.append("    const S* __restrict__ scr, long long stride, R X0, R X1, R X2, R Y0, R Y1, R Y2) {")
            hdr += ["  " + l for l in hrr_col_code(la, lb, lc, ld)]
            hdr.append("}")
        hdr.append("")
    hdr.append("template <int LA, int LB, int LC, int LD> struct EriRows;")
    for (la, lb, lc, ld) in quartets:
        if not is_split_class(la, lb, lc, ld):
            continue
        tag = f"{la}{lb}{lc}{ld}"
        hdr.append(f"template <> struct EriRows<{la}, {lb}, {lc}, {ld}> {{")
        hdr.append("  template <class R, class S> static __device__ __forceinline__ void row(R* out, int ab, const S* scr,")
        hdr.append("      long long stride, R X0, R X1, R X2, R Y0, R Y1, R Y2) {")
        hdr.append(f"    eri_hrr_row_{tag}<R, S>(out, ab, scr, stride, X0, X1, X2, Y0, Y1, Y2);")
        hdr.append("  }")
        hdr.append("  template <class R, class S> static __device__ __forceinline__ void col(R* out, int ab, const S* scr,")
        hdr.append("      long long stride, R X0, R X1, R X2, R Y0, R Y1, R Y2) {")
        if (la, lb, lc, ld) == (2, 2, 2, 2):
            hdr.append(f"    eri_hrr_col_{tag}<R, S>(out, ab, scr, stride, X0, X1, X2, Y0, Y1, Y2);")
        hdr.append("  }")
        hdr.append("};")
    with open(os.path.join(out_dir, "eri_split_gen.cuh"), "w") as fh:
        fh.write("\n".join(hdr) + "\n")
    modes = ("kStorePacked", "kJkRhf", "kJkUhf")

    def launch(lines, ind, k, ref, grid):
        tail = f"(v, cl, ch, {grid}, s);" if k.startswith("launch_") else f"<<<{grid}, kThreads, 0, s>>>(v, cl, ch);"
        if ref:
            lines.append(f"{ind}if (ref) {k.format(r='true')}{tail}")
            lines.append(f"{ind}else {k.format(r='false')}{tail}")
        else:
            lines.append(f"{ind}{k.format(r='false')}{tail}")

    head = ["  const int slots = ch.ntasks * 32;",
            "  const int gridA = (slots + kThreads - 1) / kThreads;",
            "  const int gridB = ch.ntasks;  // one block per task"]
    for (a, b, c, d) in quartets:
        if not is_split_class(a, b, c, d):
            continue
        ref = (c + d) >= a + 2
        tag = f"{a}{b}{c}{d}"
        lines = [f"// Generated by gen_eri.py: split-path launchers for the ({a}{b}|{c}{d}) class.",
                 '#include "eri_split.cuh"', '#include "eri_split_dispatch.cuh"', "", "namespace hfg {", "",
                 f"void launch_split_{tag}(const EngineView &v, const ClassLaunch &cl, const SplitChunk &ch, int mode,",
                 "                        bool ref, int prec, cudaStream_t s) {",
                 "  if (prec != 0 && (mode == kJkRhf || mode == kJkUhf)) {",
                 f"    launch_split_{tag}_scr(v, cl, ch, mode, ref, prec, s);",
                 "    return;", "  }"] + head
        launch(lines, "  ", f"launch_prim_split<{a}, {b}, {c}, {d}, {{r}}>", ref, "gridA")
        lines.append("  switch (mode) {")
        for mode in modes:
            lines.append(f"    case {mode}:")
            if mode == "kStorePacked":
                launch(lines, "      ", f"eri_hrr_store_kernel<{a}, {b}, {c}, {d}, {{r}}>", ref, "gridB")
            else:
                launch(lines, "      ", f"launch_hrr_jk<{a}, {b}, {c}, {d}, {mode}, {{r}}>", ref, "gridB")
            lines.append("      break;")
        lines += ["    default:", "      break;", "  }"]
        if not ref:
            lines.append("  (void)ref;")
        lines += ["}", "", "}  // namespace hfg", ""]
        with open(os.path.join(out_dir, f"eri_split_{tag}.cu"), "w") as fh:
            fh.write("\n".join(lines))
        lines = [f"// Generated by gen_eri.py: density-screened split-path launchers for the ({a}{b}|{c}{d}) class.",
                 '#include "eri_split.cuh"', '#include "eri_split_dispatch.cuh"', "", "namespace hfg {", "",
                 f"void launch_split_{tag}_scr(const EngineView &v, const ClassLaunch &cl, const SplitChunk &ch, int mode,",
                 "                            bool ref, int prec, cudaStream_t s) {"] + head
        lines.append("  if (prec == 2) {")
        launch(lines, "    ", f"launch_prim_split<{a}, {b}, {c}, {d}, {{r}}, kScreenMixed>", ref, "gridA")
        lines.append("  } else {")
        launch(lines, "    ", f"launch_prim_split<{a}, {b}, {c}, {d}, {{r}}, kScreenFp64>", ref, "gridA")
        lines.append("  }")
        lines.append("  switch (mode) {")
        for mode in ("kJkRhf", "kJkUhf"):
            lines.append(f"    case {mode}:")
            launch(lines, "      ", f"launch_hrr_jk<{a}, {b}, {c}, {d}, {mode}, {{r}}, true>", ref, "gridB")
            lines.append("      break;")
        lines += ["    default:", "      break;", "  }"]
        if not ref:
            lines.append("  (void)ref;")
        lines += ["}", "", "}  // namespace hfg", ""]
        with open(os.path.join(out_dir, f"eri_split_{tag}_scr.cu"), "w") as fh:
            fh.write("\n".join(lines))
    lines = ["// Generated by gen_eri.py: split-path launcher table.", "#pragma once", '#include "hfg_internal.cuh"', "",
             "namespace hfg {", "",
             "using SplitLauncher = void (*)(const EngineView &, const ClassLaunch &, const SplitChunk &, int, bool, int, cudaStream_t);"]
    for (a, b, c, d) in quartets:
        if is_split_class(a, b, c, d):
            for suf in ("", "_scr"):
                lines.append(f"void launch_split_{a}{b}{c}{d}{suf}(const EngineView &v, const ClassLaunch &cl, const SplitChunk &ch, int mode, bool ref, int prec, cudaStream_t s);")
    lines.append("")
    lines.append("// split launcher per class (same order as kClasses), nullptr for fused-only classes")
    lines.append("static const SplitLauncher kSplit[] = {")
    for (a, b, c, d) in quartets:
        lines.append(f"    {'launch_split_%d%d%d%d' % (a, b, c, d) if is_split_class(a, b, c, d) else 'nullptr'},")
    lines += ["};", "", "}  // namespace hfg", ""]
    with open(os.path.join(out_dir, "eri_split_dispatch.cuh"), "w") as fh:
        fh.write("\n".join(lines))


# ---------------------------------------------------------------------------
# Warp-cooperative programs for the large classes.  One warp evaluates one
# shell quartet: the per-primitive recursions (vertical recursion and
# electron transfer, the same nodes, directions and reference-convention
# pruning as ClassGen) become a list of operations ordered by dependency
# depth; the warp's lanes run the operations of one depth level side by side
# on intermediates held in shared memory, with a warp barrier between levels.
# Every operation has one of the two forms
#   vertical (kind 0):  out = PA_i w[a] + WP_i w[b] + n1 oo2z (w[c] - roz w[d])
#   transfer (kind 1):  out = delta_i w[a] - zoe w[b] + oo2e (n1 w[c] + n2 w[d])
# with per-primitive coefficients selected by kind and Cartesian direction.
# Absent operands read slot 0, which always holds zero.  Slots are assigned
# by a liveness scan (a slot is reused from the level after its last read),
# so the shared-memory footprint is the peak live set, not the node count.
# ---------------------------------------------------------------------------
class WarpProgram:
    def __init__(self, la, lb, lc, ld, reference):
        self.la, self.lb, self.lc, self.ld = la, lb, lc, ld
        self.ltot = la + lb + lc + ld
        self.reference = reference
        self.nodes = []  # (kind, dir, operands(4 node ids or None), n1, n2); kind 'F' = Boys input
        self.vmemo, self.tmemo = {}, {}
        self.fnodes = []
        for m in range(self.ltot + 1):
            self.fnodes.append(self._node(("F", 0, (None,) * 4, 0, 0)))

    def _node(self, spec):
        self.nodes.append(spec)
        return len(self.nodes) - 1

    def vrr(self, e, m):
        key = (e, m)
        if key in self.vmemo:
            return self.vmemo[key]
        if tot(e) == 0:
            nid = self.fnodes[m]
        else:
            i = direction(e)
            e1 = add(e, i, -1)
            a, b = self.vrr(e1, m), self.vrr(e1, m + 1)
            c = d = None
            n1 = 0
            if e1[i] > 0:
                e2 = add(e, i, -2)
                c, d = self.vrr(e2, m), self.vrr(e2, m + 1)
                n1 = e1[i]
            nid = self._node((0, i, (a, b, c, d), n1, 0))
        self.vmemo[key] = nid
        return nid

    def et(self, e, f):
        key = (e, f)
        if key in self.tmemo:
            return self.tmemo[key]
        if tot(f) == 0:
            nid = self.vrr(e, 0)
        elif self.reference and tot(e) < tot(f) - 1:
            nid = None
        else:
            i = direction(f)
            f1 = add(f, i, -1)
            t1 = self.et(e, f1)
            t2 = self.et(add(e, i, 1), f1)
            t3 = self.et(add(e, i, -1), f1) if e[i] > 0 else None
            t4 = self.et(e, add(f, i, -2)) if f1[i] > 0 else None
            if t1 is None and t2 is None and t3 is None and t4 is None:
                nid = None
            else:
                nid = self._node((1, i, (t1, t2, t3, t4), e[i] if t3 is not None else 0,
                                  f1[i] if t4 is not None else 0))
        self.tmemo[key] = nid
        return nid

    def build(self):
        E = comps_range(self.la, self.la + self.lb)
        Fc = comps_range(self.lc, self.lc + self.ld)
        accn = [self.et(e, f) for e in E for f in Fc]
        n = len(self.nodes)
        level = [0] * n
        for k, (kind, _, ops, _, _) in enumerate(self.nodes):
            if kind != "F":
                level[k] = 1 + max(level[o] for o in ops if o is not None)
        nlev = max(level) if n else 0
        last = [-1] * n
        for k, (kind, _, ops, _, _) in enumerate(self.nodes):
            for o in ops:
                if o is not None:
                    last[o] = max(last[o], level[k])
        for o in accn:
            if o is not None:
                last[o] = nlev + 1  # read by the contraction after the last level
        # slot 0: zero; F nodes first (written before level 1)
        slot = [0] * n
        free, nslots = [], 1
        order = sorted(range(n), key=lambda k: (level[k], k))
        by_level = {}
        for k in order:
            by_level.setdefault(level[k], []).append(k)
        released = {}
        for k in range(n):
            if last[k] >= 0:
                released.setdefault(last[k] + 1, []).append(k)
        for L in range(nlev + 1):
            for k in released.get(L, []):
                free.append(slot[k])
            free.sort(reverse=True)
            for k in by_level.get(L, []):
                if last[k] < 0 and self.nodes[k][0] != "F":
                    raise RuntimeError("dead node")
                if free:
                    slot[k] = free.pop()
                else:
                    slot[k] = nslots
                    nslots += 1
        ops, bounds = [], [0]
        for L in range(1, nlev + 1):
            for k in by_level.get(L, []):
                kind, i, operands, n1, n2 = self.nodes[k]
                sl = [slot[o] if o is not None else 0 for o in operands]
                ops.append((slot[k], i, kind, n1, n2, sl))
            bounds.append(len(ops))
        fslots = [slot[k] for k in self.fnodes]
        acc = [slot[o] if o is not None else 0 for o in accn]
        return dict(ops=ops, bounds=bounds, nslots=nslots, fslots=fslots, acc=acc, ne=len(E), nf=len(Fc))


def warp_flops(prog):
    """flops of one primitive quartet's recursions as the generated straight-line code counts them"""
    return None


def emit_warp(out_dir):
    """eri_warp_gen.cuh: the level-ordered programs and traits of the large
    classes (WarpProg<LA,LB,LC,LD,REF>), one launcher TU per large class and
    the dispatch table kWarp[] (nullptr for the classes the per-thread kernel
    serves)."""
    pairs, quartets = canonical_classes()
    hdr = ["// Generated by gen_eri.py -- do not edit.", "#pragma once", "", "#include <stdint.h>", "",
           "namespace hfg {", "", "template <int LA, int LB, int LC, int LD, bool REF> struct WarpProg;"]
    for (la, lb, lc, ld) in quartets:
        if not is_split_class(la, lb, lc, ld):
            continue
        for ref in (False, True):
            has_ref = (lc + ld) >= la + 2
            pr = WarpProgram(la, lb, lc, ld, ref and has_ref).build()
            tag = f"{la}{lb}{lc}{ld}" + ("r" if ref else "")
            words = []
            for (out, i, kind, n1, n2, sl) in pr["ops"]:
                assert max(sl + [out]) < 65536 and n1 < 16 and n2 < 16
                x = out | (i << 16) | (kind << 18) | (n1 << 20) | (n2 << 24)
                words.append(f"{{{x}u, {sl[0] | (sl[1] << 16)}u, {sl[2] | (sl[3] << 16)}u, 0u}}")
            hdr.append(f"// ({la}{lb}|{lc}{ld}) {'reference' if ref else 'exact'}: {len(pr['ops'])} operations in "
                       f"{len(pr['bounds']) - 1} levels, {pr['nslots']} slots")
            hdr.append(f"static __device__ const uint4 kWarpOps_{tag}[] = {{")
            for k in range(0, len(words), 4):
                hdr.append("    " + ", ".join(words[k:k + 4]) + ",")
            hdr.append("};")
            hdr.append(f"static __device__ const uint16_t kWarpAcc_{tag}[] = {{")
            for k in range(0, len(pr["acc"]), 16):
                hdr.append("    " + ", ".join(str(v) for v in pr["acc"][k:k + 16]) + ",")
            hdr.append("};")
            hdr.append(f"template <> struct WarpProg<{la}, {lb}, {lc}, {ld}, {'true' if ref else 'false'}> {{")
            hdr.append(f"  static constexpr int kSlots = {pr['nslots']};")
            hdr.append(f"  static constexpr int kOps = {len(pr['ops'])};")
            hdr.append(f"  static constexpr int kLevels = {len(pr['bounds']) - 1};")
            hdr.append(f"  static constexpr int kAcc = {pr['ne'] * pr['nf']};")
            hdr.append("  static __device__ __forceinline__ const uint4 *ops() { return kWarpOps_%s; }" % tag)
            hdr.append("  static __device__ __forceinline__ const uint16_t *acc() { return kWarpAcc_%s; }" % tag)
            hdr.append("  static __device__ __forceinline__ int bound(int l) {")
            hdr.append("    constexpr int b[] = {" + ", ".join(str(v) for v in pr["bounds"]) + "};")
            hdr.append("    return b[l];")
            hdr.append("  }")
            hdr.append("  static __device__ __forceinline__ int fslot(int m) {")
            hdr.append("    constexpr int f[] = {" + ", ".join(str(v) for v in pr["fslots"]) + "};")
            hdr.append("    return f[m];")
            hdr.append("  }")
            hdr.append("};")
    hdr += ["", "}  // namespace hfg", ""]
    with open(os.path.join(out_dir, "eri_warp_gen.cuh"), "w") as fh:
        fh.write("\n".join(hdr) + "\n")
    # one translation unit per (class, mode) and precision variant, so the
    # large classes' instantiations compile in parallel; launch_warp_<tag>
    # dispatches on the mode and the precision form
    modes = ("kStorePacked", "kJkRhf", "kJkUhf")
    decls = []
    for (a, b, c, d) in quartets:
        if not is_split_class(a, b, c, d):
            continue
        has_ref = (c + d) >= a + 2
        tag = f"{a}{b}{c}{d}"
        parts = [(m, False) for m in modes] + [(m, True) for m in ("kJkRhf", "kJkUhf")]
        for mode, scr in parts:
            fn = f"launch_warp_{tag}_{'s' if scr else 'm'}{modes.index(mode)}"
            decls.append(f"void {fn}(const EngineView &v, const ClassLaunch &cl, bool ref, int prec, int grid, "
                         "cudaStream_t s);")
            lines = [f"// Generated by gen_eri.py: warp-cooperative ({a}{b}|{c}{d}) kernels, mode {mode}"
                     + (", density-screened." if scr else "."),
                     '#include "eri_warp.cuh"', '#include "eri_warp_dispatch.cuh"', "", "namespace hfg {", "",
                     f"void {fn}(const EngineView &v, const ClassLaunch &cl, bool ref, int prec, int grid, "
                     "cudaStream_t s) {"]
            variants = [("kScreenMixed", "prec == 2"), ("kScreenFp64", None)] if scr else [("kScreenNone", None)]
            for r in ((True, False) if has_ref else (False,)):
                cond = "ref" if (has_ref and r) else ("!ref" if has_ref else None)
                for sv, pc in variants:
                    conds = " && ".join(x for x in (cond, pc) if x)
                    call = f"launch_warp<{a}, {b}, {c}, {d}, {mode}, {'true' if r else 'false'}, {sv}>(v, cl, grid, s);"
                    lines.append(f"  if ({conds}) {{ {call} return; }}" if conds else f"  {call}")
            lines += ["  (void)ref;", "  (void)prec;", "}", "", "}  // namespace hfg", ""]
            with open(os.path.join(out_dir, f"eri_warp_{tag}_{'s' if scr else 'm'}{modes.index(mode)}.cu"), "w") as fh:
                fh.write("\n".join(lines))
        lines = [f"// Generated by gen_eri.py: warp-cooperative launcher of the ({a}{b}|{c}{d}) class.",
                 '#include "eri_warp_dispatch.cuh"', "", "namespace hfg {", "",
                 f"void launch_warp_{tag}(const EngineView &v, const ClassLaunch &cl, int mode, bool ref, int prec, "
                 "int grid, cudaStream_t s) {",
                 "  const bool scr = prec != 0 && (mode == kJkRhf || mode == kJkUhf);",
                 "  switch (mode) {"]
        for k, mode in enumerate(modes):
            lines.append(f"    case {mode}:")
            if mode == "kStorePacked":
                lines.append(f"      launch_warp_{tag}_m{k}(v, cl, ref, prec, grid, s);")
            else:
                lines.append(f"      if (scr) launch_warp_{tag}_s{k}(v, cl, ref, prec, grid, s);")
                lines.append(f"      else launch_warp_{tag}_m{k}(v, cl, ref, prec, grid, s);")
            lines.append("      break;")
        lines += ["    default:", "      break;", "  }", "}", "", "}  // namespace hfg", ""]
        with open(os.path.join(out_dir, f"eri_warp_{tag}.cu"), "w") as fh:
            fh.write("\n".join(lines))
    lines = ["// Generated by gen_eri.py: warp-cooperative launcher table.", "#pragma once",
             '#include "hfg_internal.cuh"', "", "namespace hfg {", "",
             "using WarpLauncher = void (*)(const EngineView &, const ClassLaunch &, int, bool, int, int, cudaStream_t);"]
    lines += decls
    for (a, b, c, d) in quartets:
        if is_split_class(a, b, c, d):
            lines.append(f"void launch_warp_{a}{b}{c}{d}(const EngineView &v, const ClassLaunch &cl, int mode, "
                         "bool ref, int prec, int grid, cudaStream_t s);")
    lines.append("")
    lines.append("// warp-cooperative launcher per class (same order as kClasses), nullptr for per-thread classes")
    lines.append("static const WarpLauncher kWarp[] = {")
    for (a, b, c, d) in quartets:
        lines.append(f"    {'launch_warp_%d%d%d%d' % (a, b, c, d) if is_split_class(a, b, c, d) else 'nullptr'},")
    lines += ["};", "", "}  // namespace hfg", ""]
    with open(os.path.join(out_dir, "eri_warp_dispatch.cuh"), "w") as fh:
        fh.write("\n".join(lines))


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    out_dir = sys.argv[1] if len(sys.argv) > 1 else here
    main(os.path.join(out_dir, "eri_gen.cuh"))
    emit_launchers(out_dir)
    emit_split(out_dir)
    emit_warp(out_dir)
