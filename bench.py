"""Benchmark: direct FP64 Fock build (ERI evaluation + J/K digestion) of a
water cluster, (H2O)_32 / 6-31G* (608 Cartesian basis functions), seeded
synthetic geometry -- the cluster of the precision-form target.

A step is one two-electron Fock build G[P] over every Schwarz-significant
shell quartet (threshold 1e-12).  The metric is ERI quartets/s: 8-fold
unique contracted function quartets of the screened build per second.

The same line carries
  "precision_form": the same cluster with the precision form (FP32 below a
      bound of 1e-4, density screening, incremental builds): a first full
      build and an incremental build, with their FP64+FP32 roofline;
  "scf": complete RHF runs of (H2O)_32 through the C++ host API (hfd_scf),
      plain FP64 vs the precision form, with energy and density errors;
  "scf_vs_reference": the reference's own RHF (compiled headless) timed on
      the host -- Init, Calculate, iterations -- beside the GPU SCF of the
      same molecules;
  "serving", "batching": the request loop and the batched SCF;
  "cpu_baseline": the reference's own ERI path on one host thread, on a
      uniform sample of the same build's quartets, as a time-to-solution rate.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 (torchrun, one rank per GPU, NCCL) the one build is sharded: each
rank evaluates its cost-balanced share of each quartet class's tasks and one
all-reduce sums the partial G (hartreefock_b200/shards.py); scaling "strong"
(the molecule is fixed), value = the whole build's quartets / the slowest
rank's time.  `--impl reference` times the reference's own CPU ERI path
(oracle/_ref, compiled headless from the reference sources) on a uniform
sample of the same build's quartets with all host threads.

Rates against the reference are time-to-solution rates: the reference
evaluates every unique quartet (it does not screen), the engine only the
Schwarz-significant ones, and both give the same G within the screening
threshold; so the reference's rate is the engine's quartet count divided by
the reference's time for its whole build (extrapolated from the sample).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WATERS = 32
BASIS = "6-31g*"
SEED = 0
THRESHOLD = 1e-12
METRIC = "ERI quartets/s"


def workload():
    from hartreefock_b200 import molecules
    Z, xyz = molecules.water_cluster(WATERS, seed=SEED)
    return Z, xyz


# DRAM bytes (read + write) per launch of a class kernel on this workload,
# from one ncu capture of the bench's own build, caches flushed before the
# launch (profiles/eri_class_kernel_ps_ss_h2o32_traffic.md)
TRAFFIC = {(1, 0, 0, 0): 26716928, (0, 0, 0, 0): 21508864}

# the large classes with a split path (primitive kernel, then HRR/digest)
SPLIT_CLASSES = {(2, 1, 1, 1), (2, 1, 2, 0), (2, 1, 2, 1), (2, 2, 1, 0), (2, 2, 1, 1), (2, 2, 2, 0), (2, 2, 2, 1),
                 (2, 2, 2, 2)}


def synthetic_density(n, seed=1):
    """A symmetric density of realistic magnitude: 2 C C^T of random
    orthonormal occupied vectors."""
    rng = np.random.default_rng(seed)
    nocc = max(1, n // 4)
    Q, _ = np.linalg.qr(rng.normal(size=(n, nocc)))
    return 2.0 * Q @ Q.T


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 25 ms from before
    the timed region to after it; the summary keeps the samples that arrived
    inside it (`mark_start` / `mark_end`), or the nearest ones when the region
    is shorter than the sampling interval."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.rows = []  # (arrival time, fields)
        self.proc = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "25"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.perf_counter() + 3.0
            while not self.rows and time.perf_counter() < deadline:  # sampler running before timing starts
                time.sleep(0.01)
        except OSError:
            self.proc = None
        return self

    def mark_start(self):
        self.t0 = time.perf_counter()

    def mark_end(self):
        self.t1 = time.perf_counter()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.perf_counter(), [x.strip() for x in line.split(",")]))

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.06)  # one more sample after the region
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = [r for t, r in self.rows if len(r) > 8]
        if self.t0 is not None and self.t1 is not None:
            inside = [r for t, r in self.rows if len(r) > 8 and self.t0 <= t <= self.t1 + 0.03]
            if not inside and rows:  # region shorter than the interval: the sample nearest its middle
                mid = 0.5 * (self.t0 + self.t1)
                inside = [min(((abs(t - mid), r) for t, r in self.rows if len(r) > 8), key=lambda x: x[0])[1]]
            rows = inside
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, name in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O  # test infrastructure: the reference built headless, and the oracle
    if not os.path.exists(O.DRIVER_PATH):
        raise RuntimeError("oracle/_ref/ref_driver missing (build with make -C oracle ref)")
    return O


def reference_rate(sample_per_thread: int, threads: int, waters: int) -> dict:
    """The reference's own CPU ERI path (IntegralsRepository::getElectronElectron,
    one repository per thread) on quartets drawn uniformly from every 8-fold
    unique quartet of the build, and the same rate as a time-to-solution rate
    on the engine's unit: the Schwarz-significant quartets of the workload
    (counted by the oracle with the engine's rule) over the time the
    reference needs for its whole build."""
    O = _oracle()
    from hartreefock_b200 import molecules
    from hartreefock_b200.basis_io import basis_path
    Z, xyz = molecules.water_cluster(waters, seed=SEED)
    mol = O.Molecule(Z, xyz, basis_path(BASIS))
    r = O.run_reference(mol, "bench", "/dev/null", extra=f"sample {sample_per_thread}\nthreads {threads}")
    out = json.loads(r["stdout"].strip().splitlines()[-1])
    raw = out["quartets"] / out["seconds"]
    cnt = O.screened_quartets(mol, THRESHOLD)
    build_s = out["unique_quartets"] / raw
    return {"raw_quartets_per_s": raw, "sampled_quartets": out["quartets"], "sample_seconds": out["seconds"],
            "threads": threads, "unique_quartets": out["unique_quartets"], "screened_quartets": cnt["kept"],
            "reference_build_s": build_s, "value": cnt["kept"] / build_s}


def reference_scf(cases) -> list:
    """The reference's own RestrictedHartreeFock (Init + Calculate, compiled
    headless) on the host, one thread, beside the GPU SCF of the same
    molecule through the C++ host API."""
    O = _oracle()
    from hartreefock_b200 import molecules, scf
    from hartreefock_b200.basis_io import basis_path
    out = []
    for name, (Z, xyz), basis, alpha, guess in cases:
        mol = O.Molecule(Z, xyz, basis_path(basis))
        t0 = time.perf_counter()
        r = O.run_reference(mol, "rhf", os.path.join(ROOT, "gpurun_out", "_ref_scf.bin") if os.path.isdir(
            os.path.join(ROOT, "gpurun_out")) else "/tmp/_ref_scf.bin", alpha=alpha, init_guess=guess, post_diis=0)
        wall = time.perf_counter() - t0
        g = scf.run_scf(Z, xyz, basis, alpha=alpha, init_guess=guess, post_diis=0)
        it = int(r["iterations"][0])
        out.append({"molecule": name, "basis": basis, "nbf": mol.nbf, "alpha": alpha, "init_guess": guess,
                    "reference": {"init_s": float(r["init_seconds"][0]), "scf_s": float(r["scf_seconds"][0]),
                                  "iterations": it, "s_per_iter": float(r["scf_seconds"][0]) / max(1, it),
                                  "wall_s": wall, "energy": float(r["energy"][0]), "cores": 1},
                    "gpu": {"init_s": g["seconds_init"], "scf_s": g["seconds_total"], "iterations": g["iterations"],
                            "s_per_iter": g["seconds_total"] / max(1, g["iterations"]), "energy": g["energy"]},
                    "abs_dE": abs(g["energy"] - float(r["energy"][0]))})
    return out


SCF_WATERS = 32


def scf_comparison(waters: int):
    """Plain FP64 vs precision-form RHF of (H2O)_waters / 6-31G*, through the
    one-call driver (C++ host API: device-resident SCF over the engine).  Each
    form runs three times and keeps its fastest wall time (the first SCF of a
    form also pays one-off costs: library handles, first allocations; the
    wall time outside Init + SCF moves by ~0.2 s between runs)."""
    from hartreefock_b200 import molecules, scf
    Z, xyz = molecules.water_cluster(waters, seed=SEED)
    kw = dict(alpha=0.75, init_guess=0.75, post_diis=0, schwarz_threshold=THRESHOLD, concurrent_classes=2)
    runs = {}
    for name, extra in (("fp64", {}), ("mixed", {"mixed_cutoff": 1e-4}),
                        ("fp64_same_criteria", {"stop_at_precision_test": True})):
        for _ in range(3):
            t0 = time.perf_counter()
            r = scf.run_scf(Z, xyz, BASIS, **kw, **extra)
            wall = time.perf_counter() - t0
            if name not in runs or wall < runs[name][0]:
                runs[name] = (wall, r)
    ref_wall, ref = runs["fp64"]

    def summary(name):
        wall, r = runs[name]
        out = {"wall_s": wall, "init_s": r["seconds_init"], "scf_s": r["seconds_total"],
               "iterations": r["iterations"], "converged": r["converged"],
               "s_per_iter": r["seconds_total"] / max(1, r["iterations"]), "energy": r["energy"],
               "fock_s": r["fock_ms_total"] / 1e3, "eigen_s": r["seconds_eigen"], "diis_s": r["seconds_diis"],
               "fock_builds": r["fock_builds"]}
        if name != "fp64":
            out["dE_vs_fp64"] = r["energy"] - ref["energy"]
            out["max_dD_vs_fp64"] = float(np.abs(r["density"] - ref["density"]).max())
        q = r["fp32_quartets"] + r["fp64_quartets"]
        if r["fp32_quartets"]:
            out["fp32_quartet_fraction"] = r["fp32_quartets"] / q
            out["incremental_builds"] = r["mixed_steps"]
        return out

    return {
        "workload": f"(H2O)_{waters} {BASIS} RHF, direct SCF, seed {SEED}; initGuess 0.75, alpha 0.75, DIIS 6/5, "
                    "no post-DIIS steps",
        "nbf": runs["fp64"][1]["nbf"],
        "fp64": dict(summary("fp64"), criteria="reference: |dE|<=1e-11, rmsD<1e-10, DIIS error<1e-10"),
        "mixed": dict(summary("mixed"), criteria="|dE|<1e-7 and rmsD<1e-7 in the incremental FP32/FP64 phase, "
                                                 "then 2 full FP64 iterations"),
        "fp64_same_criteria": dict(summary("fp64_same_criteria"), criteria="plain FP64 builds, the mixed run's rule"),
        "speedup_wall": ref_wall / runs["mixed"][0],
        "speedup_wall_same_criteria": runs["fp64_same_criteria"][0] / runs["mixed"][0],
        "speedup_init_plus_scf": (ref["seconds_init"] + ref["seconds_total"]) /
                                 (runs["mixed"][1]["seconds_init"] + runs["mixed"][1]["seconds_total"]),
        "timing": "wall of the faster of two runs per form; init_plus_scf excludes basis parsing and teardown",
    }


def serving(count: int, slots: int = 8, seed: int = 5, batch_nbf: int = 60):
    """The request loop (hartreefock_b200.serve) on a seeded Poisson stream of
    `count` RHF/UHF jobs, precision form and plain FP64 builds: saturation
    (every job submitted at once), then offered rates below it (0.25, 0.5 and
    0.75 of saturation for the precision form, 0.5 for plain FP64)."""
    from hartreefock_b200 import serve
    from hartreefock_b200.basis_io import shell_table
    jobs = serve.draw_jobs(count, seed=seed)
    out = {"workload": f"{count} jobs, seed {seed}: 80% RHF water clusters / C1-C10 alkanes, sizes log-uniform "
                       "over 5-600 functions; 20% UHF OH / planar CH3; bases 6-31G, 6-31G*, 6-31+G** (Cartesian)",
           "nbf": sorted(shell_table(Z, x, b).nbf for Z, x, b, u in jobs), "slots": slots,
           "hbm_budget_gib": 40, "eri_convention": "exact",
           "batch_lane": f"jobs of <= {batch_nbf} functions share batched SCFs (plain FP64 builds)" if batch_nbf
           else "off"}
    energies, converged = {}, {}
    for name, mixed in (("mixed", True), ("fp64", False)):
        runs = {}
        with serve.Server(slots=slots, hbm_budget=40 << 30, mixed=mixed, batch_nbf=batch_nbf) as s:
            hs, sat = serve.poisson_stream(s, jobs, rate=0.0, seed=1)
        energies[name] = [h.result["energy"] if h.error is None else None for h in hs]
        converged[name] = [h.error is None and h.result["converged"] for h in hs]
        sat["not_converged"] = sum(1 for h in hs if h.error is not None or not h.result["converged"])
        runs["saturation"] = sat
        for frac in ((0.25, 0.5, 0.75) if mixed else (0.5,)):
            with serve.Server(slots=slots, hbm_budget=40 << 30, mixed=mixed, batch_nbf=batch_nbf) as s:
                hs, part = serve.poisson_stream(s, jobs, rate=frac * sat["jobs_per_s"], seed=1)
            runs["half_load" if frac == 0.5 else f"load_{frac:.2f}"] = part
        out[name] = runs
    both = [i for i in range(len(jobs)) if converged["mixed"][i] and converged["fp64"][i]]
    d = [abs(energies["mixed"][i] - energies["fp64"][i]) for i in both]
    out["max_abs_dE_mixed_vs_fp64"] = max(d) if d else None
    out["dE_over"] = f"{len(both)} jobs converged in both forms (1000-iteration cap)"
    return out


def batch_molecules(count: int, seed: int = 0):
    """The batched-molecule mix: (H2O)_k k=1..6, staggered alkanes C1-C10,
    UHF OH / planar CH3, bases STO-3G / 6-31G drawn per molecule from a seed."""
    from hartreefock_b200 import molecules
    rng = np.random.default_rng(seed)
    kinds = [("w", k) for k in range(1, 7)] + [("a", n) for n in range(1, 11)] + [("oh", 0), ("ch3", 0)]
    rhf, uhf = [], []
    for i in range(count):
        kind, k = kinds[int(rng.integers(0, len(kinds)))]
        basis = ("sto-3g", "6-31g")[int(rng.integers(0, 2))]
        if kind == "w":
            Z, xyz = molecules.water_cluster(k, seed=int(rng.integers(0, 1 << 30)))
        elif kind == "a":
            Z, xyz = molecules.alkane(k)
        else:
            Z, xyz = molecules.hydroxyl() if kind == "oh" else molecules.methyl_planar()
        name = {"w": f"(H2O)_{k}", "a": f"C{k}H{2 * k + 2}", "oh": "OH", "ch3": "CH3"}[kind] + " " + basis
        (uhf if kind in ("oh", "ch3") else rhf).append(dict(Z=list(Z), xyz=xyz, basis=basis, name=name))
    return rhf, uhf


def batching(count: int, check: int = 8):
    """BatchSCF over the batched-molecule mix (one Fock launch per quartet
    class over every molecule per iteration); molecules/s, and |dE| against
    single-molecule FP64 runs of `check` of them."""
    import torch
    from hartreefock_b200 import batch, scf
    rhf, uhf = batch_molecules(count)
    out = {"workload": f"{count} molecules: (H2O)_1-6, alkanes C1-C10, UHF OH / CH3; STO-3G / 6-31G",
           "scf": "alpha 0.5, initGuess 0.75 (RHF and UHF), DIIS 6/5, the reference's convergence test per molecule",
           "runs": {}}
    total_wall = 0.0
    # alpha 0.5: with the reference's default 0.75 a few of the random water
    # clusters oscillate without converging (the oracle's SCF agrees)
    for name, mols, un, kw in (("rhf", rhf, False, dict(alpha=0.5, init_guess=0.75)),
                               ("uhf", uhf, True, dict(alpha=0.5, init_guess=0.75))):
        if not mols:
            continue
        t0 = time.perf_counter()
        bs = batch.BatchSCF(mols, unrestricted=un, max_iter=1000, graphs=True, **kw)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        e = bs.run()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        total_wall += t2 - t0
        errs = []
        for i in list(range(0, len(mols), max(1, len(mols) // check)))[:check]:
            m = mols[i]
            r = scf.run_scf(m["Z"], m["xyz"], m["basis"], unrestricted=un, post_diis=0, want_density=False, **kw)
            errs.append(abs(r["energy"] - e[i]))
        out["runs"][name] = {"molecules": len(mols), "setup_s": t1 - t0, "scf_s": t2 - t1,
                             "seconds": {k: round(v, 4) for k, v in bs.seconds.items()}, "fock_launch_rounds": bs.builds,
                             "max_iterations": int(bs.iterations.max()), "converged": int(bs.converged.sum()),
                             "nbf_max": bs.nmax, "max_abs_dE_vs_single_fp64": max(errs) if errs else None,
                             "cuda_graph_captures": bs.graph_captures, "graph_captured_loop": bool(bs.graphs_used),
                             "not_converged": sorted({m["name"] for m, ok in zip(mols, bs.converged) if not ok})}
    out["molecules_per_s"] = count / total_wall if total_wall else None
    return out


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    per_step, last = [], None
    for _ in range(args.warmup):
        reference_rate(500, threads, WATERS)
    for _ in range(args.steps):
        last = reference_rate(args.ref_sample, threads, WATERS)
        per_step.append(last["value"])
    value = float(np.mean(per_step))
    line = {
        "metric": METRIC, "value": value, "unit": "quartets/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * last["screened_quartets"] / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"(H2O)_{WATERS} {BASIS} direct RHF Fock build, seed {SEED}", "nbf": 19 * WATERS,
                   "schwarz_threshold": THRESHOLD, "function_quartets": last["screened_quartets"]},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "quartets/s", "cores": threads, "kind": "reference",
                         "sample": f"{args.ref_sample} quartets per thread drawn uniformly from all "
                                   f"{last['unique_quartets']} unique quartets of the build, through "
                                   "IntegralsRepository::getElectronElectron, one repository per thread; value = "
                                   "the build's Schwarz-significant quartets / the reference's extrapolated time "
                                   "for its whole (unscreened) build",
                         "raw_quartets_per_s": float(np.mean([last["raw_quartets_per_s"]])),
                         "reference_build_s": last["reference_build_s"]},
        "e2e": {"value": value, "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def precision_form(Z, xyz, P_host, local, peak64, peak32, steps=5):
    """The workload's first full build and an incremental build in the
    precision form (FP32 below a density-weighted bound of 1e-4, density
    screening at the Schwarz threshold, incremental from the density
    difference), with their FP64 + FP32 roofline: the time the evaluated
    quartets' flops need at the two measured peaks over the measured time
    (flops split by the FP64 / FP32 quartet counts)."""
    import torch
    from hartreefock_b200 import engine as E
    eng = E.Engine(Z, xyz, BASIS, schwarz_threshold=THRESHOLD, device=local, mixed_cutoff=1e-4,
                   density_screening=True, incremental=True)
    eng.set_streams(True)
    sptr = E._torch_stream()
    n = eng.nbf
    rng = np.random.default_rng(7)
    A = rng.normal(size=(n, n)) * 1e-4
    P0 = torch.from_numpy(P_host).cuda()
    P1 = torch.from_numpy(P_host + A + A.T).cuda()  # a mid-SCF-sized density change
    G = torch.empty_like(P0)
    out = {}
    for name, seq in (("first_full_build", [P0]), ("incremental_build", [P0, P1])):
        times, st = [], None
        for _ in range(steps + 1):
            eng.fock_reset()
            for k, P in enumerate(seq):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                a.record()
                eng.fock_rhf_device(P.data_ptr(), G.data_ptr(), sptr)
                b.record()
                torch.cuda.synchronize()
                if k == len(seq) - 1:
                    times.append(a.elapsed_time(b))
                    st = eng.stats()
        ms = float(np.median(times[1:]))
        q64, q32 = st["fp64_shell_quartets"], st["fp32_shell_quartets"]
        frac_eval = (q64 + q32) / max(1, st["shell_quartets"])
        f64 = st["flops"] * q64 / max(1, st["shell_quartets"])
        f32 = st["flops"] * q32 / max(1, st["shell_quartets"])
        t_min = f64 / (peak64 * 1e12) + f32 / (peak32 * 1e12)
        out[name] = {"ms": ms, "quartets_per_s": st["function_quartets"] * frac_eval / (ms / 1e3),
                     "shell_quartets_fp64": q64, "shell_quartets_fp32": q32,
                     "evaluated_fraction": frac_eval,
                     "roofline": {"bound": "fp64+fp32", "achieved_fp64_tflops": f64 / (ms / 1e3) / 1e12,
                                  "achieved_fp32_tflops": f32 / (ms / 1e3) / 1e12, "peak_fp64": peak64,
                                  "peak_fp32": peak32, "frac": t_min / (ms / 1e3),
                                  "note": "frac = (F64/peak64 + F32/peak32) / time; flops split by quartet counts"}}
    eng.close()
    return out


def main():
    global WATERS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--ref-sample", type=int, default=30000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--waters", type=int, default=WATERS,
                    help="cluster size; the benchmark workload is 32 (smaller values size profiler captures)")
    ap.add_argument("--scf-waters", type=int, default=SCF_WATERS, help="cluster of the SCF comparison (0: skip)")
    ap.add_argument("--serve-jobs", type=int, default=24, help="jobs of the serving stream (0: skip)")
    ap.add_argument("--batch-mols", type=int, default=512, help="molecules of the batched SCF (0: skip)")
    ap.add_argument("--no-reference-scf", action="store_true", help="skip the reference's SCF timing")
    ap.add_argument("--no-precision", action="store_true", help="skip the precision-form builds")
    ap.add_argument("--no-autotune", action="store_true", help="fixed grid (4 blocks per SM) for every class")
    ap.add_argument("--no-streams", action="store_true", help="every class kernel on the build stream")
    ap.add_argument("--no-graphs", action="store_true", help="launch every build's kernels (no CUDA graph replay)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    WATERS = args.waters

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    from hartreefock_b200 import engine as E

    Z, xyz = workload()
    eng = E.Engine(Z, xyz, BASIS, schwarz_threshold=THRESHOLD, device=local)
    n = eng.nbf
    P_host = synthetic_density(n)
    # a created stream: the builds on it can be captured as a CUDA graph (the
    # legacy default stream cannot)
    torch.cuda.set_stream(torch.cuda.Stream())
    stream = torch.cuda.current_stream()
    sptr = E._torch_stream()  # the builds run on torch's stream, between the timing events
    dP = torch.from_numpy(P_host).cuda()
    dG = torch.empty_like(dP)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2

    # the whole molecule's build (units of the metric; reference G for the check)
    eng.fock_rhf_device(dP.data_ptr(), dG.data_ptr(), sptr)
    torch.cuda.synchronize()
    stats_full = eng.stats()
    G_full = dG.clone()
    # the classes of every build over concurrent streams, then the grid from
    # the autotuner (timed on this density, before warm-up)
    # task shapes (lanes per quartet for long contractions) from the task
    # autotuner, then the classes of every build over concurrent streams
    # and the grid from the grid autotuner (both timed on this density,
    # before warm-up)
    # (one rank only: the lane-group targets decide how the quartets split
    # into tasks, and the shards are task ranges, so every rank of a sharded
    # run must build the same task lists: they keep the default target)
    tasks = eng.autotune_tasks(dP) if not args.no_autotune and world == 1 else {}
    # the large classes' kernel (warp-cooperative or split), timed both ways
    paths = eng.autotune_paths(dP) if not args.no_autotune else {}
    eng.set_streams(not args.no_streams)
    grids = eng.autotune(dP) if not args.no_autotune else {}
    # the plain-form build replays one CUDA graph per buffers and stream
    # (captured during the warm-up steps; the host-buffer entry point gets
    # its own on the context's stream)
    eng.set_graphs(not args.no_graphs)
    # N > 1: every rank builds its shard of each class's tasks, one NCCL
    # all-reduce of G per build (hartreefock_b200/shards.py)
    sf = None
    if dist:
        from hartreefock_b200.shards import ShardedFock
        sf = ShardedFock(eng)

    def step():
        if sf:
            sf.fock_rhf(dP, dG)
        else:
            eng.fock_rhf_device(dP.data_ptr(), dG.data_ptr(), sptr)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    stats = eng.stats()
    assert torch.allclose(dG, G_full, atol=1e-9)

    # ---- device-timed value: per-step events, L2 flushed between steps
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        clocks.mark_start()
        for a, b in evs:
            flush.zero_()
            a.record(stream)
            step()
            b.record(stream)
        torch.cuda.synchronize()
        clocks.mark_end()
    if dist:
        dist.barrier()
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    quartets = stats_full["function_quartets"]
    value = quartets * args.steps / (total_ms / 1e3)

    # ---- end to end from host buffers: N = 1 through the public host-buffer
    # entry point hfg_fock_rhf (H2D of P, build, D2H of G inside the call);
    # N > 1 the same by hand around the sharded build and its all-reduce
    P_pin = torch.from_numpy(P_host).pin_memory()
    G_pin = torch.empty(n, n, dtype=torch.float64).pin_memory()

    def e2e_step():
        if sf:
            dP.copy_(P_pin, non_blocking=True)
            sf.fock_rhf(dP, dG)
            G_pin.copy_(dG, non_blocking=True)
            torch.cuda.current_stream().synchronize()
        else:
            eng.fock_rhf(P_pin.numpy(), out=G_pin.numpy())

    for _ in range(2):  # the second call captures the host-buffer build's graph
        e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_ms = (time.perf_counter() - t0) * 1e3
    assert np.allclose(G_pin.numpy(), G_full.cpu().numpy(), atol=1e-9)
    if dist:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = quartets * args.steps / (e2e_ms / 1e3)

    # ---- roofline of the dominant class kernel (profiled pass, events per class)
    eng.set_profiling(True)
    step()
    torch.cuda.synchronize()
    prof = eng.class_profile()
    eng.set_profiling(False)
    top = max(prof, key=lambda c: c["ms"])
    peak = E.measure_fp64_peak(local)
    peak32 = E.measure_fp32_peak(local)
    # algorithmic flops: the reference's recursion loops walked per class
    # (hartreefock_b200/flops.py) x the class's primitive and shell quartets;
    # the engine's own count of its generated code beside it.  Class figures
    # are whole-class; a shard runs 1/world of them.
    from hartreefock_b200 import flops as FL

    def walk(c):
        fp, fs = FL.class_flops(c["la"], c["lb"], c["lc"], c["ld"])
        return c["primitive_quartets"] * fp + c["shell_quartets"] * fs

    achieved = walk(top) / world / (top["ms"] / 1e3) / 1e12
    achieved_gen = top["flops"] / world / (top["ms"] / 1e3) / 1e12
    build_flops = sum(walk(c) for c in prof)
    build_flops_gen = stats_full["flops"]

    line = {
        "metric": METRIC, "value": value, "unit": "quartets/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"(H2O)_{WATERS} {BASIS} direct RHF Fock build, seed {SEED}", "nbf": n,
                   "schwarz_threshold": THRESHOLD, "shell_quartets": stats_full["shell_quartets"],
                   "function_quartets": stats_full["function_quartets"],
                   "l2": "flushed (256 MB write) between steps",
                   "grid_blocks_per_sm": grids or ("fixed 4" if args.no_streams else "fixed 1"),
                   "large_class_kernels": paths or "default: warp for (22|22), split for the rest",
                   "prim_quartets_per_lane_target": tasks or "fixed 96",
                   "class_streams": 1 if args.no_streams else 13,
                   "cuda_graph": not args.no_graphs,
                   "parallelism": f"task shards x{world}, one NCCL all-reduce of G per build" if world > 1
                   else "single GPU"},
        "e2e": {"value": e2e, "unit": "quartets/s", "h2d_bytes_per_step": n * n * 8, "d2h_bytes_per_step": n * n * 8},
        "gpu_launches": stats["kernel_launches"] * args.steps,
        "roofline": {"bound": "fp64", "kernel": f"({top['la']}{top['lb']}|{top['lc']}{top['ld']}) J/K class kernel",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "peak_source": "measured in-run: FP64 FMA microbenchmark (hfg_measure_fp64_peak)",
                     "flop_count": "reference recursion loops walked per class (hartreefock_b200/flops.py)",
                     "achieved_generated_code_count": achieved_gen,
                     "traffic": TRAFFIC.get((top["la"], top["lb"], top["lc"], top["ld"])),
                     "traffic_unit": "DRAM bytes per launch (ncu capture of this workload, profiles/)",
                     "build": {"achieved": build_flops / world / (total_ms / args.steps / 1e3) / 1e12,
                               "frac": build_flops / world / (total_ms / args.steps / 1e3) / 1e12 / peak,
                               "achieved_generated_code_count":
                                   build_flops_gen / world / (total_ms / args.steps / 1e3) / 1e12},
                     "fp32_peak": peak32},
        "classes": [{"class": f"({c['la']}{c['lb']}|{c['lc']}{c['ld']})", "ms": round(c["ms"], 4),
                     "tflops": round(c["flops"] / max(c["ms"], 1e-9) / 1e9, 3), "tasks": c["tasks"],
                     "lane_occupancy": round(c["lane_occupancy"], 3),
                     "kernel": "warp per quartet" if c["warp_kernel"] else
                     "split: thread per quartet, then HRR/digest" if (c["la"], c["lb"], c["lc"], c["ld"]) in SPLIT_CLASSES
                     else "thread per quartet"} for c in prof],
        "clocks": clocks.summary(),
    }
    eng.close()
    torch.cuda.synchronize()
    torch.cuda.set_stream(torch.cuda.default_stream())  # the remaining parts as before
    if rank == 0 and world == 1 and not args.no_precision:
        line["precision_form"] = precision_form(Z, xyz, P_host, local, peak, peak32)
        line["roofline"]["fp32"] = line["precision_form"]["first_full_build"]["roofline"]
    if rank == 0 and world == 1 and args.scf_waters > 0:
        line["scf"] = scf_comparison(args.scf_waters)
    if rank == 0 and world == 1 and not args.no_reference_scf:
        from hartreefock_b200 import molecules
        line["scf_vs_reference"] = reference_scf([
            ("H2O (README geometry)", molecules.H2O_README, "sto-3g", 0.5, 0.0),
            ("(H2O)_2 seed 0", molecules.water_cluster(2, seed=0), "6-31g*", 0.75, 0.75)])
    if rank == 0 and world == 1 and args.serve_jobs > 0:
        line["serving"] = serving(args.serve_jobs)
    if rank == 0 and world == 1 and args.batch_mols > 0:
        line["batching"] = batching(args.batch_mols)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = reference_rate(args.ref_sample, 1, WATERS)
        line["cpu_baseline"] = {"value": cb["value"], "unit": "quartets/s", "cores": 1, "kind": "reference",
                                "sample": f"{cb['sampled_quartets']} quartets drawn uniformly from all "
                                          f"{cb['unique_quartets']} unique quartets of the same cluster, through the "
                                          "reference's IntegralsRepository::getElectronElectron, 1 thread; value = "
                                          "the build's Schwarz-significant quartets / the reference's extrapolated "
                                          "time for its whole (unscreened) build",
                                "raw_quartets_per_s": cb["raw_quartets_per_s"],
                                "reference_build_s": cb["reference_build_s"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
