"""Request loop for RHF/UHF jobs: continuous admission against an HBM budget.

Jobs arrive at any time (Server.submit).  Each job is one SCF run through
the driver (hfd_scf: RestrictedHartreeFock / UnrestrictedHartreeFock Init +
Calculate over the direct GPU Fock builds), so its engine context (shell
pairs, Schwarz and screening tables, quartet task lists) and its density,
Fock matrix and DIIS history stay resident in HBM for the life of the job,
on the job's own CUDA stream.  A fixed number of slots (worker threads; the
driver call releases the GIL) run jobs at the same time, so the kernels of
different jobs overlap on the device.  Jobs are admitted in arrival order as
soon as a slot is free and the job's estimated device footprint fits in what
is left of the budget; a job larger than the whole budget is refused with
HFG_OOM_BUDGET.  Latency = completion time - submit time.

The reference runs one algorithm object per std::thread with no shared
state (HartreeFockDoc.cpp:372-405); a slot here is that thread, with the
device as the shared resource the budget guards.

Jobs use the exact electron-transfer recursion (HFG_ERI_EXACT) by
default: the reference's (dd|dd) transfer (GaussianTwoElectrons.cpp:162)
drops terms that matter when d shells on neighbouring atoms overlap, and
propane in 6-31G* then has no physical solution (its SCF wanders below
-1100 Eh instead of converging near -118.25 Eh).  The parity tests keep the
reference convention; a caller can pass eri_convention to Server.

draw_jobs() and poisson_stream() make and replay the synthetic request
stream: 80% RHF water clusters / alkanes (C1-C10, larger sizes as water
clusters) with sizes log-uniform over a function-count range, 20% UHF
doublets (OH, planar CH3), bases drawn uniformly from 6-31G, 6-31G*,
6-31+G** (Cartesian).
"""
from __future__ import annotations

import collections
import ctypes
import math
import threading
import time

import numpy as np

from . import engine as E
from . import molecules
from . import scf as _scf
from .basis_io import basis_path, shell_table

HFG_OOM_BUDGET = 3
SERVE_BASES = ("6-31g", "6-31g*", "6-31+g**")


def footprint_bytes(Z, xyz, basis: str, unrestricted: bool = False) -> int:
    """Estimated device bytes of one job, the estimate the native pool uses
    too (job_footprint_bytes in hartreefock_b200/csrc/host.cpp): quartet task
    lists (16 B per task of up to 32 ket pairs over the triangle of shell
    pairs), primitive-pair tables (96 B FP64 + 48 B FP32 per primitive pair),
    the SCF's n x n FP64 matrices (h, S, V, F, P, new P, C, G, work, 2 x 6
    DIIS entries, the incremental history; about 32 per spin), plus a fixed
    16 MiB for the Boys table, counters and library handles."""
    t = shell_table(Z, xyz, basis)
    ns = len(t.L)
    pairs = ns * (ns + 1) // 2
    prim_pairs = int(np.sum(np.triu(np.outer(t.nprim, t.nprim))))
    tasks = pairs * (pairs + 1) // 2 // 32 + pairs
    spins = 2 if unrestricted else 1
    return int(16 * tasks + 144 * prim_pairs + 8 * t.nbf * t.nbf * 32 * spins + (16 << 20))


class Job:
    """One request; wait() blocks until it has finished."""

    def __init__(self, jid, Z, xyz, basis, unrestricted, kwargs):
        self.id, self.Z, self.xyz, self.basis = jid, list(Z), np.asarray(xyz, dtype=np.float64), basis
        self.unrestricted, self.kwargs = unrestricted, dict(kwargs)
        self.bytes = footprint_bytes(self.Z, self.xyz, basis, unrestricted)
        self.nbf = shell_table(self.Z, self.xyz, basis).nbf
        self.t_submit = self.t_start = self.t_end = None
        self.result, self.error = None, None
        self._done = threading.Event()

    def wait(self, timeout=None):
        if not self._done.wait(timeout):
            raise TimeoutError(f"job {self.id} still running")
        if self.error is not None:
            raise self.error
        return self.result

    @property
    def latency(self) -> float:
        return self.t_end - self.t_submit

    @property
    def done(self) -> bool:
        return self._done.is_set()


def _driver_runner(job: Job):
    from . import scf
    return scf.run_scf(job.Z, job.xyz, job.basis, unrestricted=job.unrestricted, want_density=False, **job.kwargs)


class Server:
    """slots: jobs on the device at once.  hbm_budget: bytes the admitted
    jobs' footprints may add up to.  mixed: precision form of the Fock
    builds (FP32 below mixed_cutoff, incremental, FP64 finish) for every
    job; otherwise plain FP64 builds.  Both stop on the precision form's
    rule (|dE| < 1e-7, rms dD < 1e-7, DIIS error < 1e-7, then two full FP64
    iterations), so the two differ only in their kernels.  scf_kwargs go to every job's SCF
    (scf.run_scf keywords); the defaults here are post_diis 0 (the
    reference's convergence test alone), at most 1000 iterations, the exact
    ERI convention and each job's class kernels on concurrent streams (no
    CUDA graphs: their capture does not mix with other threads' device-wide
    synchronisation).  runner(job) -> result replaces the driver call
    (host-side tests)."""

    def __init__(self, slots: int = 8, hbm_budget: int = 32 << 30, mixed: bool = True, mixed_cutoff: float = 1e-4,
                 scf_kwargs=None, runner=None, concurrent_classes: bool = True, batch_nbf: int = 0,
                 batch_min: int = 4, batch_max: int = 64, batch_window_s: float = 0.005):
        if slots < 1 or hbm_budget <= 0:
            raise ValueError("slots >= 1 and a positive budget are required")
        self.slots, self.budget = slots, int(hbm_budget)
        # batch lane for small jobs (at most batch_nbf functions): when at
        # least batch_min of them with the same SCF settings wait in the queue,
        # one more worker takes them (up to batch_max, after batch_window_s for
        # others arriving together) and runs them as one batched SCF
        # (hartreefock_b200.batch.BatchSCF: one Fock launch per quartet class
        # over all of them per iteration, plain FP64 builds, the reference's
        # convergence test per molecule).  Below that the slots take them in
        # arrival order like any job: a batch of one or two runs the batched
        # loop's per-iteration host work for little gain.
        self.batch_nbf, self.batch_max, self.batch_window_s = int(batch_nbf), int(batch_max), float(batch_window_s)
        self.batch_min = int(batch_min)
        self.batches = []  # sizes of the batches run
        # the switch rule's DIIS error at 1e-7 (the SCF default is 1e-6): jobs of
        # the stream with diffuse functions otherwise end up to ~1.3e-6 Eh apart
        # between the two forms
        self.defaults = dict(post_diis=0, max_iterations=1000, eri_convention=E.ERI_EXACT, mixed_switch_diis=1e-7,
                             concurrent_classes=1 if concurrent_classes else 0)
        if mixed:
            self.defaults["mixed_cutoff"] = mixed_cutoff
        else:
            self.defaults["stop_at_precision_test"] = True
        self.defaults.update(scf_kwargs or {})
        self.runner = runner or _driver_runner
        self._cv = threading.Condition()
        self._queue = collections.deque()
        self._in_use = 0
        self._running = 0
        self._next_id = 0
        self._closing = False
        self.peak_bytes = 0
        self.peak_running = 0
        self.finished = []
        self._workers = [threading.Thread(target=self._work, name=f"hfg-slot-{i}", daemon=True) for i in range(slots)]
        if self.batch_nbf > 0:
            self._workers.append(threading.Thread(target=self._batch_work, name="hfg-batch", daemon=True))
        for w in self._workers:
            w.start()

    def submit(self, Z, xyz, basis: str, unrestricted: bool = False, **kwargs) -> Job:
        kw = dict(self.defaults)
        kw.update(kwargs)
        with self._cv:
            if self._closing:
                raise RuntimeError("server is closed")
            job = Job(self._next_id, Z, xyz, basis, unrestricted, kw)
            self._next_id += 1
            job.t_submit = time.perf_counter()
            if job.bytes > self.budget:
                from .engine import HfgError
                job.error = HfgError(HFG_OOM_BUDGET, f"job needs ~{job.bytes} B, budget {self.budget} B")
                job.t_start = job.t_end = job.t_submit
                job._done.set()
                return job
            self._queue.append(job)
            self._cv.notify_all()
        return job

    def _small_groups(self):
        """{SCF settings: queued small jobs} (caller holds the lock)."""
        groups = {}
        if self.batch_nbf > 0 and self.runner is _driver_runner:
            for j in self._queue:
                if j.nbf <= self.batch_nbf:
                    groups.setdefault(self._batch_key(j), []).append(j)
        return groups

    @staticmethod
    def _batch_key(job):
        k = job.kwargs
        return (job.unrestricted, k.get("alpha", 0.75), k.get("init_guess", 0.75), k.get("max_iterations", 0),
                k.get("eri_convention", E.ERI_REFERENCE), k.get("schwarz_threshold", 1e-12))

    def _take_batch(self):
        """The largest group of queued small jobs with the same settings if it
        has batch_min of them, up to batch_max that fit the budget together,
        out of the queue (caller holds the lock)."""
        groups = self._small_groups()
        if not groups:
            return []
        group = max(groups.values(), key=len)
        if len(group) < self.batch_min:
            return []
        picked, used = [], 0
        for j in group[:self.batch_max]:
            if self._in_use + used + j.bytes <= self.budget:
                picked.append(j)
                used += j.bytes
        if len(picked) < self.batch_min:
            return []
        ids = {id(j) for j in picked}
        self._queue = collections.deque(j for j in self._queue if id(j) not in ids)
        self._in_use += used
        self._running += len(picked)
        self.peak_bytes = max(self.peak_bytes, self._in_use)
        self.peak_running = max(self.peak_running, self._running)
        return picked

    def _batch_work(self):
        from . import batch as _batch
        while True:
            with self._cv:
                while max((len(g) for g in self._small_groups().values()), default=0) < self.batch_min:
                    if self._closing:
                        from . import scf
                        scf.release_thread()
                        return
                    self._cv.wait(0.05)
            time.sleep(self.batch_window_s)  # let jobs arriving together share the batch
            with self._cv:
                jobs = self._take_batch()
                if not jobs:
                    self._cv.wait(0.01)  # taken by the slots meanwhile, or the budget is held
                    continue
            t0 = time.perf_counter()
            for j in jobs:
                j.t_start = t0
            try:
                k = jobs[0].kwargs
                bs = _batch.BatchSCF([dict(Z=j.Z, xyz=j.xyz, basis=j.basis) for j in jobs],
                                     unrestricted=jobs[0].unrestricted, alpha=k.get("alpha", 0.75),
                                     init_guess=k.get("init_guess", 0.75), max_iter=k.get("max_iterations", 0) or 3000,
                                     schwarz_threshold=k.get("schwarz_threshold", 1e-12),
                                     eri_convention=k.get("eri_convention", E.ERI_REFERENCE), graphs=False)
                energies = bs.run()
                for i, j in enumerate(jobs):
                    j.result = {"energy": float(energies[i]), "converged": bool(bs.converged[i]),
                                "iterations": int(bs.iterations[i]), "batched": len(jobs)}
                bs.eng.close()
            except Exception as e:  # reported through Job.wait
                for j in jobs:
                    j.error = e
            t1 = time.perf_counter()
            with self._cv:
                for j in jobs:
                    j.t_end = t1
                    self._in_use -= j.bytes
                    self._running -= 1
                    self.finished.append(j)
                self.batches.append(len(jobs))
                self._cv.notify_all()
            for j in jobs:
                j._done.set()

    def _admit(self):
        """Head of the queue if it fits (caller holds the lock)."""
        if self._queue and self._in_use + self._queue[0].bytes <= self.budget:
            job = self._queue.popleft()
            self._in_use += job.bytes
            self._running += 1
            self.peak_bytes = max(self.peak_bytes, self._in_use)
            self.peak_running = max(self.peak_running, self._running)
            return job
        return None

    def _work(self):
        while True:
            with self._cv:
                job = self._admit()
                while job is None:
                    if self._closing and not self._queue:
                        if self.runner is _driver_runner:
                            from . import scf
                            scf.release_thread()  # this thread's handles, while CUDA is up
                        return
                    self._cv.wait()
                    job = self._admit()
            job.t_start = time.perf_counter()
            try:
                job.result = self.runner(job)
            except Exception as e:  # reported through Job.wait
                job.error = e
            job.t_end = time.perf_counter()
            with self._cv:
                self._in_use -= job.bytes
                self._running -= 1
                self.finished.append(job)
                self._cv.notify_all()
            job._done.set()

    def drain(self, timeout=None):
        """Wait until every submitted job has finished."""
        deadline = None if timeout is None else time.monotonic() + timeout
        with self._cv:
            while self._queue or self._running:
                left = None if deadline is None else deadline - time.monotonic()
                if left is not None and left <= 0:
                    raise TimeoutError("jobs still queued or running")
                self._cv.wait(left)

    def close(self):
        with self._cv:
            self._closing = True
            self._cv.notify_all()
        for w in self._workers:
            w.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---------------------------------------------------------------------------
# the native pool (C ABI hfg_pool_*, hartreefock_b200/csrc/pool.cpp)

class hfg_job_spec(ctypes.Structure):
    _fields_ = [("basis_path", ctypes.c_char_p), ("natoms", ctypes.c_int32), ("Z", ctypes.c_void_p),
                ("xyz", ctypes.c_void_p), ("opts", _scf.hfd_scf_opts), ("timeout_s", ctypes.c_double)]


class hfg_job_info(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("status", ctypes.c_int32), ("queue_s", ctypes.c_double),
                ("run_s", ctypes.c_double), ("latency_s", ctypes.c_double), ("footprint_bytes", ctypes.c_int64),
                ("result", _scf.hfd_scf_result)]


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_CANCELLED, JOB_TIMEOUT = range(6)
POOL_SYMBOLS = ["hfg_pool_create", "hfg_job_submit", "hfg_job_poll", "hfg_job_wait", "hfg_job_cancel",
                "hfg_pool_stats", "hfg_pool_last_error", "hfg_pool_destroy"]


def _pool_lib():
    L = E.library()
    if not getattr(L, "_pool_ready", False):
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
        L.hfg_pool_create.argtypes = [i32, i64, ctypes.POINTER(vp)]
        L.hfg_job_submit.argtypes = [vp, ctypes.POINTER(hfg_job_spec), ctypes.POINTER(i64)]
        L.hfg_job_poll.argtypes = [vp, i64, ctypes.POINTER(hfg_job_info)]
        L.hfg_job_wait.argtypes = [vp, i64, ctypes.c_double, ctypes.POINTER(hfg_job_info)]
        L.hfg_job_cancel.argtypes = [vp, i64]
        L.hfg_pool_stats.argtypes = [vp, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i64)]
        L.hfg_pool_last_error.restype = ctypes.c_char_p
        L.hfg_pool_destroy.argtypes = [vp]
        L.hfg_pool_destroy.restype = None
        for n in ("hfg_pool_create", "hfg_job_submit", "hfg_job_poll", "hfg_job_wait", "hfg_job_cancel",
                  "hfg_pool_stats"):
            getattr(L, n).restype = ctypes.c_int
        L._pool_ready = True
    return L


class NativeJob:
    """A job of the native pool: wait(), cancel(), state, result, latency."""

    def __init__(self, server, jid, t_submit, keep):
        self.server, self.id, self.t_submit, self._keep = server, jid, t_submit, keep
        self.result, self.error, self.info = None, None, None
        self.t_end = None
        self._done = self  # poisson_stream waits on job._done.wait(timeout)

    def _update(self, info):
        self.info = info
        if info.state >= JOB_DONE and self.t_end is None:
            self.t_end = self.t_submit + info.latency_s
            r = _scf.result_dict(info.result)
            if info.state == JOB_DONE:
                self.result = r
            else:
                self.result = r
                self.error = E.HfgError(info.status, {JOB_FAILED: "failed", JOB_CANCELLED: "cancelled",
                                                      JOB_TIMEOUT: "timed out"}[info.state])

    def wait(self, timeout=None):
        info = hfg_job_info()
        st = _pool_lib().hfg_job_wait(self.server._h, self.id, float(timeout or 0), ctypes.byref(info))
        self._update(info)
        if st != 0 and info.state < JOB_DONE:
            raise TimeoutError(f"job {self.id} still running")
        if self.error is not None:
            raise self.error
        return self.result

    def poll(self) -> int:
        info = hfg_job_info()
        _check_pool(_pool_lib().hfg_job_poll(self.server._h, self.id, ctypes.byref(info)))
        self._update(info)
        return info.state

    def cancel(self):
        _check_pool(_pool_lib().hfg_job_cancel(self.server._h, self.id))

    @property
    def latency(self) -> float:
        return self.info.latency_s

    @property
    def done(self) -> bool:
        return self.poll() >= JOB_DONE


def _check_pool(st):
    if st != 0:
        raise E.HfgError(st, _pool_lib().hfg_pool_last_error().decode())


class NativeServer:
    """The request loop in native code (hfg_pool_*): the same slots, budget,
    arrival-order admission and SCF defaults as Server, with the queue,
    admission, cancellation and timeouts in C++ worker threads."""

    def __init__(self, slots: int = 8, hbm_budget: int = 32 << 30, mixed: bool = True, mixed_cutoff: float = 1e-4,
                 scf_kwargs=None, concurrent_classes: bool = True):
        self.slots, self.budget = slots, int(hbm_budget)
        self.defaults = dict(post_diis=0, max_iterations=1000, eri_convention=E.ERI_EXACT, mixed_switch_diis=1e-7,
                             concurrent_classes=1 if concurrent_classes else 0)
        if mixed:
            self.defaults["mixed_cutoff"] = mixed_cutoff
        else:
            self.defaults["stop_at_precision_test"] = True
        self.defaults.update(scf_kwargs or {})
        h = ctypes.c_void_p()
        _check_pool(_pool_lib().hfg_pool_create(slots, self.budget, ctypes.byref(h)))
        self._h = h
        self.peak_running, self.peak_bytes = 0, 0
        self._stop = threading.Event()
        self._sampler = threading.Thread(target=self._sample, daemon=True)
        self._sampler.start()

    def _sample(self):
        r, q, b = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        while not self._stop.wait(0.005):
            if _pool_lib().hfg_pool_stats(self._h, ctypes.byref(r), ctypes.byref(q), ctypes.byref(b)) == 0:
                self.peak_running = max(self.peak_running, r.value)
                self.peak_bytes = max(self.peak_bytes, b.value)

    def submit(self, Z, xyz, basis: str, unrestricted: bool = False, timeout_s: float = 0.0, **kwargs) -> NativeJob:
        kw = dict(self.defaults)
        kw.update(kwargs)
        z = np.ascontiguousarray(Z, dtype=np.int32)
        x = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
        spec = hfg_job_spec()
        path = basis_path(basis).encode()
        spec.basis_path, spec.natoms = path, len(z)
        spec.Z, spec.xyz = z.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p)
        spec.opts = _scf.scf_opts(unrestricted=unrestricted, **kw)
        spec.timeout_s = float(timeout_s)
        jid = ctypes.c_int64()
        t = time.perf_counter()
        _check_pool(_pool_lib().hfg_job_submit(self._h, ctypes.byref(spec), ctypes.byref(jid)))
        return NativeJob(self, jid.value, t, (z, x, path))

    def close(self):
        if getattr(self, "_h", None):
            self._stop.set()
            self._sampler.join()
            _pool_lib().hfg_pool_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---------------------------------------------------------------------------
# synthetic request stream

def _functions_per_atom(basis: str) -> dict:
    return {z: shell_table([z], np.zeros((1, 3)), basis).nbf for z in (1, 6, 8)}


def _rhf_molecule(target: float, basis: str, rng, fpa):
    """Water cluster or alkane (C1-C10) whose function count is nearest the
    target; targets beyond decane are water clusters."""
    water = fpa[8] + 2 * fpa[1]
    per_c, base = fpa[6] + 2 * fpa[1], 2 * fpa[1]
    if rng.random() < 0.5 or target > 10 * per_c + base:
        k = max(1, int(round(target / water)))
        Z, xyz = molecules.water_cluster(k, seed=int(rng.integers(0, 1 << 30)))
    else:
        n = max(1, int(round((target - base) / per_c)))
        Z, xyz = molecules.alkane(n)
    return list(Z), xyz


def draw_jobs(count: int, seed: int = 0, nbf_range=(5, 600), uhf_fraction: float = 0.2, bases=SERVE_BASES):
    """[(Z, xyz, basis, unrestricted)]: RHF sizes log-uniform over nbf_range
    (realised as the nearest water cluster or alkane), UHF OH / planar CH3."""
    rng = np.random.default_rng(seed)
    fpa = {b: _functions_per_atom(b) for b in bases}
    lo, hi = math.log(nbf_range[0]), math.log(nbf_range[1])
    out = []
    for _ in range(count):
        basis = bases[int(rng.integers(0, len(bases)))]
        if rng.random() < uhf_fraction:
            Z, xyz = molecules.hydroxyl() if rng.random() < 0.5 else molecules.methyl_planar()
            out.append((list(Z), xyz, basis, True))
        else:
            Z, xyz = _rhf_molecule(math.exp(rng.uniform(lo, hi)), basis, rng, fpa[basis])
            out.append((Z, xyz, basis, False))
    return out


# SCF settings of the stream (HartreeFockAlgorithm::alpha / initGuess): the
# pair under which most jobs of the mix converge within the iteration cap
UHF_KW = dict(alpha=0.75, init_guess=0.75)
RHF_KW = dict(alpha=0.5, init_guess=0.0)


def poisson_stream(server: Server, jobs, rate: float, seed: int = 0, timeout=None):
    """Submit `jobs` with exponential inter-arrival times of mean 1/rate
    seconds (rate in jobs/s; rate <= 0 submits all at once), wait for all,
    and return (job objects, summary dict)."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=len(jobs)) if rate > 0 else np.zeros(len(jobs))
    handles = []
    t0 = time.perf_counter()
    t_next = t0
    for (Z, xyz, basis, uhf), gap in zip(jobs, gaps):
        t_next += gap
        delay = t_next - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        handles.append(server.submit(Z, xyz, basis, unrestricted=uhf, **(UHF_KW if uhf else RHF_KW)))
    for h in handles:
        try:
            h._done.wait(timeout)
        except E.HfgError:
            pass  # counted below through h.error
    t_end = max(h.t_end for h in handles)
    lat = np.array([h.latency for h in handles if h.error is None]) * 1e3
    summary = {"offered_rate": rate, "jobs": len(handles), "failed": sum(h.error is not None for h in handles),
               "jobs_per_s": len(handles) / (t_end - t0), "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
               "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
               "peak_running": server.peak_running, "peak_bytes": server.peak_bytes}
    if getattr(server, "batch_nbf", 0) > 0:
        summary["batched_jobs"] = int(sum(server.batches))
        summary["batches"] = len(server.batches)
    return handles, summary
