"""ctypes binding of the one-call SCF driver (include/hfgpu_driver.h).

The SCF itself is the C++ host code (include/hfgpu_host.hpp): the
reference's RestrictedHartreeFock / UnrestrictedHartreeFock loop with its
defaults, DIIS and convergence thresholds, over the GPU Fock builds.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import engine as E
from .basis_io import basis_path


class hfd_scf_opts(ctypes.Structure):
    _fields_ = [("unrestricted", ctypes.c_int32), ("alpha", ctypes.c_double), ("init_guess", ctypes.c_double),
                ("use_diis", ctypes.c_int32), ("post_diis", ctypes.c_int32), ("alpha_electrons", ctypes.c_int32),
                ("beta_electrons", ctypes.c_int32), ("eri_convention", ctypes.c_int32),
                ("schwarz_threshold", ctypes.c_double), ("mixed_cutoff", ctypes.c_double),
                ("mixed_switch_energy", ctypes.c_double), ("mixed_switch_density", ctypes.c_double),
                ("mixed_switch_diis", ctypes.c_double),
                ("fp64_final_iterations", ctypes.c_int32), ("fp64_final_converge", ctypes.c_int32),
                ("incremental", ctypes.c_int32), ("trace", ctypes.c_int32),
                ("stop_at_precision_test", ctypes.c_int32), ("max_iterations", ctypes.c_int32),
                ("mp2", ctypes.c_int32), ("concurrent_classes", ctypes.c_int32),
                ("electric_field", ctypes.c_double * 3), ("shard_rank", ctypes.c_int32),
                ("shard_count", ctypes.c_int32), ("allreduce", ctypes.c_void_p), ("allreduce_user", ctypes.c_void_p)]


# hfd_allreduce_fn: (device G, count, stream, user)
ALLREDUCE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p)


class hfd_scf_result(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("homo", ctypes.c_double), ("converged", ctypes.c_int32),
                ("iterations", ctypes.c_int32), ("nbf", ctypes.c_int32), ("fock_builds", ctypes.c_int32),
                ("fock_ms_total", ctypes.c_double), ("fp32_quartets", ctypes.c_int64),
                ("fp64_quartets", ctypes.c_int64), ("mixed_steps", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("seconds_fock", ctypes.c_double), ("seconds_eigen", ctypes.c_double),
                ("seconds_diis", ctypes.c_double), ("seconds_total", ctypes.c_double),
                ("seconds_init", ctypes.c_double), ("mp2_energy", ctypes.c_double), ("dipole", ctypes.c_double * 3)]


DRIVER_SYMBOLS = ["hfd_default_scf_opts", "hfd_last_error", "hfd_scf", "hfd_one_electron", "hfd_pulay_solve",
                  "hfd_release_thread", "hfd_load_xyz"]


def _lib():
    L = E.library()
    if not getattr(L, "_hfd_ready", False):
        L.hfd_default_scf_opts.argtypes = [ctypes.POINTER(hfd_scf_opts)]
        L.hfd_default_scf_opts.restype = None
        L.hfd_last_error.restype = ctypes.c_char_p
        L.hfd_scf.argtypes = [ctypes.c_char_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.POINTER(hfd_scf_opts), ctypes.POINTER(hfd_scf_result), ctypes.c_void_p,
                              ctypes.c_int64]
        L.hfd_scf.restype = ctypes.c_int
        L.hfd_one_electron.argtypes = [ctypes.c_char_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                       ctypes.POINTER(ctypes.c_int32)]
        L.hfd_one_electron.restype = ctypes.c_int
        L.hfd_load_xyz.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]
        L.hfd_load_xyz.restype = ctypes.c_int
        L.hfg_copy_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
        L.hfg_copy_device.restype = ctypes.c_int
        L.hfd_pulay_solve.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]
        L.hfd_pulay_solve.restype = ctypes.c_int
        L.hfd_release_thread.argtypes = []
        L.hfd_release_thread.restype = None
        L._hfd_ready = True
    return L


def scf_opts(unrestricted=False, alpha=0.75, init_guess=0.75, use_diis=True, post_diis=500,
             alpha_electrons=0, beta_electrons=0, eri_convention=E.ERI_REFERENCE, schwarz_threshold=1e-12,
             mixed_cutoff=0.0, mixed_switch_energy=1e-7, mixed_switch_density=1e-7, mixed_switch_diis=1e-6,
             fp64_final_iterations=2, fp64_final_converge=False, incremental=False, trace=False,
             stop_at_precision_test=False, max_iterations=0, mp2=False, concurrent_classes=False,
             electric_field=(0.0, 0.0, 0.0)) -> hfd_scf_opts:
    """hfd_scf_opts from keywords (the defaults of hfd_default_scf_opts where
    not given)."""
    L = _lib()
    o = hfd_scf_opts()
    L.hfd_default_scf_opts(ctypes.byref(o))
    o.unrestricted, o.alpha, o.init_guess = int(unrestricted), alpha, init_guess
    o.use_diis, o.post_diis = int(use_diis), post_diis
    o.alpha_electrons, o.beta_electrons = alpha_electrons, beta_electrons
    o.eri_convention, o.schwarz_threshold = eri_convention, schwarz_threshold
    o.mixed_cutoff, o.mixed_switch_energy = mixed_cutoff, mixed_switch_energy
    o.fp64_final_iterations, o.incremental = fp64_final_iterations, int(incremental)
    o.mixed_switch_density, o.fp64_final_converge = mixed_switch_density, int(fp64_final_converge)
    o.mixed_switch_diis = mixed_switch_diis
    o.trace = int(trace)
    o.stop_at_precision_test = int(stop_at_precision_test)
    o.max_iterations = int(max_iterations)
    o.mp2 = int(mp2)
    o.concurrent_classes = int(concurrent_classes)  # 0, 1 streams, 2 streams + graphs
    for d in range(3):
        o.electric_field[d] = float(electric_field[d])
    return o


def result_dict(r: hfd_scf_result) -> dict:
    return {"energy": r.energy, "homo": r.homo, "converged": bool(r.converged), "iterations": r.iterations,
            "nbf": r.nbf, "fock_builds": r.fock_builds, "fock_ms_total": r.fock_ms_total,
            "fp32_quartets": r.fp32_quartets, "fp64_quartets": r.fp64_quartets, "mixed_steps": r.mixed_steps,
            "seconds_fock": r.seconds_fock, "seconds_eigen": r.seconds_eigen, "seconds_diis": r.seconds_diis,
            "seconds_total": r.seconds_total, "seconds_init": r.seconds_init, "mp2_energy": r.mp2_energy,
            "dipole": [r.dipole[0], r.dipole[1], r.dipole[2]]}


def torch_allreduce(group=None):
    """An hfd_allreduce_fn that sums G over a torch.distributed group: the
    device buffer is copied into a torch tensor (through host memory for the
    gloo backend), all-reduced and copied back."""
    import torch
    import torch.distributed as dist

    def fn(dG, count, stream, user):
        t = torch.empty(int(count), dtype=torch.float64, device="cuda")
        E._check(_lib().hfg_copy_device(ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(dG), int(count) * 8,
                                        ctypes.c_void_p(stream)))
        if dist.get_backend(group) == "gloo":
            h = t.cpu()
            dist.all_reduce(h, group=group)
            t.copy_(h)
        else:
            dist.all_reduce(t, group=group)
        torch.cuda.synchronize()
        E._check(_lib().hfg_copy_device(ctypes.c_void_p(dG), ctypes.c_void_p(t.data_ptr()), int(count) * 8,
                                        ctypes.c_void_p(stream)))
    return fn


def run_scf(Z, xyz, basis: str, unrestricted=False, want_density=True, shard=None, allreduce=None, **kw):
    """RestrictedHartreeFock / UnrestrictedHartreeFock Init + Calculate
    (scf_opts keywords).

    mixed_cutoff > 0 selects the precision form of the Fock builds (FP32
    below the cutoff, incremental from the density difference, all-FP64
    final iterations); incremental=True alone gives FP64 incremental builds.
    shard=(rank, count) with allreduce(dG_ptr, count, stream, user) (e.g.
    torch_allreduce()) runs the sharded SCF: every build evaluates this
    rank's shard and the callback sums G over the ranks."""
    L = _lib()
    o = scf_opts(unrestricted=unrestricted, **kw)
    cb = None
    if shard is not None and shard[1] > 1:
        cb = ALLREDUCE_FN(allreduce)
        o.shard_rank, o.shard_count = int(shard[0]), int(shard[1])
        o.allreduce = ctypes.cast(cb, ctypes.c_void_p)
    z = np.ascontiguousarray(Z, dtype=np.int32)
    x = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
    nbf_guess = 40 * len(z) + 64
    cap = (2 if unrestricted else 1) * nbf_guess * nbf_guess
    dens = np.zeros(cap) if want_density else None
    r = hfd_scf_result()
    st = L.hfd_scf(basis_path(basis).encode(), len(z), z.ctypes.data_as(ctypes.c_void_p),
                   x.ctypes.data_as(ctypes.c_void_p), ctypes.byref(o), ctypes.byref(r),
                   dens.ctypes.data_as(ctypes.c_void_p) if dens is not None else None, cap if dens is not None else 0)
    if st != 0:
        raise E.HfgError(st, L.hfd_last_error().decode())
    out = result_dict(r)
    if dens is not None:
        n = r.nbf
        if unrestricted:
            out["density_alpha"] = dens[:n * n].reshape(n, n).copy()
            out["density_beta"] = dens[n * n:2 * n * n].reshape(n, n).copy()
        else:
            out["density"] = dens[:n * n].reshape(n, n).copy()
    return out


def load_xyz(path: str, basis: str, cap: int = 4096):
    """Systems::Molecule::LoadXYZ through the driver: (Z, xyz, nbf), or None
    when LoadXYZ returns false."""
    L = _lib()
    z = np.zeros(cap, dtype=np.int32)
    x = np.zeros(3 * cap)
    n, nbf = ctypes.c_int32(), ctypes.c_int32()
    st = L.hfd_load_xyz(path.encode(), basis_path(basis).encode(), cap, ctypes.byref(n),
                        z.ctypes.data_as(ctypes.c_void_p), x.ctypes.data_as(ctypes.c_void_p), ctypes.byref(nbf))
    if st != 0:
        return None
    return z[:n.value].tolist(), x[:3 * n.value].reshape(-1, 3), nbf.value


def one_electron(Z, xyz, basis: str):
    """Overlap and core Hamiltonian from the host one-electron code."""
    L = _lib()
    z = np.ascontiguousarray(Z, dtype=np.int32)
    x = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
    cap = (40 * len(z) + 64) ** 2
    S, h = np.zeros(cap), np.zeros(cap)
    n = ctypes.c_int32()
    st = L.hfd_one_electron(basis_path(basis).encode(), len(z), z.ctypes.data_as(ctypes.c_void_p),
                            x.ctypes.data_as(ctypes.c_void_p), S.ctypes.data_as(ctypes.c_void_p),
                            h.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(n))
    if st != 0:
        raise E.HfgError(st, L.hfd_last_error().decode())
    k = n.value
    return S[:k * k].reshape(k, k).copy(), h[:k * k].reshape(k, k).copy()


def pulay_solve(B: np.ndarray) -> np.ndarray:
    """Solutions c of B c = (0, ..., 0, 1) for a stack of bordered Pulay
    matrices [batch, m+1, m+1] (hfd_pulay_solve: the SCF's own QR)."""
    L = _lib()
    B = np.ascontiguousarray(B, dtype=np.float64)
    b, m1, _ = B.shape
    c = np.empty((b, m1))
    st = L.hfd_pulay_solve(B.ctypes.data_as(ctypes.c_void_p), m1, b, c.ctypes.data_as(ctypes.c_void_p))
    if st != 0:
        raise E.HfgError(st, "hfd_pulay_solve")
    return c


def release_thread():
    """Free the calling thread's library handles (hfd_release_thread); worker
    threads call it before they exit."""
    _lib().hfd_release_thread()
