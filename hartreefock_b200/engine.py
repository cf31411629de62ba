"""ctypes binding of the engine's C ABI (include/hfgpu.h).

The library is built in-tree (hartreefock_b200/libhfgpu.so, see build.py).
There is no CPU fallback: loading fails loudly when the library or a CUDA
device is missing.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .basis_io import ShellTable, shell_table

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libhfgpu.so")

HFG_OK = 0
STATUS = {0: "HFG_OK", 1: "HFG_INVALID_ARG", 2: "HFG_UNSUPPORTED_L", 3: "HFG_OOM_BUDGET", 4: "HFG_DEVICE_ERROR",
          5: "HFG_TIMEOUT", 6: "HFG_CANCELLED", 7: "HFG_NO_DEVICE"}
ERI_REFERENCE, ERI_EXACT = 0, 1

# every symbol include/hfgpu.h declares
EXPORTED = ["hfg_default_opts", "hfg_last_error", "hfg_device_count", "hfg_ctx_create", "hfg_ctx_destroy",
            "hfg_ctx_nbf", "hfg_packed_size", "hfg_eri_packed", "hfg_eri_packed_device", "hfg_eri_quartet",
            "hfg_fock_rhf", "hfg_fock_uhf", "hfg_fock_rhf_device", "hfg_fock_uhf_device", "hfg_schwarz",
            "hfg_ctx_stats", "hfg_set_profiling", "hfg_class_profile", "hfg_measure_fp64_peak", "hfg_measure_fp32_peak",
            "hfg_fock_rhf_noalloc", "hfg_fock_reset", "hfg_set_mixed_cutoff", "hfg_set_incremental",
            "hfg_set_shard", "hfg_copy_device", "hfg_batch_create", "hfg_batch_size", "hfg_batch_layout", "hfg_fock_rhf_batch_device",
            "hfg_fock_uhf_batch_device", "hfg_fock_rhf_batch_async", "hfg_fock_uhf_batch_async", "hfg_eigh_batched", "hfg_one_electron",
            "hfg_pulay_solve_device", "hfg_mo_eri_ovov", "hfg_mp2_rhf", "hfg_mp2_uhf", "hfg_mo_eri_full", "hfg_spin_orbital_eri", "hfg_autotune", "hfg_autotune_tasks", "hfg_set_prim_target", "hfg_set_graphs",
            "hfg_set_class_path", "hfg_autotune_paths", "hfg_shard_range",
            "hfg_set_streams",
            "hfg_release_thread"]


class HfgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class hfg_shells(ctypes.Structure):
    _fields_ = [("nshells", ctypes.c_int32), ("center", ctypes.c_void_p), ("L", ctypes.c_void_p),
                ("nprim", ctypes.c_void_p), ("prim_offset", ctypes.c_void_p), ("ao_offset", ctypes.c_void_p),
                ("exponent", ctypes.c_void_p), ("coefficient", ctypes.c_void_p), ("nbf", ctypes.c_int32)]


class hfg_opts(ctypes.Structure):
    _fields_ = [("schwarz_threshold", ctypes.c_double), ("mixed_cutoff", ctypes.c_double),
                ("eri_convention", ctypes.c_int32), ("device", ctypes.c_int32),
                ("density_screening", ctypes.c_int32), ("incremental", ctypes.c_int32),
                ("density_threshold", ctypes.c_double), ("cuda_graphs", ctypes.c_int32), ("concurrent_classes", ctypes.c_int32)]


class hfg_stats(ctypes.Structure):
    _fields_ = [("shell_pairs", ctypes.c_int64), ("shell_quartets", ctypes.c_int64),
                ("function_quartets", ctypes.c_int64), ("primitive_quartets", ctypes.c_int64),
                ("fp32_shell_quartets", ctypes.c_int64), ("fp64_shell_quartets", ctypes.c_int64),
                ("flops", ctypes.c_double),
                ("last_build_ms", ctypes.c_double), ("kernel_launches", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class hfg_class_time(ctypes.Structure):
    _fields_ = [("la", ctypes.c_int32), ("lb", ctypes.c_int32), ("lc", ctypes.c_int32), ("ld", ctypes.c_int32),
                ("shell_quartets", ctypes.c_int64), ("function_quartets", ctypes.c_int64),
                ("primitive_quartets", ctypes.c_int64), ("flops", ctypes.c_double), ("ms", ctypes.c_double),
                ("tasks", ctypes.c_int64), ("lane_occupancy", ctypes.c_double), ("warp_kernel", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


_lib = None


def library(path: str = LIB_PATH):
    """Load libhfgpu.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m hartreefock_b200.build`")
    L = ctypes.CDLL(path)
    vp, i32, i64, dp = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p
    L.hfg_default_opts.argtypes = [ctypes.POINTER(hfg_opts)]
    L.hfg_default_opts.restype = None
    L.hfg_last_error.restype = ctypes.c_char_p
    L.hfg_device_count.restype = i32
    L.hfg_ctx_create.argtypes = [ctypes.POINTER(hfg_shells), ctypes.POINTER(hfg_opts), ctypes.POINTER(vp)]
    L.hfg_ctx_destroy.argtypes = [vp]
    L.hfg_ctx_destroy.restype = None
    L.hfg_ctx_nbf.argtypes = [vp]
    L.hfg_ctx_nbf.restype = i32
    L.hfg_packed_size.argtypes = [i32]
    L.hfg_packed_size.restype = i64
    L.hfg_eri_packed.argtypes = [vp, dp, i64]
    L.hfg_eri_packed_device.argtypes = [vp, dp, i64, vp]
    L.hfg_eri_quartet.argtypes = [vp, i32, i32, i32, i32, ctypes.POINTER(ctypes.c_double)]
    L.hfg_fock_rhf.argtypes = [vp, dp, dp]
    L.hfg_fock_uhf.argtypes = [vp, dp, dp, dp, dp]
    L.hfg_fock_rhf_device.argtypes = [vp, dp, dp, vp]
    L.hfg_fock_uhf_device.argtypes = [vp, dp, dp, dp, dp, vp]
    L.hfg_schwarz.argtypes = [vp, dp, i64]
    L.hfg_ctx_stats.argtypes = [vp, ctypes.POINTER(hfg_stats)]
    L.hfg_fock_rhf_noalloc.argtypes = [vp, dp, dp, vp]
    L.hfg_batch_create.argtypes = [ctypes.POINTER(hfg_shells), i32, ctypes.POINTER(hfg_opts), ctypes.POINTER(vp)]
    L.hfg_batch_size.argtypes = [vp]
    L.hfg_batch_size.restype = i32
    L.hfg_batch_layout.argtypes = [vp, vp, vp, ctypes.POINTER(i64)]
    L.hfg_fock_rhf_batch_device.argtypes = [vp, dp, dp, vp, vp]
    L.hfg_fock_uhf_batch_device.argtypes = [vp, dp, dp, dp, dp, vp, vp]
    L.hfg_fock_rhf_batch_async.argtypes = [vp, dp, dp, vp, vp]
    L.hfg_fock_uhf_batch_async.argtypes = [vp, dp, dp, dp, dp, vp, vp]
    for name in ("hfg_batch_create", "hfg_batch_layout", "hfg_fock_rhf_batch_device", "hfg_fock_uhf_batch_device",
                 "hfg_fock_rhf_batch_async", "hfg_fock_uhf_batch_async"):
        getattr(L, name).restype = ctypes.c_int
    L.hfg_fock_rhf_noalloc.restype = ctypes.c_int
    L.hfg_set_profiling.argtypes = [vp, i32]
    L.hfg_class_profile.argtypes = [vp, ctypes.POINTER(hfg_class_time), i32, ctypes.POINTER(i32)]
    L.hfg_measure_fp64_peak.argtypes = [i32, ctypes.POINTER(ctypes.c_double)]
    L.hfg_measure_fp32_peak.argtypes = [i32, ctypes.POINTER(ctypes.c_double)]
    L.hfg_fock_reset.argtypes = [vp]
    L.hfg_set_mixed_cutoff.argtypes = [vp, ctypes.c_double]
    L.hfg_set_incremental.argtypes = [vp, i32]
    L.hfg_set_shard.argtypes = [vp, i32, i32]
    L.hfg_shard_range.argtypes = [dp, ctypes.c_int64, i32, i32, ctypes.POINTER(ctypes.c_int64),
                                  ctypes.POINTER(ctypes.c_int64)]
    L.hfg_shard_range.restype = ctypes.c_int
    L.hfg_eigh_batched.argtypes = [dp, dp, dp, i32, i32, i32, vp]
    L.hfg_eigh_batched.restype = ctypes.c_int
    L.hfg_pulay_solve_device.argtypes = [dp, i32, i32, dp, vp]
    L.hfg_pulay_solve_device.restype = ctypes.c_int
    L.hfg_one_electron.argtypes = [ctypes.POINTER(hfg_shells), dp, dp, i32, i32, dp, dp, dp]
    L.hfg_one_electron.restype = ctypes.c_int
    L.hfg_mo_eri_ovov.argtypes = [vp, dp, i32, i32, i32, i32, dp, vp]
    L.hfg_mo_eri_ovov.restype = ctypes.c_int
    L.hfg_mp2_rhf.argtypes = [vp, dp, dp, i32, ctypes.POINTER(ctypes.c_double)]
    L.hfg_mp2_rhf.restype = ctypes.c_int
    L.hfg_mp2_uhf.argtypes = [vp, dp, dp, i32, dp, dp, i32, ctypes.POINTER(ctypes.c_double)]
    L.hfg_mp2_uhf.restype = ctypes.c_int
    L.hfg_spin_orbital_eri.argtypes = [vp, dp, dp, ctypes.c_int64]
    L.hfg_spin_orbital_eri.restype = ctypes.c_int
    L.hfg_autotune.argtypes = [vp, dp, vp, i32, ctypes.POINTER(i32), vp]
    L.hfg_autotune.restype = ctypes.c_int
    L.hfg_autotune_tasks.argtypes = [vp, dp, vp, i32, ctypes.POINTER(i32), vp]
    L.hfg_autotune_tasks.restype = ctypes.c_int
    L.hfg_set_prim_target.argtypes = [vp, i32]
    L.hfg_set_prim_target.restype = ctypes.c_int
    L.hfg_set_class_path.argtypes = [vp, i32, i32, i32, i32, i32]
    L.hfg_set_class_path.restype = ctypes.c_int
    L.hfg_autotune_paths.argtypes = [vp, dp, vp, i32, ctypes.POINTER(i32), vp]
    L.hfg_autotune_paths.restype = ctypes.c_int
    L.hfg_set_graphs.argtypes = [vp, i32]
    L.hfg_set_graphs.restype = ctypes.c_int
    L.hfg_set_streams.argtypes = [vp, i32]
    L.hfg_set_streams.restype = ctypes.c_int
    for name in ("hfg_fock_reset", "hfg_set_mixed_cutoff", "hfg_set_incremental", "hfg_set_shard", "hfg_set_profiling", "hfg_class_profile", "hfg_measure_fp64_peak", "hfg_measure_fp32_peak", "hfg_ctx_create", "hfg_eri_packed", "hfg_eri_packed_device", "hfg_eri_quartet", "hfg_fock_rhf",
                 "hfg_fock_uhf", "hfg_fock_rhf_device", "hfg_fock_uhf_device", "hfg_schwarz", "hfg_ctx_stats"):
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def _torch_stream() -> int:
    """torch's current stream as a handle for the C ABI.  torch's default
    stream is the legacy default stream, whose handle 0 the ABI reads as "the
    context's own stream"; pass cudaStreamLegacy (1) instead, so that our
    kernels stay ordered with torch's."""
    import torch
    return torch.cuda.current_stream().cuda_stream or 1


def _check(st):
    if st != HFG_OK:
        raise HfgError(st, library().hfg_last_error().decode())


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def shard_range(cost_prefix, rank: int, count: int) -> tuple:
    """Task range (first, n) of shard `rank` of `count` for tasks with
    running cost `cost_prefix` (len = tasks + 1, starting at 0): the
    partition the sharded builds use (hfg_shard_range; host only)."""
    pre = np.ascontiguousarray(cost_prefix, dtype=np.float64)
    first, n = ctypes.c_int64(), ctypes.c_int64()
    _check(library().hfg_shard_range(_ptr(pre), len(pre) - 1, int(rank), int(count), ctypes.byref(first),
                                     ctypes.byref(n)))
    return first.value, n.value


def measure_fp64_peak(device: int = 0) -> float:
    v = ctypes.c_double()
    _check(library().hfg_measure_fp64_peak(device, ctypes.byref(v)))
    return v.value


def measure_fp32_peak(device: int = 0) -> float:
    v = ctypes.c_double()
    _check(library().hfg_measure_fp32_peak(device, ctypes.byref(v)))
    return v.value


def one_electron(Z, xyz, basis: str, device: int = 0):
    """(S, T, V) of a molecule from the device one-electron kernels
    (hfg_one_electron), row-major nbf x nbf float64 arrays."""
    t = shell_table(Z, xyz, basis)
    keep = [np.ascontiguousarray(x) for x in (t.center.ravel(), t.L, t.nprim, t.prim_offset, t.ao_offset,
                                              t.exponent, t.coefficient)]
    sh = hfg_shells(len(t.L), *[_ptr(x) for x in keep], t.nbf)
    x = np.ascontiguousarray(np.asarray(xyz, dtype=np.float64).reshape(-1, 3))
    z = np.ascontiguousarray(Z, dtype=np.int32)
    out = [np.zeros((t.nbf, t.nbf)) for _ in range(3)]
    _check(library().hfg_one_electron(ctypes.byref(sh), _ptr(x), _ptr(z), len(z), device, *[_ptr(o) for o in out]))
    return tuple(out)


def _autotune(handle, P) -> dict:
    import torch
    dP = torch.as_tensor(np.asarray(P) if not isinstance(P, torch.Tensor) else P, dtype=torch.float64)
    dP = dP.cuda().contiguous()
    rec = np.zeros(5 * 32, dtype=np.int32)
    n = ctypes.c_int32()
    _check(library().hfg_autotune(handle, ctypes.c_void_p(dP.data_ptr()), _ptr(rec), len(rec), ctypes.byref(n),
                                  ctypes.c_void_p(_torch_stream())))
    return {("all" if r[0] < 0 else f"({r[0]}{r[1]}|{r[2]}{r[3]})"): int(r[4]) for r in rec[:5 * n.value].reshape(-1, 5)}


def eigh_batched(A, method: int = 0):
    """Eigenvalues (ascending) and eigenvectors of a stack of symmetric
    matrices, a contiguous float64 CUDA tensor [batch, n, n], by one batched
    cuSOLVER call (hfg_eigh_batched) on torch's current stream.  Returns
    (w [batch, n], U [batch, n, n]) with A = U diag(w) U^T, as
    torch.linalg.eigh does."""
    import torch
    assert A.is_cuda and A.dtype == torch.float64 and A.dim() == 3 and A.shape[1] == A.shape[2]
    A = A.contiguous()
    b, n, _ = A.shape
    X = torch.empty_like(A)
    w = torch.empty(b, n, dtype=torch.float64, device=A.device)
    _check(library().hfg_eigh_batched(ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(X.data_ptr()),
                                      ctypes.c_void_p(w.data_ptr()), n, b, method,
                                      ctypes.c_void_p(_torch_stream())))
    return w, X.transpose(1, 2)


def pulay_solve_device(B, out=None):
    """DIIS solutions of a [batch, m1, m1] float64 CUDA tensor on torch's
    current stream (hfg_pulay_solve_device); returns [batch, m1]."""
    import torch
    B = B.contiguous()
    if out is None:
        out = torch.empty(B.shape[0], B.shape[1], dtype=torch.float64, device=B.device)
    _check(library().hfg_pulay_solve_device(B.data_ptr(), B.shape[1], B.shape[0], out.data_ptr(), _torch_stream()))
    return out


def default_opts() -> hfg_opts:
    o = hfg_opts()
    library().hfg_default_opts(ctypes.byref(o))
    return o


class Engine:
    """One molecule's ERI / Fock-build context on one GPU."""

    def __init__(self, Z, xyz, basis: str, schwarz_threshold: float = 1e-12, eri_convention: int = ERI_REFERENCE,
                 device: int = 0, mixed_cutoff: float = 0.0, density_screening: bool = False,
                 incremental: bool = False, density_threshold: float = 0.0):
        self.table: ShellTable = shell_table(Z, xyz, basis)
        self.Z, self.xyz, self.basis = list(Z), np.asarray(xyz, dtype=np.float64).reshape(-1, 3), basis
        t = self.table
        self._keep = [np.ascontiguousarray(x) for x in (t.center.ravel(), t.L, t.nprim, t.prim_offset, t.ao_offset,
                                                         t.exponent, t.coefficient)]
        sh = hfg_shells(len(t.L), *[_ptr(x) for x in self._keep], t.nbf)
        o = default_opts()
        o.schwarz_threshold = schwarz_threshold
        o.eri_convention = eri_convention
        o.device = device
        o.mixed_cutoff = mixed_cutoff
        o.density_screening = int(density_screening)
        o.incremental = int(incremental)
        o.density_threshold = density_threshold
        self.opts = o
        h = ctypes.c_void_p()
        _check(library().hfg_ctx_create(ctypes.byref(sh), ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self.nbf = t.nbf

    def close(self):
        if getattr(self, "_h", None):
            library().hfg_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def packed_size(self) -> int:
        return library().hfg_packed_size(self.nbf)

    def eri_packed(self) -> np.ndarray:
        out = np.empty(self.packed_size(), dtype=np.float64)
        _check(library().hfg_eri_packed(self._h, _ptr(out), out.size))
        return out

    def eri_packed_device(self, out_ptr: int, count: int, stream: int = 0):
        _check(library().hfg_eri_packed_device(self._h, ctypes.c_void_p(out_ptr), count, ctypes.c_void_p(stream)))

    def eri(self, i, j, k, l) -> float:
        v = ctypes.c_double()
        _check(library().hfg_eri_quartet(self._h, i, j, k, l, ctypes.byref(v)))
        return v.value

    def fock_rhf(self, P: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        P = np.ascontiguousarray(P, dtype=np.float64)
        G = np.empty_like(P) if out is None else out
        assert G.flags.c_contiguous and G.dtype == np.float64 and G.shape == P.shape
        _check(library().hfg_fock_rhf(self._h, _ptr(P), _ptr(G)))
        return G

    def fock_uhf(self, Pa: np.ndarray, Pb: np.ndarray):
        Pa = np.ascontiguousarray(Pa, dtype=np.float64)
        Pb = np.ascontiguousarray(Pb, dtype=np.float64)
        Ga, Gb = np.empty_like(Pa), np.empty_like(Pb)
        _check(library().hfg_fock_uhf(self._h, _ptr(Pa), _ptr(Pb), _ptr(Ga), _ptr(Gb)))
        return Ga, Gb

    def fock_rhf_device(self, P_ptr: int, G_ptr: int, stream: int = 0):
        _check(library().hfg_fock_rhf_device(self._h, ctypes.c_void_p(P_ptr), ctypes.c_void_p(G_ptr),
                                             ctypes.c_void_p(stream)))

    def fock_rhf_tensor(self, P, G):
        """Direct build between torch CUDA tensors (contiguous n x n float64),
        on torch's current stream."""
        import torch
        assert P.is_cuda and G.is_cuda and P.dtype == torch.float64 and P.is_contiguous() and G.is_contiguous()
        self.fock_rhf_device(P.data_ptr(), G.data_ptr(), _torch_stream())

    def fock_uhf_tensor(self, Pa, Pb, Ga, Gb):
        import torch
        for t in (Pa, Pb, Ga, Gb):
            assert t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
        self.fock_uhf_device(Pa.data_ptr(), Pb.data_ptr(), Ga.data_ptr(), Gb.data_ptr(),
                             _torch_stream())

    def fock_rhf_noalloc(self, P_ptr: int, G_ptr: int, stream: int = 0):
        """Allocation-free direct RHF build (fixed 1024-function scratch)."""
        _check(library().hfg_fock_rhf_noalloc(self._h, ctypes.c_void_p(P_ptr), ctypes.c_void_p(G_ptr),
                                              ctypes.c_void_p(stream)))

    def fock_uhf_device(self, Pa_ptr, Pb_ptr, Ga_ptr, Gb_ptr, stream: int = 0):
        _check(library().hfg_fock_uhf_device(self._h, ctypes.c_void_p(Pa_ptr), ctypes.c_void_p(Pb_ptr),
                                             ctypes.c_void_p(Ga_ptr), ctypes.c_void_p(Gb_ptr),
                                             ctypes.c_void_p(stream)))

    def set_streams(self, on: bool = True):
        """Run a build's class kernels concurrently over the context's
        auxiliary streams (hfg_set_streams)."""
        _check(library().hfg_set_streams(self._h, int(on)))

    def set_graphs(self, on: bool = True):
        """Replay the plain direct build as a CUDA graph (hfg_set_graphs)."""
        _check(library().hfg_set_graphs(self._h, int(on)))

    def autotune(self, P) -> dict:
        """Pick each fused class's grid (blocks per SM) by timing it on the
        density P (numpy or torch CUDA tensor); returns {class: blocks/SM}."""
        return _autotune(self._h, P)

    def autotune_tasks(self, P) -> dict:
        """Pick each thread-per-quartet class's lane-group target (primitive
        quartets per lane; 0 = one lane per quartet) by timing it on the
        density P; returns {class: target}."""
        import torch
        dP = torch.as_tensor(np.asarray(P) if not isinstance(P, torch.Tensor) else P, dtype=torch.float64)
        dP = dP.cuda().contiguous()
        rec = np.zeros(5 * 32, dtype=np.int32)
        n = ctypes.c_int32()
        _check(library().hfg_autotune_tasks(self._h, ctypes.c_void_p(dP.data_ptr()), _ptr(rec), len(rec),
                                            ctypes.byref(n), ctypes.c_void_p(_torch_stream())))
        return {f"({r[0]}{r[1]}|{r[2]}{r[3]})": int(r[4]) for r in rec[:5 * n.value].reshape(-1, 5)}

    def set_prim_target(self, target: int):
        _check(library().hfg_set_prim_target(self._h, int(target)))

    def set_class_path(self, cls: str, warp: bool):
        """Kernel of a large class with two, e.g. cls="(22|22)": the
        warp-cooperative kernel (warp=True) or the split path."""
        la, lb, lc, ld = (int(ch) for ch in cls.strip("()").replace("|", ""))
        _check(library().hfg_set_class_path(self._h, la, lb, lc, ld, int(bool(warp))))

    def autotune_paths(self, P) -> dict:
        """Time both kernels of every large class with two on the density P
        and keep the faster; returns {class: "warp" | "split"}."""
        import torch
        dP = torch.as_tensor(np.asarray(P) if not isinstance(P, torch.Tensor) else P, dtype=torch.float64)
        dP = dP.cuda().contiguous()
        rec = np.zeros(5 * 32, dtype=np.int32)
        n = ctypes.c_int32()
        _check(library().hfg_autotune_paths(self._h, ctypes.c_void_p(dP.data_ptr()), _ptr(rec), len(rec),
                                            ctypes.byref(n), ctypes.c_void_p(_torch_stream())))
        return {f"({r[0]}{r[1]}|{r[2]}{r[3]})": ("warp" if r[4] else "split") for r in rec[:5 * n.value].reshape(-1, 5)}

    def mp2_rhf(self, C: np.ndarray, eps: np.ndarray, nocc: int) -> float:
        """RHF MP2 correlation energy (hfg_mp2_rhf) from MO coefficients C
        (nbf x nbf, AO rows, MO columns) and orbital energies."""
        C = np.ascontiguousarray(C, dtype=np.float64)
        eps = np.ascontiguousarray(eps, dtype=np.float64)
        out = ctypes.c_double()
        _check(library().hfg_mp2_rhf(self._h, _ptr(C), _ptr(eps), nocc, ctypes.byref(out)))
        return out.value

    def mp2_uhf(self, Cp, ep, nplus: int, Cm, em, nminus: int) -> float:
        """UHF MP2 energy as the reference computes it (hfg_mp2_uhf)."""
        out = ctypes.c_double()
        arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (Cp, ep, Cm, em)]
        _check(library().hfg_mp2_uhf(self._h, _ptr(arrs[0]), _ptr(arrs[1]), nplus, _ptr(arrs[2]), _ptr(arrs[3]),
                                     nminus, ctypes.byref(out)))
        return out.value

    def spin_orbital_eri(self, C: np.ndarray) -> np.ndarray:
        """The (2 nbf)^4 antisymmetrised spin-orbital tensor of MO coefficients C
        (SpinOrbitalsElectronElectronIntegralsRepository::Compute)."""
        m = 2 * self.nbf
        out = np.empty((m, m, m, m), dtype=np.float64)
        C = np.ascontiguousarray(C, dtype=np.float64)
        _check(library().hfg_spin_orbital_eri(self._h, _ptr(C), _ptr(out), out.size))
        return out

    def mo_eri_ovov_tensor(self, C, i0: int, ni: int, a0: int, na: int):
        """(ia|jb) block as a torch CUDA tensor [ni*na, ni*na] (hfg_mo_eri_ovov)."""
        import torch
        C = C.contiguous()
        X = torch.empty(ni * na, ni * na, dtype=torch.float64, device=C.device)
        _check(library().hfg_mo_eri_ovov(self._h, ctypes.c_void_p(C.data_ptr()), i0, ni, a0, na,
                                          ctypes.c_void_p(X.data_ptr()),
                                          ctypes.c_void_p(_torch_stream())))
        return X

    def fock_reset(self):
        """Drop the incremental history: the next build starts from the full density."""
        _check(library().hfg_fock_reset(self._h))

    def set_mixed_cutoff(self, cutoff: float):
        _check(library().hfg_set_mixed_cutoff(self._h, float(cutoff)))

    def set_incremental(self, on: bool):
        _check(library().hfg_set_incremental(self._h, int(on)))

    def set_shard(self, rank: int, count: int):
        """Direct builds return shard `rank` of `count`'s partial G (hfg_set_shard)."""
        _check(library().hfg_set_shard(self._h, int(rank), int(count)))

    def schwarz(self) -> np.ndarray:
        n = len(self.table.L)
        out = np.empty(n * (n + 1) // 2)
        _check(library().hfg_schwarz(self._h, _ptr(out), out.size))
        return out

    def set_profiling(self, on: bool = True):
        _check(library().hfg_set_profiling(self._h, int(on)))

    def class_profile(self) -> list:
        arr = (hfg_class_time * 64)()
        n = ctypes.c_int32()
        _check(library().hfg_class_profile(self._h, arr, 64, ctypes.byref(n)))
        return [{k: getattr(arr[i], k) for k, _ in hfg_class_time._fields_ if k != "reserved"} for i in range(n.value)]

    def stats(self) -> dict:
        s = hfg_stats()
        _check(library().hfg_ctx_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in hfg_stats._fields_ if k != "reserved"}


class BatchEngine:
    """Many independent molecules in one context (hfg_batch_create): every
    direct build is one launch per quartet class over all molecules' tasks.
    Matrices are flat float64 CUDA tensors in the batch layout (molecule m's
    nbf[m] x nbf[m] block at offset[m])."""

    def __init__(self, molecules, schwarz_threshold: float = 1e-12, eri_convention: int = ERI_REFERENCE,
                 device: int = 0):
        """molecules: sequence of (Z, xyz_bohr, basis)."""
        self.tables = [shell_table(Z, xyz, basis) for Z, xyz, basis in molecules]
        self._keep = []
        arr = (hfg_shells * len(self.tables))()
        for i, t in enumerate(self.tables):
            keep = [np.ascontiguousarray(x) for x in (t.center.ravel(), t.L, t.nprim, t.prim_offset, t.ao_offset,
                                                      t.exponent, t.coefficient)]
            self._keep.append(keep)
            arr[i] = hfg_shells(len(t.L), *[_ptr(x) for x in keep], t.nbf)
        o = default_opts()
        o.schwarz_threshold = schwarz_threshold
        o.eri_convention = eri_convention
        o.device = device
        h = ctypes.c_void_p()
        _check(library().hfg_batch_create(arr, len(self.tables), ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self.nmol = len(self.tables)
        self.nbf = np.zeros(self.nmol, dtype=np.int32)
        self.offset = np.zeros(self.nmol, dtype=np.int64)
        total = ctypes.c_int64()
        _check(library().hfg_batch_layout(self._h, _ptr(self.nbf), _ptr(self.offset), ctypes.byref(total)))
        self.total = total.value

    def close(self):
        if getattr(self, "_h", None):
            library().hfg_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _active(self, active):
        if active is None:
            return None, None
        a = np.ascontiguousarray(np.asarray(active, dtype=np.uint8))
        assert a.size == self.nmol
        return a, _ptr(a)

    def fock_rhf(self, P, G, active=None):
        """G blocks of the active molecules from the P blocks (flat CUDA
        float64 tensors of `total` elements), on torch's current stream."""
        import torch
        keep, ap = self._active(active)
        _check(library().hfg_fock_rhf_batch_device(self._h, ctypes.c_void_p(P.data_ptr()),
                                                   ctypes.c_void_p(G.data_ptr()), ap,
                                                   ctypes.c_void_p(_torch_stream())))
        return G

    def fock_rhf_async(self, P, G, active_dev):
        """fock_rhf with the active mask a uint8 CUDA tensor (nmol): no host
        synchronisation, capturable in a CUDA graph after a first call."""
        _check(library().hfg_fock_rhf_batch_async(self._h, ctypes.c_void_p(P.data_ptr()),
                                                  ctypes.c_void_p(G.data_ptr()),
                                                  ctypes.c_void_p(active_dev.data_ptr()),
                                                  ctypes.c_void_p(_torch_stream())))
        return G

    def fock_uhf_async(self, Pa, Pb, Ga, Gb, active_dev):
        _check(library().hfg_fock_uhf_batch_async(self._h, ctypes.c_void_p(Pa.data_ptr()),
                                                  ctypes.c_void_p(Pb.data_ptr()), ctypes.c_void_p(Ga.data_ptr()),
                                                  ctypes.c_void_p(Gb.data_ptr()),
                                                  ctypes.c_void_p(active_dev.data_ptr()),
                                                  ctypes.c_void_p(_torch_stream())))

    def fock_uhf(self, Pa, Pb, Ga, Gb, active=None):
        import torch
        keep, ap = self._active(active)
        _check(library().hfg_fock_uhf_batch_device(self._h, ctypes.c_void_p(Pa.data_ptr()),
                                                   ctypes.c_void_p(Pb.data_ptr()), ctypes.c_void_p(Ga.data_ptr()),
                                                   ctypes.c_void_p(Gb.data_ptr()), ap,
                                                   ctypes.c_void_p(_torch_stream())))
        return Ga, Gb

    def set_streams(self, on: bool = True):
        """Run a build's class kernels concurrently over the context's
        auxiliary streams (hfg_set_streams)."""
        _check(library().hfg_set_streams(self._h, int(on)))

    def autotune(self, P) -> dict:
        """Grid autotuner over the batch (P: flat density, batch layout)."""
        return _autotune(self._h, P)

    def stats(self) -> dict:
        s = hfg_stats()
        _check(library().hfg_ctx_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in hfg_stats._fields_ if k != "reserved"}
