"""Build the engine's shared library for sm_100a, in-tree.

    python -m hartreefock_b200.build          # or __graft_entry__.build()

1. gen_eri.py writes the per-class recursion code and launchers;
2. every .cu / .cpp under csrc/ compiles in parallel into _build/ (objects
   newer than their inputs are reused);
3. nvcc links hartreefock_b200/libhfgpu.so (static CUDA runtime + cuBLAS /
   cuSOLVER for the device SCF algebra).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libhfgpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "-I" + os.path.join(ROOT, "include")]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    gen = os.path.join(CSRC, "gen_eri.py")
    stamp = os.path.join(CSRC, "eri_gen.cuh")
    if _stale(stamp, [gen]):
        _run([sys.executable, gen, CSRC])
    kernel_headers = glob.glob(os.path.join(CSRC, "*.cuh"))
    all_headers = kernel_headers + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    units = sorted(glob.glob(os.path.join(CSRC, "*.cu"))) + sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
    jobs_list = []
    for src in units:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        if src.endswith(".cu"):
            cmd = [NVCC] + CUFLAGS + ["-Xptxas", "-v", "-c", src, "-o", obj]
        else:
            cmd = ["g++"] + CXXFLAGS + ["-c", src, "-o", obj]
        # the generated class kernels see only the kernel headers
        headers = kernel_headers if os.path.basename(src).startswith("eri_") else all_headers
        jobs_list.append((src, obj, cmd, _stale(obj, [src] + headers)))
    logs = []
    todo = [j for j in jobs_list if j[3]]
    if todo:
        with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            for out in ex.map(lambda j: _run(j[2]), todo):
                logs.append(out)
    objs = [j[1] for j in jobs_list]
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcublas", "-lcusolver"])
    log = "\n".join(logs)
    with open(os.path.join(BUILD, "ptxas.log"), "a") as fh:
        fh.write(log)
    if verbose:
        print(log)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
