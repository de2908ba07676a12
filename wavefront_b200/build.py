"""Builds the sm_100a CUDA library libwavefront_gpu.so in-tree, and its
bounds-checked variant libwavefront_gpu_checked.so (-DWF_BOUNDS_CHECK: every
checked device access tests its index and latches an error flag instead of
touching memory out of range; the library loads it when WF_BOUNDS_CHECK=1).

nvcc compiles every source under csrc/ for `-gencode arch=compute_100a,
code=sm_100a` with FMA contraction off (the exact arithmetic path relies on
explicit __fmul_rn/__fadd_rn intrinsics as well), IEEE division/square root
and denormals kept (no --use_fast_math).  The CUDA runtime is linked
statically; the TMA descriptor encoder is reached through
cudaGetDriverEntryPoint, so no libcuda link is needed at build time.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(OUT_DIR, "libwavefront_gpu.so")
LIB_CHECKED = os.path.join(OUT_DIR, "libwavefront_gpu_checked.so")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
OBJ_DIR_CHECKED = os.path.join(OUT_DIR, "obj_checked")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--ftz=false",
                  "--prec-div=true", "--prec-sqrt=true",
                  "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-Xptxas", "-v"]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(src: str, checked: bool = False) -> tuple[str, str]:
    obj = os.path.join(OBJ_DIR_CHECKED if checked else OBJ_DIR, src + ".o")
    inp = os.path.join(CSRC, src)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "wavefront_gpu.h")]
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj, ""
    cmd = [NVCC] + NVFLAGS + (["-DWF_BOUNDS_CHECK"] if checked else []) + ["-c", inp, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-O2", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off", "-x", "c++",
               "-c", inp, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def _link(lib: str, objs: list) -> None:
    if not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")


def build(verbose: bool = False, checked: bool = True) -> str:
    """Compiles every source (and, with `checked`, the bounds-checked
    variant) in parallel; returns the path of the normal library."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR_CHECKED, exist_ok=True)
    srcs = _sources()
    jobs = [(f, False) for f in srcs] + ([(f, True) for f in srcs] if checked else [])
    with cf.ThreadPoolExecutor(max_workers=min(os.cpu_count() or 8, len(jobs))) as ex:
        results = list(ex.map(lambda j: _compile(*j), jobs))
    if verbose:
        for _, log in results:
            if log:
                print(log)
    _link(LIB, [o for (o, _), (_, c) in zip(results, jobs) if not c])
    if checked:
        _link(LIB_CHECKED, [o for (o, _), (_, c) in zip(results, jobs) if c])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
