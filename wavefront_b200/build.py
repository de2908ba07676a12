"""Builds the sm_100a CUDA library libwavefront_gpu.so in-tree.

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
OBJ_DIR = os.path.join(OUT_DIR, "obj")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--ftz=false",
                  "--prec-div=true", "--prec-sqrt=true",
                  "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-Xptxas", "-v"]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(src: str) -> tuple[str, str]:
    obj = os.path.join(OBJ_DIR, src + ".o")
    inp = os.path.join(CSRC, src)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "wavefront_gpu.h")]
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj, ""
    cmd = [NVCC] + NVFLAGS + ["-c", inp, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-O2", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off", "-x", "c++",
               "-c", inp, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(_compile, srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
