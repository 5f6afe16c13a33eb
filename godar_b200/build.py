"""Builds the in-tree native libraries.

- ``libgodar_gpu.so``: the CUDA kernels and the C ABI (include/godar_gpu.h),
  compiled for sm_100a only.  Translation units whose FP64 results must be
  bit-reproducible are compiled with ``--fmad=false`` (no fused multiply-add)
  and their host code with ``-ffp-contract=off``; the mixed-precision step is
  compiled without contraction too (every instance of a kernel rounds alike)
  and with approximate FP32 division and square root.
- ``libgodar_gen.so``: the host-side synthetic field placement.

Run ``python -m godar_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgodar_gpu.so")
GEN_LIB = os.path.join(HERE, "libgodar_gen.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"),
          "-Xptxas", "-warn-spills"]
EXACT = ["--fmad=false", "-Xcompiler", "-ffp-contract=off"]

UNITS = {
    "build.cu": EXACT,
    "bonds_init.cu": EXACT,
    "step_fp64.cu": EXACT,
    # FP32 divisions and roots to 2 ulp and fast log/exp in the mixed step
    # (FP64 arithmetic there is unaffected); no contraction into fused
    # multiply-adds, so that every instance of a kernel (diagnostic or not,
    # walls or not) rounds the same expression the same way and a result
    # does not depend on which steps computed diagnostics
    "step_mixed.cu": ["--fmad=false", "-prec-div=false", "-prec-sqrt=false"],
    "outputs.cu": EXACT,
    "engine.cu": EXACT,
    "noalloc.cu": EXACT,
    "checkpoint.cu": EXACT,
    "posts.cu": EXACT,
    "place.cu": [],
}
HEADERS = ["common.cuh", "physics.cuh", "detmath.cuh", "step_kernel.cuh", "kernels.h"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(unit: str, flags, verbose: bool) -> str:
    src = os.path.join(CSRC, unit)
    obj = os.path.join(BUILD, unit + ".o")
    deps = [src] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "godar_gpu.h")]
    if _newer(obj, deps):
        cmd = [NVCC] + ARCH + COMMON + flags + ["-c", src, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {unit}:\n{r.stderr}")
        if verbose and r.stderr:
            sys.stderr.write(r.stderr)
    return obj


def build_gpu(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda kv: _compile(kv[0], kv[1], verbose), UNITS.items()))
    if _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB


def build_gen() -> str:
    src = os.path.join(CSRC, "gen.cpp")
    if _newer(GEN_LIB, [src]):
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", GEN_LIB, src])
    return GEN_LIB


def build_all(verbose: bool = False) -> None:
    build_gen()
    build_gpu(verbose)


if __name__ == "__main__":
    build_all(verbose="-v" in sys.argv)
    print(LIB)
