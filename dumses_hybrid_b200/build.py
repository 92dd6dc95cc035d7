"""Build libdumses_gpu.so in-tree for sm_100a.

nvcc compiles each CUDA translation unit with
  -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo
plus --fmad=false for the FP64 path and the host code (no multiply-add
contraction: the FP64 path is bit-identical to the CPU reference arithmetic)
and --use_fast_math for the FP32 mixed path, and links them, with the host-side initial conditions,
into dumses_hybrid_b200/libdumses_gpu.so against the static CUDA runtime, and builds the
C++ driver dumses_hybrid_b200/dg_driver (the reference's main program over the C-ABI) against it.  A second
library, libdumses_gpu_chk.so, is the same with the step kernels compiled with
-DDG_CHECK_BOUNDS: every array access of the step kernels checked against the registered
device buffers (a debug stand-in for a memory sanitizer, used by the tests).
Everything is rebuilt, translation units in parallel, when a source or header is newer than
a library.

Usage: python -m dumses_hybrid_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libdumses_gpu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(INCLUDE), "-I", str(CSRC)]
# FP64 path and host code: no multiply-add contraction (bit-identical arithmetic);
# FP32 mixed path: fast FP32 math (contraction, approximate division and sqrt, FTZ)
EXACT = ["--fmad=false"]
FAST = ["--use_fast_math"]
CU_SOURCES = {"step_fp64.cu": EXACT, "step_fp32.cu": FAST, "dg_api.cu": EXACT, "dg_noalloc.cu": EXACT,
              "nn_flux.cu": FAST}
CXX_SOURCES = ["condinit.cpp"]
LIB_CHK = PKG / "libdumses_gpu_chk.so"
CHECKED_SOURCES = ("step_fp64.cu", "step_fp32.cu")  # compiled again with -DDG_CHECK_BOUNDS
# the reference's main program over the C-ABI (a C++ executable linked to LIB)
DRIVER_SOURCE = "dg_driver.cpp"
DRIVER = PKG / "dg_driver"


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    # the environment's CC/CXX may point at a wrapper; the system compiler is enough here
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("g++ not found")


def _newest_input() -> float:
    files = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h")) + [pathlib.Path(__file__)]
    return max(f.stat().st_mtime for f in files if f.is_file())


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if verbose and (res.stdout or res.stderr):
        print(res.stdout + res.stderr, flush=True)
    if res.returncode != 0:
        raise RuntimeError(f"command failed ({res.returncode}): {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> pathlib.Path:
    newest = _newest_input()
    if not force and all(f.exists() and f.stat().st_mtime >= newest for f in (LIB, LIB_CHK, DRIVER)):
        return LIB
    BUILD.mkdir(exist_ok=True)
    nvcc, cxx = _nvcc(), _cxx()
    jobs = {}  # object -> command
    for src, flags in CU_SOURCES.items():
        extra = ["-Xptxas", "-v"] if ptxas_info else []
        jobs[BUILD / (src + ".o")] = [nvcc, *NVCC_FLAGS, *flags, *extra, "-c", str(CSRC / src), "-o", str(BUILD / (src + ".o"))]
        if src in CHECKED_SOURCES:
            obj = BUILD / (src + ".chk.o")
            jobs[obj] = [nvcc, *NVCC_FLAGS, *flags, "-DDG_CHECK_BOUNDS", "-c", str(CSRC / src), "-o", str(obj)]
    for src in CXX_SOURCES:
        obj = BUILD / (src + ".o")
        jobs[obj] = [cxx, "-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-I", str(INCLUDE), "-c", str(CSRC / src),
                     "-o", str(obj)]
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(_run, cmd, verbose or ptxas_info) for cmd in jobs.values()]:
            f.result()
    plain = [BUILD / (src + ".o") for src in CU_SOURCES] + [BUILD / (src + ".o") for src in CXX_SOURCES]
    checked = [BUILD / (src + (".chk.o" if src in CHECKED_SOURCES else ".o")) for src in CU_SOURCES] + \
              [BUILD / (src + ".o") for src in CXX_SOURCES]
    for lib, objs in ((LIB, plain), (LIB_CHK, checked)):
        tmp = lib.with_suffix(".so.tmp")
        _run([nvcc, *ARCH, "-shared", "-cudart", "static", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(tmp)], verbose)
        tmp.replace(lib)
    tmp = DRIVER.with_suffix(".tmp")
    _run([cxx, "-O2", "-std=c++17", "-I", str(INCLUDE), str(CSRC / DRIVER_SOURCE), "-L", str(PKG), "-ldumses_gpu",
          "-Wl,-rpath,$ORIGIN", "-o", str(tmp)], verbose)
    tmp.replace(DRIVER)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
