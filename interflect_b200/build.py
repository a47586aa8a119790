"""Builds the native parts of interflect_b200 in-tree.

Outputs
  interflect_b200/lib/libinterflect_b200.so   CUDA kernels + C ABI (sm_100a)
  interflect_b200/lib/libinterflect_b200_checked.so
                                              the same with -DIFX_CHECKED: scene-array
                                              indices bounds-checked in every kernel and
                                              the transfer's structures validated, a
                                              failure reported as an error (tests only;
                                              selected by IFX_CHECKED=1)
  interflect_b200/bin/interflect              the `interflect render` CLI
  interflect_b200/bin/compare                 the image comparison tool (host only)

The kernels are compiled with --fmad=false and IEEE division and square
root so that every f32 expression rounds exactly as the reference's unfused
arithmetic does; host code that computes values the device reuses is built
with -ffp-contract=off for the same reason.

Usage: python -m interflect_b200.build [--force] [--verbose] [--checked]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libinterflect_b200.so")
LIB_CHECKED = os.path.join(HERE, "lib", "libinterflect_b200_checked.so")
CLI = os.path.join(HERE, "bin", "interflect")
COMPARE = os.path.join(HERE, "bin", "compare")

CU_SOURCES = ["k_surfels.cu", "k_transfer.cu", "k_solve.cu", "k_shade.cu", "k_batch.cu", "k_diff.cu", "k_multi.cu",
              "k_path.cu", "k_leafgrid.cu", "capi.cu", "noalloc.cu"]
CPP_SOURCES = ["scene_host.cpp"]
HEADERS = ["layout.h", "scene_host.h", "kernels.h", "device.cuh", "kcommon.cuh", "shade.cuh", "flop_model.h",
           "sqcmp.h", "pixorder.h", "libm_f32.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
              "-ftz=false", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2", "-I", os.path.join(ROOT, "include")]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Wextra",
             "-Wno-unused-parameter"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build interflect_b200")


def cuda_root() -> str:
    return os.path.dirname(os.path.dirname(os.path.realpath(nvcc())))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=not verbose, text=True)
    if r.returncode != 0:
        out = (r.stdout or "") + (r.stderr or "")
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(cmd)}\n{out}")


def build_library(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    obj_dir = OBJ + ("_checked" if checked else "")
    lib = LIB_CHECKED if checked else LIB
    extra = ["-DIFX_CHECKED"] if checked else []
    os.makedirs(obj_dir, exist_ok=True)
    os.makedirs(os.path.dirname(lib), exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "interflect.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(obj_dir, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs + [__file__]):
            _run([nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", s, "-o", o], verbose)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(obj_dir, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs + [__file__]):
            _run(["g++", *CXX_FLAGS, "-c", s, "-o", o], verbose)
    cudalib = os.path.join(cuda_root(), "lib64")
    if force or _stale(lib, objs):
        _run([nvcc(), *ARCH, "-shared", "-o", lib, *objs, "-L", cudalib, "-lcudart_static", "-lpthread", "-ldl",
              "-lrt"], verbose)
    return lib


def build(force: bool = False, verbose: bool = False, checked: bool = True) -> str:
    """Both library variants, the CLI and the compare tool."""
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "interflect.h")]
    build_library(force, verbose)
    if checked:
        build_library(force, verbose, checked=True)
    cli_src = os.path.join(CSRC, "cli.cpp")
    png_src = os.path.join(CSRC, "png.cpp")
    if os.path.exists(cli_src) and (force or _stale(CLI, [cli_src, png_src, LIB] + hdrs)):
        _run(["g++", *CXX_FLAGS, "-I", os.path.join(ROOT, "include"), cli_src, png_src, "-o", CLI,
              "-L", os.path.dirname(LIB), "-linterflect_b200", "-Wl,-rpath,$ORIGIN/../lib", "-lz"], verbose)
    cmp_src = os.path.join(CSRC, "compare.cpp")
    if os.path.exists(cmp_src) and (force or _stale(COMPARE, [cmp_src, png_src])):
        _run(["g++", *CXX_FLAGS, cmp_src, png_src, "-o", COMPARE, "-lz"], verbose)
    return LIB


if __name__ == "__main__":
    if "--checked" in sys.argv:
        print(build_library(force="--force" in sys.argv, verbose="--verbose" in sys.argv, checked=True))
    else:
        build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
        print(LIB)
