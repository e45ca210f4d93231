"""Build recipe for libfdzb.so (sm_100a) and the CPU oracle.

``python -m`` is not usable on a package whose name starts with a digit, so run
it as ``python 4dzb_b200/build.py`` or call :func:`build` from Python.  The
library is built in-tree (``4dzb_b200/libfdzb.so``) so that it travels with a
snapshot of the repository.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfdzb.so")

SOURCES = ["fdzb_pipeline.cu", "fdzb_shade.cu", "fdzb_raster.cu", "fdzb_api.cpp", "fdzb_serve.cpp",
           "fdzb_light.cpp"]
HEADERS = ["fdzb_internal.h", "fdzb_engine.h", "fdzb_device.cuh", "fdzb_sort.cuh", "fdzb_occlusion.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # every parity-path float operation is an _rn intrinsic; --fmad=false also
    # keeps any remaining plain expression unfused
    "--fmad=false",
    "-Xptxas", "-v",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math,-O2",
    "-I", os.path.join(ROOT, "include"),
    "-shared", "-cudart", "static",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force: bool = False, verbose: bool = False, defines: tuple = (),
                  out: str | None = None) -> str:
    """Compile libfdzb.so; `defines` are extra -D macros (tuning switches of
    fdzb_occlusion.cuh) and `out` an alternative output path."""
    lib = out or LIB
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "fdzb.h"))
    if not force and not defines and not _stale(lib, deps):
        return lib
    tmp = lib + ".tmp"
    cmd = [_nvcc(), *NVCC_FLAGS, *[f"-D{d}" for d in defines], "-o", tmp,
           *[os.path.join(CSRC, f) for f in SOURCES]]
    env = dict(os.environ)
    # the host compiler must be the system g++ (an alternative gcc on PATH may
    # lack the runtime libraries)
    env.pop("CC", None)
    env.pop("CXX", None)
    res = subprocess.run(cmd, cwd=HERE, capture_output=True, text=True, env=env)
    if verbose or res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode})")
    os.replace(tmp, lib)
    if out is None:
        with open(os.path.join(HERE, "ptxas_info.txt"), "w") as fh:
            fh.write(res.stderr)
    return lib


def build_oracle(verbose: bool = False) -> None:
    env = dict(os.environ)
    env.pop("CC", None)
    res = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], capture_output=True,
                         text=True, env=env)
    if verbose or res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError("oracle build failed")


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True)
    build_oracle(verbose=True)
    print(LIB)
