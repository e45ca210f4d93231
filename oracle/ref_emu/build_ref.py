#!/usr/bin/env python3
"""Build recipe of the reference harness: 4DZB's own soft-shadow sources,
compiled for the CPU into oracle/_ref/libref4dzb.so (test infrastructure).

Reads the reference where it lies (oracle/refpath.py: $FDZB_REFERENCE or its default)
and writes only into oracle/_ref/.  Nothing from the reference is copied into
the repository:

* FS/api.cpp, FS/util/cudaBuffer.cpp, FS/util/channel.cpp and
  FS/util/layeredSurface.cpp compile unmodified with g++ against the shim
  headers in oracle/ref_emu/shim (vector helpers, GL scalar types, error
  macros) and the CUDA runtime calls of oracle/ref_emu/emu_runtime.cpp;
* the kernel files K/*.inl are streamed to g++ through a pipe, in the order of
  K/FourD.cu:230-257, between harness_pre.h and harness_post.h.  The stream
  rewrites three things only: the kernel-launch syntax `k<<<g, b[, s]>>>(args)`
  becomes `emu_launch(emu_cfg(g, b[, s]), [&]{ k(args); })`;
  `extern __shared__ T x[];` becomes a pointer to the launch's dynamic shared
  buffer; and the nested includes of Step2_3 (already streamed) and the
  backslash path in moveModel.inl are dropped / normalised.
  K/blockAABBReduce.inl is replaced by the sequential block reduction of
  oracle/ref_emu/emu.h (its warp-synchronous tail needs lock-step warps).
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT_DIR = os.path.join(ORACLE, "_ref")
LIB = os.path.join(OUT_DIR, "libref4dzb.so")
sys.path.insert(0, ORACLE)
from refpath import reference_root  # noqa: E402

REF = reference_root()
FS = os.path.join(REF, "4DZB", "FDZB_Soft_Shadow")
K = os.path.join(FS, "cuda")

INL_ORDER = ["FDprojection.inl", "binRaster.inl", "Step0_triangleSetup.inl",
             "Step2_1_samplerRectangleAABB.inl", "Step2_2_modelRectangleAABB.inl",
             "Step2_3_defineFDbuffer.inl", "Step3_bindSampleToBin.inl",
             "Step4_RasterizeTriangleToBin.inl", "Step5_1_prepareBin.inl", "Step5_2_shadowCal.inl",
             "Step5_2_calRef.inl", "Step5_2_shadowCalPerSample.inl", "moveModel.inl"]
HOST_SOURCES = [os.path.join(FS, "api.cpp"), os.path.join(FS, "util", "cudaBuffer.cpp"),
                os.path.join(FS, "util", "channel.cpp"), os.path.join(FS, "util", "layeredSurface.cpp")]

LAUNCH = re.compile(r"^(\s*)([A-Za-z_][A-Za-z0-9_]*(?:<[^<>]*>)?)\s*(?:/\*.*?\*/)?\s*<<\s*<\s*(.*?)\s*>>\s*>\s*\((.*)\)\s*;")
EXTERN_SHARED = re.compile(r"extern\s+__shared__\s+(volatile\s+)?(\w+)\s+(\w+)\s*\[\s*\]\s*;")


def _read(path: str) -> str:
    raw = open(path, "rb").read()
    try:
        return raw.decode("gbk")
    except UnicodeDecodeError:
        return raw.decode("latin-1")


def kernel_stream() -> str:
    parts = ['#include "harness_pre.h"\n']
    for name in INL_ORDER:
        text = _read(os.path.join(K, name))
        out = [f'# 1 "{name}"']
        for line in text.splitlines():
            s = line
            if name == "Step2_3_defineFDbuffer.inl" and s.strip().startswith('#include "Step2_'):
                s = "// (streamed above)"
            s = s.replace("#include <glm\\glm.hpp>", "#include <glm/glm.hpp>")
            m = LAUNCH.match(s)
            if m and not s.lstrip().startswith("//"):
                s = f"{m.group(1)}emu_launch(emu_cfg({m.group(3)}), [&] {{ {m.group(2)}({m.group(4)}); }});"
            s = EXTERN_SHARED.sub(lambda mm: f"{mm.group(2)} *{mm.group(3)} = emu_extern_shared<{mm.group(2)}>();", s)
            out.append(s)
        parts.append("\n".join(out) + "\n")
    parts.append('#include "harness_post.h"\n')
    return "".join(parts)


def build(verbose: bool = False) -> str:
    if not os.path.isdir(K):
        raise FileNotFoundError(f"reference sources not found under {REF}")
    os.makedirs(OUT_DIR, exist_ok=True)
    inc = ["-I", os.path.join(HERE, "shim"), "-I", HERE, "-I", K, "-I", os.path.join(FS, "util"), "-I", FS,
           "-I", os.path.join(REF, "4DZB"), "-I", "/usr/local/cuda/include"]
    flags = ["-std=c++17", "-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-w",
             "-DTHRUST_DEVICE_SYSTEM=THRUST_DEVICE_SYSTEM_CPP", "-DGLM_FORCE_PURE"]
    cxx = "g++"
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    objs = []

    def run(cmd, stdin=None):
        r = subprocess.run(cmd, input=stdin, capture_output=True, text=True, env=env)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr[-20000:])
        if r.returncode:
            raise RuntimeError(f"reference harness build failed: {' '.join(cmd[:3])} ...")

    obj = os.path.join(OUT_DIR, "kernels.o")
    run([cxx, *flags, *inc, "-x", "c++", "-c", "-", "-o", obj], stdin=kernel_stream())
    objs.append(obj)
    for src in HOST_SOURCES + [os.path.join(HERE, "emu_runtime.cpp")]:
        o = os.path.join(OUT_DIR, os.path.splitext(os.path.basename(src))[0] + ".o")
        run([cxx, *flags, *inc, "-include", os.path.join(HERE, "emu.h"), "-c", src, "-o", o])
        objs.append(o)
    run([cxx, "-shared", "-fopenmp", "-Wl,-Bsymbolic", "-o", LIB + ".tmp", *objs])
    os.replace(LIB + ".tmp", LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
