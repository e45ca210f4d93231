#!/usr/bin/env python3
"""Build recipe of the reference GPU harness: 4DZB's own soft-shadow sources,
compiled for sm_100a into oracle/_ref/ (test infrastructure).

Six libraries, same sources, at three bin grids and two FMA settings:

* libref4dzb_gpu.so      -- --fmad=false: every float expression is the IEEE
  sequence of operations the source spells, so its shadows can be compared
  bit for bit with the oracle and with libfdzb.so;
* libref4dzb_gpu_fmad.so -- nvcc's default --fmad=true, as the reference's own
  project builds it: the timing build;
* libref4dzb_gpu_b32[_fmad].so, libref4dzb_gpu_b128[_fmad].so -- the same at
  32 x 32 and 128 x 128 light-plane bins.  The reference fixes its bin grid at
  compile time (FD_MAX_LP_GRID_SIZE_LOG2 = 4, FS/constants.h:13); these builds
  set it to 5 and 7, the grids of the small and HD workloads.  The edit is made
  on a temporary copy of FS/constants.h, next to a temporary verbatim copy of
  FS/api.cpp (its quoted #include "constants.h" then finds the edited copy;
  the kernel translation unit includes it first, and the header's include
  guard keeps the original out).  Both copies live under oracle/_ref/ while the
  build runs and are deleted after it.

Reads the reference where it lies (oracle/refpath.py: $FDZB_REFERENCE or its default)
and writes only into oracle/_ref/.  Nothing from the reference is copied into
the repository:

* FS/api.cpp (with nvcc, like the kernels: it shares glm types by value with
  them), FS/util/cudaBuffer.cpp, FS/util/channel.cpp and
  FS/util/layeredSurface.cpp (with g++) compile unmodified against the shim headers in
  oracle/ref_gpu/shim (then oracle/ref_emu/shim: GL scalar types, header-name
  case), with oracle/ref_gpu/refgpu.h force-included (the CUDA-GL interop calls
  renamed to the harness registry of gl_runtime.cpp; there is no graphics stack);
* the kernel files K/*.inl are concatenated, in the order of K/FourD.cu:230-257,
  between harness_pre.cuh and harness_post.cuh into a temporary .cu under
  oracle/_ref/ that is deleted after compiling.  The concatenation changes
  five things only, each checked to apply exactly once:
    - the nested includes of Step2_3 (already concatenated) are dropped and the
      backslash include path of moveModel.inl is normalised;
    - the unguarded per-frame pair dump `showBinTriPair(pairNum);`
      (K/Step4_RasterizeTriangleToBin.inl:218, a full device-to-host copy and
      an fprintf per pair into a Windows path) is removed from bindTriToBin;
    - writeTriBinPair_kernel (:161-204) counts each pair it writes beyond the
      count the counting kernel gave its triangle (REFGPU_Q2_MARK): the write
      kernel tests the unclamped AABB and the counting kernel the clamped one
      (:74-94 against :177-193), so a triangle can write into the next
      triangle's slots, and which write lands there depends on scheduling;
    - in the per-sample kernel's row loop
      (K/Step5_2_shadowCalPerSample.inl:204-222) a row index >= N is counted
      and skipped instead of indexing past the sample's N rows of shared
      memory (inverted partial row filters can keep bits >= N set);
    - after that kernel's shadow store (:231) the sample's final rows are
      copied to a harness buffer when one is set (REFGPU_MASK_DUMP), so that
      the reference's masks, not only its shadows, can be compared.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT_DIR = os.path.join(ORACLE, "_ref")
sys.path.insert(0, ORACLE)
from refpath import reference_root  # noqa: E402

# log2 of the bins per side of each build: 16 (the reference's own), 32, 128
BIN_LOG2S = (4, 5, 7)


def lib_name(bins_log2: int, fmad: bool) -> str:
    tag = "" if bins_log2 == 4 else f"_b{1 << bins_log2}"
    return os.path.join(OUT_DIR, f"libref4dzb_gpu{tag}{'_fmad' if fmad else ''}.so")


LIB_EXACT = lib_name(4, False)
LIB_FMAD = lib_name(4, True)
REF = reference_root()
FS = os.path.join(REF, "4DZB", "FDZB_Soft_Shadow")
K = os.path.join(FS, "cuda")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

INL_ORDER = ["FDprojection.inl", "blockAABBReduce.inl", "binRaster.inl", "Step0_triangleSetup.inl",
             "Step2_1_samplerRectangleAABB.inl", "Step2_2_modelRectangleAABB.inl",
             "Step2_3_defineFDbuffer.inl", "Step3_bindSampleToBin.inl",
             "Step4_RasterizeTriangleToBin.inl", "Step5_1_prepareBin.inl", "Step5_2_shadowCal.inl",
             "Step5_2_calRef.inl", "Step5_2_shadowCalPerSample.inl", "moveModel.inl"]
HOST_SOURCES = [os.path.join(FS, "api.cpp"), os.path.join(FS, "util", "cudaBuffer.cpp"),
                os.path.join(FS, "util", "channel.cpp"), os.path.join(FS, "util", "layeredSurface.cpp")]

# (file, exact stripped line, replacement) -- each must match exactly once
EDITS = [
    ("Step4_RasterizeTriangleToBin.inl", "showBinTriPair(pairNum);",
     "/* per-frame pair dump removed by the harness */"),
    ("Step4_RasterizeTriangleToBin.inl", "triPos[cnt] = tid;",
     "triPos[cnt] = tid; REFGPU_Q2_MARK(cnt, tid)"),
    ("Step5_2_shadowCalPerSample.inl", "mask[rowID*32] |= M0 & M1 & M2;",
     "REFGPU_ROW_GUARD(rowID, lightResHeight) mask[rowID*32] |= M0 & M1 & M2;"),
    ("Step5_2_shadowCalPerSample.inl", "shadowResult[sampleID] = (float)result / (float)lightResNum;",
     "shadowResult[sampleID] = (float)result / (float)lightResNum; "
     "REFGPU_MASK_DUMP(sampleID, mask, lightResHeight)"),
]


def _read(path: str) -> str:
    raw = open(path, "rb").read()
    try:
        return raw.decode("gbk")
    except UnicodeDecodeError:
        return raw.decode("latin-1")


def kernel_source() -> str:
    parts = ['#include "harness_pre.cuh"\n']
    hits = {i: 0 for i in range(len(EDITS))}
    for name in INL_ORDER:
        text = _read(os.path.join(K, name))
        out = [f'#line 1 "{name}"']
        for line in text.splitlines():
            s = line
            stripped = s.strip()
            if name == "Step2_3_defineFDbuffer.inl" and stripped.startswith('#include "Step2_'):
                s = "// (concatenated above)"
            s = s.replace("#include <glm\\glm.hpp>", "#include <glm/glm.hpp>")
            for i, (fname, old, new) in enumerate(EDITS):
                if name == fname and stripped == old:
                    s = s.replace(old, new)
                    hits[i] += 1
            out.append(s)
        parts.append("\n".join(out) + "\n")
    for i, n in hits.items():
        if n != 1:
            raise RuntimeError(f"harness edit {EDITS[i][:2]} matched {n} times (expected 1)")
    parts.append('#include "harness_post.cuh"\n')
    return "".join(parts)


CONST_LINE = "const int FD_MAX_LP_GRID_SIZE_LOG2 = 4;"


def constants_source(bins_log2: int) -> str:
    """FS/constants.h with the bin-grid constant set to bins_log2 (the line must
    appear exactly once)."""
    text = _read(os.path.join(FS, "constants.h"))
    out, hits = [], 0
    for line in text.splitlines():
        if line.strip().startswith(CONST_LINE):
            line = line.replace(CONST_LINE, f"const int FD_MAX_LP_GRID_SIZE_LOG2 = {bins_log2};")
            hits += 1
        out.append(line)
    if hits != 1:
        raise RuntimeError(f"bin-grid constant matched {hits} times in constants.h (expected 1)")
    return "\n".join(out) + "\n"


def build(verbose: bool = False) -> list[str]:
    if not os.path.isdir(K):
        raise FileNotFoundError(f"reference sources not found under {REF}")
    os.makedirs(OUT_DIR, exist_ok=True)
    inc = ["-I", os.path.join(HERE, "shim"), "-I", os.path.join(ORACLE, "ref_emu", "shim"), "-I", HERE,
           "-I", K, "-I", os.path.join(FS, "util"), "-I", FS, "-I", os.path.join(REF, "4DZB")]
    defs = ["-DGLM_FORCE_PURE"]
    host_flags = ["-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-w"]
    env = dict(os.environ)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True, env=env)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr[-20000:])
        if r.returncode:
            raise RuntimeError(f"reference GPU harness build failed: {' '.join(cmd[:4])} ...")

    force = ["-include", os.path.join(HERE, "refgpu.h")]
    work = os.path.join(OUT_DIR, "gpu_build")
    os.makedirs(work, exist_ok=True)
    kernels = kernel_source()
    api_text = _read(os.path.join(FS, "api.cpp"))
    libs, temps = [], []
    try:
        # host sources without the bin grid, once
        common = []
        for src in HOST_SOURCES[1:] + [os.path.join(HERE, "gl_runtime.cpp")]:
            o = os.path.join(work, "gpu_" + os.path.splitext(os.path.basename(src))[0] + ".o")
            run(["g++", "-std=c++17", *host_flags, *defs, *inc, "-I", "/usr/local/cuda/include", *force,
                 "-c", src, "-o", o])
            common.append(o)
            temps.append(o)

        def variant(bins_log2: int) -> list[tuple]:
            d = os.path.join(work, f"b{bins_log2}")
            os.makedirs(d, exist_ok=True)
            files = {"constants.h": constants_source(bins_log2), "api.cpp": api_text,
                     "ref_gpu_kernels.cu": '#include "constants.h"\n' + kernels}
            for name, text in files.items():
                with open(os.path.join(d, name), "w") as f:
                    f.write(text)
                temps.append(os.path.join(d, name))
            # FS/api.cpp takes AreaLightDes (three glm::vec3) by value from the
            # kernel translation unit; GLM declares its own copy constructor
            # under nvcc only, which changes how the struct is passed.  Both
            # sides are compiled by nvcc so that they agree.
            api_o = os.path.join(d, "gpu_api.o")
            run([NVCC, *ARCH, "-std=c++17", "-O3", "-x", "cu", "-Xcompiler", ",".join(host_flags), "-w",
                 "--expt-relaxed-constexpr", *defs, *inc, *force, "-c", os.path.join(d, "api.cpp"), "-o", api_o])
            temps.append(api_o)
            out = []
            for fmad in (False, True):
                o = os.path.join(d, f"gpu_kernels_fmad_{str(fmad).lower()}.o")
                run([NVCC, *ARCH, "-std=c++17", "-O3", "-lineinfo", f"--fmad={str(fmad).lower()}", "-Xcompiler",
                     ",".join(host_flags), "-w", "--expt-relaxed-constexpr", *defs, *inc, *force, "-c",
                     os.path.join(d, "ref_gpu_kernels.cu"), "-o", o])
                temps.append(o)
                out.append((bins_log2, fmad, o, api_o))
            return out

        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=len(BIN_LOG2S)) as pool:
            objs = [o for part in pool.map(variant, BIN_LOG2S) for o in part]
        for bins_log2, fmad, o, api_o in objs:
            lib = lib_name(bins_log2, fmad)
            run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", lib + ".tmp", o, api_o, *common,
                 "-Xlinker", "-Bsymbolic"])
            os.replace(lib + ".tmp", lib)
            libs.append(lib)
    finally:
        for t in temps:
            if os.path.exists(t):
                os.remove(t)
        for root, dirs, _ in os.walk(work, topdown=False):
            for dname in dirs:
                os.rmdir(os.path.join(root, dname))
        if os.path.isdir(work):
            os.rmdir(work)
    return libs


if __name__ == "__main__":
    for p in build(verbose="-v" in sys.argv):
        print(p)
