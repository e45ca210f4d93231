"""ctypes wrapper of oracle/_ref/libref4dzb_gpu*.so -- the reference's own
soft-shadow sources (4DZB/FDZB_Soft_Shadow) compiled for sm_100a by
oracle/ref_gpu/build_ref_gpu.py.  TEST INFRASTRUCTURE ONLY: it pins the product
against the reference running on the same GPU, and times the reference's GPU
frame.  The reference fixes its bin grid at compile time (FS/constants.h:13,
16 x 16); the harness is built at 16 x 16, 32 x 32 and 128 x 128 (BUILT_BINS),
each with --fmad=false (exact) and nvcc's default --fmad=true.

Every input is checked on the CPU first (preflight): the oracle, run with the
same bins and the reference's triangle order, must show that every sample key
stays inside the bin grid and that the triangle/bin pairs fit the reference's
fixed pair buffers (FS/constants.h:15, FS/api.cpp:132-138); the light must be
square with N <= 32 (the only form the per-sample kernel runs,
K/Step5_2_shadowCalPerSample.inl:249-254).  An input that fails is refused
before anything reaches the GPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BINS = 16                 # the reference's own compile-time grid
BUILT_BINS = (16, 32, 128)
# the reference's five stage drivers, in FDLaunch's order (FS/api.cpp:495-552)
STAGES = ["lightPlaneParamCal", "bindSampleToBin", "countTriBinPairNum", "bindTriToBin", "shadowCal_perSample"]
# FD_MAX_BT_PIAR_Num * 1.4 (FS/constants.h:15, FS/api.cpp:132-138)
PAIR_BUFFER = int(50 * 1024 * 1024 * 1.4)

f32p = ctypes.POINTER(ctypes.c_float)
i32p = ctypes.POINTER(ctypes.c_int32)


class RefGpuIn(ctypes.Structure):
    _fields_ = [("W", ctypes.c_int32), ("H", ctypes.c_int32), ("pos", f32p), ("nrm", f32p), ("vtx", f32p),
                ("V", ctypes.c_int32), ("vstride_bytes", ctypes.c_int32), ("idx", i32p), ("T", ctypes.c_int32),
                ("cull", ctypes.c_int32), ("esp", ctypes.c_float), ("rightRadius", ctypes.c_float),
                ("topRadius", ctypes.c_float), ("position", ctypes.c_float * 3), ("viewDir", ctypes.c_float * 3),
                ("upDir", ctypes.c_float * 3), ("lightRes", ctypes.c_int32), ("warmup", ctypes.c_int32),
                ("reps", ctypes.c_int32)]


class RefGpuOut(ctypes.Structure):
    _fields_ = [("shadow", f32p), ("launch_ms", f32p), ("fdlaunch_ms", f32p), ("num_bins", ctypes.c_int32),
                ("valid_samples", ctypes.c_int32), ("valid_tris", ctypes.c_int32), ("num_pairs", ctypes.c_int32),
                ("view_log2up", ctypes.c_int32), ("errors", ctypes.c_int32), ("rows_beyond_n", ctypes.c_int64),
                ("sub", ctypes.c_float * 2), ("lp_begin", ctypes.c_float * 3), ("lp_end", ctypes.c_float * 3),
                ("lp_factor", ctypes.c_float * 2), ("sample_aabb", ctypes.c_float * 8),
                ("model_aabb", ctypes.c_float * 8), ("first_error", ctypes.c_char * 160),
                ("surf_handle", ctypes.c_int64), ("pos_tex_handle", ctypes.c_int64), ("view_error", ctypes.c_int64),
                ("masks", ctypes.POINTER(ctypes.c_uint32)), ("stage_ms", f32p), ("bins", ctypes.c_int32),
                ("pad0", ctypes.c_int32), ("q2_events", ctypes.c_int64)]


_libs: dict = {}


def lib_path(fmad: bool = False, bins: int = REF_BINS) -> str:
    tag = "" if bins == REF_BINS else f"_b{bins}"
    return os.path.join(HERE, "_ref", f"libref4dzb_gpu{tag}{'_fmad' if fmad else ''}.so")


def available(fmad: bool = False, bins: int = REF_BINS) -> bool:
    return bins in BUILT_BINS and os.path.exists(lib_path(fmad, bins))


def load(fmad: bool = False, bins: int = REF_BINS) -> ctypes.CDLL:
    key = (fmad, bins)
    if key not in _libs:
        if bins not in BUILT_BINS:
            raise ValueError(f"no reference build at {bins} x {bins} bins (built: {BUILT_BINS})")
        lib = ctypes.CDLL(lib_path(fmad, bins), mode=ctypes.RTLD_LOCAL)
        lib.ref_gpu_frame.argtypes = [ctypes.POINTER(RefGpuIn), ctypes.POINTER(RefGpuOut)]
        lib.ref_gpu_frame.restype = ctypes.c_int
        _libs[key] = lib
    return _libs[key]


class PreflightError(RuntimeError):
    pass


def preflight(scene, occ_stride: int = 64, bins: int = REF_BINS) -> dict:
    """Check on the CPU, with the oracle at the build's bins, that a scene stays
    inside the reference's buffers.  occ_stride thins the oracle's occlusion
    stage (the checked quantities come from the binning stages)."""
    import dataclasses

    from . import orc

    n = scene.light.n
    if scene.light.cols != n or not (1 < n <= 32):
        raise PreflightError(f"light grid {n} x {scene.light.cols}: the per-sample kernel runs 2..32 "
                             "square grids only")
    if bins not in BUILT_BINS:
        raise PreflightError(f"no reference build at {bins} x {bins} bins")
    sb = dataclasses.replace(scene, bins=bins)
    fr = orc.frame(sb, occ_stride=occ_stride)
    sc = fr.scalars
    if sc["quirk_key_range"]:
        raise PreflightError(f"{sc['quirk_key_range']} sample keys outside the {bins} x {bins} grid")
    if sc["num_pairs"] + bins * bins > PAIR_BUFFER:
        raise PreflightError(f"{sc['num_pairs']} triangle/bin pairs exceed the reference's pair buffer")
    return sc


def run(scene, fmad: bool = False, warmup: int = 0, reps: int = 1, checked: bool = False,
        masks: bool = False, bins: int = REF_BINS) -> dict:
    """Frames through the reference on the current GPU (device 0 of this process),
    built at bins x bins light-plane bins.  The shadow buffer of the last launch
    is returned at y*W+x; launch_ms holds the CUDA-event time of each timed
    FDLaunch (L2 flushed before each), stage_ms [reps, 5] the time of each of
    its stage drivers (STAGES; -1 where one did not run).  With
    masks, "mask_rows" holds each sample's N light-row words as the reference's
    per-sample kernel left them ([S, N] uint32 at y*W+x) and "mask_written"
    where that kernel ran (binned samples)."""
    if not checked:
        preflight(scene, bins=bins)
    lib = load(fmad, bins)
    pos = np.ascontiguousarray(scene.pos, np.float32)
    nrm = np.ascontiguousarray(scene.nrm, np.float32)
    vtx = np.ascontiguousarray(scene.vtx, np.float32)
    idx = np.ascontiguousarray(scene.idx, np.int32)
    reps = max(int(reps), 1)
    shadow = np.zeros(scene.S, np.float32)
    launch_ms = np.zeros(reps, np.float32)
    own_ms = np.zeros(reps, np.float32)
    ri = RefGpuIn()
    ri.W, ri.H = scene.W, scene.H
    ri.pos, ri.nrm = pos.ctypes.data_as(f32p), nrm.ctypes.data_as(f32p)
    ri.vtx = vtx.ctypes.data_as(f32p)
    ri.V, ri.vstride_bytes = vtx.shape[0], vtx.shape[1] * 4
    ri.idx, ri.T = idx.ctypes.data_as(i32p), scene.T
    ri.cull, ri.esp = int(bool(scene.cull)), scene.esp
    L = scene.light
    ri.rightRadius, ri.topRadius = L.right_radius, L.top_radius
    ri.position[:] = list(L.position)
    ri.viewDir[:] = list(L.view_dir)
    ri.upDir[:] = list(L.up_dir)
    ri.lightRes = L.n
    ri.warmup, ri.reps = int(warmup), reps
    ro = RefGpuOut()
    dump = np.zeros(scene.S * (L.n + 1) if masks else 1, np.uint32)
    if masks:
        ro.masks = dump.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    ro.shadow = shadow.ctypes.data_as(f32p)
    ro.launch_ms = launch_ms.ctypes.data_as(f32p)
    ro.fdlaunch_ms = own_ms.ctypes.data_as(f32p)
    stage_ms = np.full(reps * len(STAGES), -1.0, np.float32)
    ro.stage_ms = stage_ms.ctypes.data_as(f32p)
    rc = lib.ref_gpu_frame(ctypes.byref(ri), ctypes.byref(ro))
    out = {"shadow": shadow, "launch_ms": launch_ms, "fdlaunch_ms": own_ms, "rc": rc,
           "stage_ms": stage_ms.reshape(reps, len(STAGES)),
           "first_error": ro.first_error.decode(errors="replace")}
    for name, _ in RefGpuOut._fields_:
        v = getattr(ro, name)
        if isinstance(v, (int, float)):
            out[name] = v
        elif hasattr(v, "_length_") and not hasattr(v, "contents") and name not in ("first_error", "stage_ms"):
            out[name] = np.array(list(v), np.float32)
    if rc == 0 and out.get("bins") != bins:
        raise RuntimeError(f"reference build reports {out.get('bins')} bins, expected {bins}")
    if rc:
        raise RuntimeError(f"reference GPU frame failed: {out['errors']} CUDA errors, first: {out['first_error']}")
    if masks:
        d = dump.reshape(scene.S, L.n + 1)
        out["mask_written"] = d[:, 0] == 1
        out["mask_rows"] = d[:, 1:]
    return out
