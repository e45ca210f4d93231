"""ctypes wrapper of oracle/_ref/libref4dzb.so -- the reference's own soft-shadow
sources (4DZB/FDZB_Soft_Shadow) compiled for the CPU by oracle/ref_emu/build_ref.py.
TEST INFRASTRUCTURE ONLY: used to generate and check golden fixtures and as the
timed reference arm of bench.py.  Its bin grid is the reference's compile-time
16 x 16 (FS/constants.h:13).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref4dzb.so")
REF_BINS = 16

f32p = ctypes.POINTER(ctypes.c_float)
i32p = ctypes.POINTER(ctypes.c_int32)


class RefIn(ctypes.Structure):
    _fields_ = [("W", ctypes.c_int32), ("H", ctypes.c_int32), ("pos", f32p), ("nrm", f32p), ("vtx", f32p),
                ("V", ctypes.c_int32), ("vstride_bytes", ctypes.c_int32), ("idx", i32p), ("T", ctypes.c_int32),
                ("cull", ctypes.c_int32), ("esp", ctypes.c_float), ("rightRadius", ctypes.c_float),
                ("topRadius", ctypes.c_float), ("position", ctypes.c_float * 3), ("viewDir", ctypes.c_float * 3),
                ("upDir", ctypes.c_float * 3), ("lightRes", ctypes.c_int32), ("nthreads", ctypes.c_int32)]


class RefOut(ctypes.Structure):
    _fields_ = [("shadow", f32p), ("sorted_keys", i32p), ("sorted_vals", i32p), ("bin_sample_start", i32p),
                ("bin_sample_end", i32p), ("bin_maxz", f32p), ("bin_range", f32p), ("tri_aabb", f32p),
                ("tri_count", i32p), ("tri_prefix", i32p), ("pair_capacity", ctypes.c_int32),
                ("sorted_pair_bin", i32p), ("sorted_pair_tri", i32p), ("bin_tri_start", i32p),
                ("bin_tri_end", i32p), ("num_bins", ctypes.c_int32), ("valid_samples", ctypes.c_int32),
                ("valid_tris", ctypes.c_int32), ("num_pairs", ctypes.c_int32), ("view_log2up", ctypes.c_int32),
                ("errors", ctypes.c_int32), ("ms", ctypes.c_float), ("mat", ctypes.c_float * 16),
                ("RF", ctypes.c_float * 2), ("corners", ctypes.c_float * 12), ("deltas", ctypes.c_float * 6),
                ("sub", ctypes.c_float * 2), ("lp_begin", ctypes.c_float * 3), ("lp_end", ctypes.c_float * 3),
                ("lp_factor", ctypes.c_float * 2), ("sample_aabb", ctypes.c_float * 8),
                ("model_aabb", ctypes.c_float * 8)]


_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(LIB)
        lib.ref_frame.argtypes = [ctypes.POINTER(RefIn), ctypes.POINTER(RefOut)]
        lib.ref_frame.restype = ctypes.c_int
        _lib = lib
    return _lib


def run(scene, nthreads: int = 0, pair_capacity: int | None = None) -> dict:
    """One frame through the reference's FD:: API.  Arrays are in the reference's
    own encodings (sample ids y << ceil(log2 W) | x), shadow at y*W+x."""
    lib = load()
    pos = np.ascontiguousarray(scene.pos, np.float32)
    nrm = np.ascontiguousarray(scene.nrm, np.float32)
    vtx = np.ascontiguousarray(scene.vtx, np.float32)
    idx = np.ascontiguousarray(scene.idx, np.int32)
    S, T, NB = scene.S, scene.T, REF_BINS * REF_BINS
    cap = pair_capacity or max(1024, 64 * T)
    a = dict(shadow=np.zeros(S, np.float32), sorted_keys=np.zeros(S, np.int32),
             sorted_vals=np.zeros(S, np.int32), bin_sample_start=np.zeros(NB + 1, np.int32),
             bin_sample_end=np.zeros(NB + 1, np.int32), bin_maxz=np.zeros(NB, np.float32),
             bin_range=np.zeros(4 * NB, np.float32), tri_aabb=np.zeros(8 * max(T, 1), np.float32),
             tri_count=np.zeros(max(T, 1), np.int32), tri_prefix=np.zeros(max(T, 1), np.int32),
             sorted_pair_bin=np.zeros(cap, np.int32), sorted_pair_tri=np.zeros(cap, np.int32),
             bin_tri_start=np.zeros(NB, np.int32), bin_tri_end=np.zeros(NB, np.int32))
    ri = RefIn()
    ri.W, ri.H = scene.W, scene.H
    ri.pos, ri.nrm = pos.ctypes.data_as(f32p), nrm.ctypes.data_as(f32p)
    ri.vtx = vtx.ctypes.data_as(f32p)
    ri.V, ri.vstride_bytes = vtx.shape[0], vtx.shape[1] * 4
    ri.idx, ri.T = idx.ctypes.data_as(i32p), T
    ri.cull, ri.esp = int(bool(scene.cull)), scene.esp
    L = scene.light
    ri.rightRadius, ri.topRadius = L.right_radius, L.top_radius
    ri.position[:] = list(L.position)
    ri.viewDir[:] = list(L.view_dir)
    ri.upDir[:] = list(L.up_dir)
    ri.lightRes = L.n
    ri.nthreads = nthreads
    ro = RefOut()
    for k, v in a.items():
        setattr(ro, k, v.ctypes.data_as(f32p if v.dtype == np.float32 else i32p))
    ro.pair_capacity = cap
    rc = lib.ref_frame(ctypes.byref(ri), ctypes.byref(ro))
    if rc:
        raise RuntimeError(f"ref_frame failed: {rc}")
    out = {k: v for k, v in a.items()}
    P = min(ro.num_pairs, cap)
    out["sorted_pair_bin"] = a["sorted_pair_bin"][:P].copy()
    out["sorted_pair_tri"] = a["sorted_pair_tri"][:P].copy()
    out["tri_aabb"] = a["tri_aabb"][:8 * T]
    out["tri_count"] = a["tri_count"][:T]
    out["tri_prefix"] = a["tri_prefix"][:T]
    for name, _ in RefOut._fields_:
        v = getattr(ro, name)
        if isinstance(v, (int, float)):
            out[name] = v
        elif hasattr(v, "_length_") and not hasattr(v, "contents"):
            out[name] = np.array(list(v), np.float32)
    return out
