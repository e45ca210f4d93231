"""ctypes wrapper of oracle/liborc.so (see fdzb_oracle.h) -- TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liborc.so")

f32p = ctypes.POINTER(ctypes.c_float)
i32p = ctypes.POINTER(ctypes.c_int32)
u32p = ctypes.POINTER(ctypes.c_uint32)


class LightDesc(ctypes.Structure):
    _fields_ = [("rightRadius", ctypes.c_float), ("topRadius", ctypes.c_float),
                ("position", ctypes.c_float * 3), ("viewDir", ctypes.c_float * 3),
                ("upDir", ctypes.c_float * 3), ("lightResWidth", ctypes.c_int32),
                ("lightResHeight", ctypes.c_int32)]


class Light(ctypes.Structure):
    _fields_ = [("rightRadius", ctypes.c_float), ("topRadius", ctypes.c_float),
                ("position", ctypes.c_float * 3), ("viewDir", ctypes.c_float * 3),
                ("upDir", ctypes.c_float * 3), ("resW", ctypes.c_int32), ("resH", ctypes.c_int32),
                ("resNum", ctypes.c_int32), ("fullBits", ctypes.c_uint32),
                ("rightDir", ctypes.c_float * 3), ("topDir", ctypes.c_float * 3),
                ("x_delt", ctypes.c_float * 3), ("y_delt", ctypes.c_float * 3),
                ("upRight", ctypes.c_float * 3), ("downLeft", ctypes.c_float * 3),
                ("upLeft", ctypes.c_float * 3), ("downRight", ctypes.c_float * 3),
                ("mat", ctypes.c_float * 16), ("RF", ctypes.c_float * 2),
                ("fullRows", ctypes.c_uint64), ("fullCols", ctypes.c_uint64)]


class FrameIn(ctypes.Structure):
    _fields_ = [("W", ctypes.c_int32), ("H", ctypes.c_int32), ("pos", f32p), ("nrm", f32p),
                ("vtx", f32p), ("vtx_stride_floats", ctypes.c_int32), ("V", ctypes.c_int32),
                ("idx", i32p), ("T", ctypes.c_int32), ("bins", ctypes.c_int32), ("cull", ctypes.c_int32),
                ("esp", ctypes.c_float), ("light", ctypes.POINTER(Light)), ("nthreads", ctypes.c_int32),
                ("occ_stride", ctypes.c_int32), ("setup_only", ctypes.c_int32),
                ("shadow_method", ctypes.c_int32), ("depth_plane", ctypes.c_int32)]


class FrameOut(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("f", ctypes.c_float), ("sub", ctypes.c_float * 2),
                ("sample_aabb", ctypes.c_float * 6), ("model_aabb", ctypes.c_float * 6),
                ("lp_begin", ctypes.c_float * 3), ("lp_end", ctypes.c_float * 3),
                ("lp_factor", ctypes.c_float * 2), ("bins_log2", ctypes.c_int32),
                ("num_bins", ctypes.c_int32), ("view_log2up", ctypes.c_int32),
                ("valid_samples", ctypes.c_int32), ("valid_tris", ctypes.c_int32),
                ("num_pairs", ctypes.c_int32), ("pair_overflow", ctypes.c_int32),
                ("pairs_tested", ctypes.c_int64), ("quirk_rows_beyond_n", ctypes.c_int64),
                ("quirk_high_bits", ctypes.c_int64), ("quirk_key_range", ctypes.c_int64),
                ("rows_evaluated", ctypes.c_int64), ("partial_masks", ctypes.c_int64),
                ("t_total_ms", ctypes.c_double), ("t_occ_ms", ctypes.c_double),
                ("keys", i32p), ("vals", i32p), ("sorted_keys", i32p), ("sorted_vals", i32p),
                ("bin_sample_start", i32p), ("bin_sample_end", i32p), ("bin_maxz", f32p),
                ("bin_range", f32p), ("tri_aabb", f32p), ("tri_count", i32p),
                ("pair_capacity", ctypes.c_int32), ("pair_bin", i32p), ("pair_tri", i32p),
                ("sorted_pair_bin", i32p), ("sorted_pair_tri", i32p), ("bin_tri_start", i32p),
                ("bin_tri_end", i32p), ("masks", u32p), ("shadow", f32p)]


_lib = None


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    src = [os.path.join(HERE, f) for f in ("fdzb_oracle.c", "fdzb_raster_oracle.c", "fdzb_oracle.h", "Makefile")]
    if not os.path.exists(LIB) or any(os.path.getmtime(s) > os.path.getmtime(LIB) for s in src):
        env = dict(os.environ)
        env.pop("CC", None)
        subprocess.run(["make", "-s", "-C", HERE], check=True, env=env)
    lib = ctypes.CDLL(LIB)
    lib.orc_mask_words.argtypes = [ctypes.c_int32]
    lib.orc_mask_words.restype = ctypes.c_int32
    lib.orc_light_setup.argtypes = [ctypes.POINTER(LightDesc), ctypes.POINTER(Light)]
    lib.orc_light_setup.restype = None
    lib.orc_frame.argtypes = [ctypes.POINTER(FrameIn), ctypes.POINTER(FrameOut)]
    lib.orc_frame.restype = ctypes.c_int32
    lib.orc_exhaustive_fp32.argtypes = [ctypes.POINTER(FrameIn), ctypes.POINTER(FrameOut), i32p,
                                        ctypes.c_int32, u32p]
    lib.orc_exhaustive_fp32.restype = ctypes.c_int64
    lib.orc_exhaustive_fp64.argtypes = [ctypes.POINTER(FrameIn), ctypes.POINTER(FrameOut), i32p,
                                        ctypes.c_int32, u32p, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    lib.orc_exhaustive_fp64.restype = None
    _lib = lib
    return lib


def mask_words(n: int, cols: int | None = None) -> int:
    return (n * (cols if cols else n) + 31) // 32


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def light_desc(light) -> LightDesc:
    d = LightDesc()
    d.rightRadius = light.right_radius
    d.topRadius = light.top_radius
    d.position[:] = list(light.position)
    d.viewDir[:] = list(light.view_dir)
    d.upDir[:] = list(light.up_dir)
    d.lightResWidth = light.n
    d.lightResHeight = light.cols
    return d


def light_setup(light) -> Light:
    L = Light()
    d = light_desc(light)
    load().orc_light_setup(ctypes.byref(d), ctypes.byref(L))
    return L


@dataclass
class OrcFrame:
    """Result of orc_frame(): scalars and every intermediate array."""
    scalars: dict
    arrays: dict
    _in: FrameIn
    _out: FrameOut
    _keep: list


def _frame_in(scene, light: Light, nthreads: int, keep: list, occ_stride: int = 1) -> FrameIn:
    pos = np.ascontiguousarray(scene.pos, dtype=np.float32)
    nrm = np.ascontiguousarray(scene.nrm, dtype=np.float32)
    vtx = np.ascontiguousarray(scene.vtx, dtype=np.float32)
    idx = np.ascontiguousarray(scene.idx, dtype=np.int32)
    keep += [pos, nrm, vtx, idx, light]
    fi = FrameIn()
    fi.W, fi.H = scene.W, scene.H
    fi.pos, fi.nrm = _p(pos, f32p), _p(nrm, f32p)
    fi.vtx = _p(vtx, f32p)
    fi.vtx_stride_floats = vtx.shape[1]
    fi.V = vtx.shape[0]
    fi.idx = _p(idx, i32p)
    fi.T = idx.shape[0]
    fi.bins = scene.bins
    fi.cull = int(bool(scene.cull))
    fi.esp = scene.esp
    fi.light = ctypes.pointer(light)
    fi.nthreads = nthreads
    fi.occ_stride = occ_stride
    fi.depth_plane = int(bool(getattr(scene, "depth_plane", False)))
    return fi


def frame(scene, nthreads: int = 0, pair_capacity: int | None = None, occ_stride: int = 1,
          setup_only: bool = False, shadow_method: int = 0) -> OrcFrame:
    """Run the FP32 restatement (O2) on a scenes.Scene.  occ_stride > 1 runs the
    occlusion stage only for every occ_stride-th sorted valid sample;
    setup_only stops after the light plane (what the exhaustive baselines need)."""
    lib = load()
    keep: list = []
    light = light_setup(scene.light)
    fi = _frame_in(scene, light, nthreads, keep, occ_stride)
    fi.shadow_method = int(shadow_method)   # 1: the reference's ray-cast check
    if setup_only:
        # scalars only: every output array pointer stays NULL
        fi.setup_only = 1
        fo = FrameOut()
        rc = lib.orc_frame(ctypes.byref(fi), ctypes.byref(fo))
        if rc != 0:
            raise RuntimeError(f"orc_frame failed: {rc}")
        sc = {}
        for name, _ in FrameOut._fields_:
            v = getattr(fo, name)
            if isinstance(v, (int, float)):
                sc[name] = v
            elif hasattr(v, "_length_") and not hasattr(v, "contents"):
                sc[name] = list(v)
        return OrcFrame(scalars=sc, arrays={}, _in=fi, _out=fo, _keep=keep)
    S, T, NB = scene.W * scene.H, scene.T, scene.bins * scene.bins
    words = mask_words(scene.light.n, scene.light.cols)
    # first a counting run to size the pair buffers
    arrs = dict(
        keys=np.zeros(S, np.int32), vals=np.zeros(S, np.int32), sorted_keys=np.zeros(S, np.int32),
        sorted_vals=np.zeros(S, np.int32), bin_sample_start=np.zeros(NB + 1, np.int32),
        bin_sample_end=np.zeros(NB + 1, np.int32), bin_maxz=np.zeros(NB, np.float32),
        bin_range=np.zeros(4 * NB, np.float32), tri_aabb=np.zeros(8 * max(T, 1), np.float32),
        tri_count=np.zeros(max(T, 1), np.int32), bin_tri_start=np.zeros(NB, np.int32),
        bin_tri_end=np.zeros(NB, np.int32), masks=np.zeros(S * words, np.uint32),
        shadow=np.zeros(S, np.float32))
    cap = pair_capacity if pair_capacity is not None else max(1024, 64 * T)
    for attempt in range(2):
        for k in ("pair_bin", "pair_tri", "sorted_pair_bin", "sorted_pair_tri"):
            arrs[k] = np.zeros(max(cap, 1), np.int32)
        fo = FrameOut()
        for k, a in arrs.items():
            t = f32p if a.dtype == np.float32 else (u32p if a.dtype == np.uint32 else i32p)
            setattr(fo, k, _p(a, t))
        fo.pair_capacity = cap
        rc = lib.orc_frame(ctypes.byref(fi), ctypes.byref(fo))
        if rc != 0:
            raise RuntimeError(f"orc_frame failed: {rc}")
        if not fo.pair_overflow:
            break
        cap = fo.num_pairs + 16
    keep.append(arrs)
    sc = {}
    for name, _ in FrameOut._fields_:
        v = getattr(fo, name)
        if isinstance(v, (int, float)):
            sc[name] = v
        elif hasattr(v, "_length_") and not hasattr(v, "contents"):
            sc[name] = list(v)
    P = fo.num_pairs
    out = dict(arrs)
    for k in ("pair_bin", "pair_tri", "sorted_pair_bin", "sorted_pair_tri"):
        out[k] = arrs[k][:P].copy()
    out["tri_aabb"] = arrs["tri_aabb"][:8 * T]
    out["tri_count"] = arrs["tri_count"][:T]
    stride = max(occ_stride, 1)
    Sv = fo.valid_samples
    if fo.state == 2:
        sv = out["sorted_vals"][:Sv:stride]
        l2 = fo.view_log2up
        out["occ_samples"] = ((sv >> l2) * scene.W + (sv & ((1 << l2) - 1))).astype(np.int64)
    else:
        out["occ_samples"] = np.zeros(0, np.int64)
    return OrcFrame(scalars=sc, arrays=out, _in=fi, _out=fo, _keep=keep)


def exhaustive_fp32(scene, fr: OrcFrame, sample_ids: np.ndarray, nthreads: int = 0):
    """CPU baseline: O2 per-pair arithmetic, every valid triangle, OpenMP.
    Returns (masks [n, words], pair tests executed)."""
    lib = load()
    ids = np.ascontiguousarray(sample_ids, dtype=np.int32)
    words = mask_words(scene.light.n, scene.light.cols)
    out = np.zeros(ids.size * words, np.uint32)
    fr._in.nthreads = nthreads
    n = lib.orc_exhaustive_fp32(ctypes.byref(fr._in), ctypes.byref(fr._out), _p(ids, i32p), ids.size,
                                _p(out, u32p))
    return out.reshape(ids.size, words), int(n)


class O3Stats(ctypes.Structure):
    _fields_ = [("triangles", ctypes.c_int64), ("candidates", ctypes.c_int64), ("evaluated", ctypes.c_int64),
                ("fallback", ctypes.c_int64), ("skipped_blocks", ctypes.c_int64)]


def exhaustive_fp64(scene, fr: OrcFrame, sample_ids: np.ndarray, nthreads: int = 0, stats: bool = False,
                    distances: bool = True):
    """O3: FP64 per-light-sample test.  Returns (masks [n, words], boundary
    distance [n, rows * cols] in light-plane units, or None without distances)
    and, with stats, a dict of the work counts."""
    lib = load()
    ids = np.ascontiguousarray(sample_ids, dtype=np.int32)
    NN = scene.light.rows * scene.light.cols
    words = mask_words(scene.light.n, scene.light.cols)
    out = np.zeros(max(ids.size * words, 1), np.uint32)
    dist = np.zeros(max(ids.size * NN, 1), np.float64) if distances else None
    st = O3Stats()
    fr._in.nthreads = nthreads
    lib.orc_exhaustive_fp64(ctypes.byref(fr._in), ctypes.byref(fr._out), _p(ids, i32p), ids.size,
                            _p(out, u32p), dist.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if distances
                            else None, ctypes.byref(st))
    res = (out[:ids.size * words].reshape(ids.size, words),
           dist[:ids.size * NN].reshape(ids.size, NN) if distances else None)
    if stats:
        return res + ({n: int(getattr(st, n)) for n, _ in O3Stats._fields_},)
    return res


def light_plane_units(light) -> float:
    """World units per light-grid step along x_delt (= 2 * right radius / rows)."""
    return 2.0 * light.right_radius / light.rows


# ---- G-buffer rasteriser oracle (fdzb_raster_oracle.c) ----------------------

class RasterIn(ctypes.Structure):
    _fields_ = [("vtx", f32p), ("vtx_stride_floats", ctypes.c_int32), ("pos_offset", ctypes.c_int32),
                ("nrm_offset", ctypes.c_int32), ("idx", u32p), ("n_tri", ctypes.c_int32), ("tri_material", i32p),
                ("materials", f32p), ("model", ctypes.c_float * 16), ("view_proj", ctypes.c_float * 16),
                ("W", ctypes.c_int32), ("H", ctypes.c_int32), ("clear", ctypes.c_int32)]


class RasterOut(ctypes.Structure):
    _fields_ = [("g0", f32p), ("g1", f32p), ("g2", f32p), ("g3", f32p), ("depth", f32p),
                ("sub_tris", ctypes.c_int64), ("dropped", ctypes.c_int64)]


def col_major(m) -> list:
    """A 4x4 matrix (out = m @ v) as 16 column-major floats."""
    return [float(v) for v in np.asarray(m, dtype=np.float32).reshape(4, 4).reshape(-1, order="F")]


def raster(vtx, idx, materials, model, view_proj, W: int, H: int, tri_material=None, clear: bool = True,
           prev: dict | None = None, pos_offset: int = 0, nrm_offset: int = 5) -> dict:
    """One draw through the rasteriser oracle.  vtx: float32 [V, floats per
    vertex]; idx: [T, 3]; materials: float32 [M, 10].  With clear=False, `prev`
    holds the earlier draw's g0..g3 and depth, which are drawn over."""
    lib = load()
    if not hasattr(lib, "_raster_ready"):
        lib.orc_raster.argtypes = [ctypes.POINTER(RasterIn), ctypes.POINTER(RasterOut)]
        lib.orc_raster.restype = ctypes.c_int32
        lib._raster_ready = True
    vtx = np.ascontiguousarray(vtx, np.float32)
    idx = np.ascontiguousarray(idx, np.uint32).reshape(-1, 3)
    mats = np.ascontiguousarray(materials, np.float32).reshape(-1, 10)
    S = W * H
    if clear or prev is None:
        out = {k: np.zeros((S, 4), np.float32) for k in ("g0", "g1", "g2", "g3")}
        out["depth"] = np.zeros(S, np.float32)
    else:
        out = {k: np.array(prev[k], np.float32, copy=True) for k in ("g0", "g1", "g2", "g3", "depth")}
    ri = RasterIn()
    ri.vtx, ri.vtx_stride_floats = _p(vtx, f32p), vtx.shape[1]
    ri.pos_offset, ri.nrm_offset = pos_offset, nrm_offset
    ri.idx, ri.n_tri = _p(idx, u32p), idx.shape[0]
    tm = None
    if tri_material is not None:
        tm = np.ascontiguousarray(tri_material, np.int32)
        ri.tri_material = _p(tm, i32p)
    ri.materials = _p(mats, f32p)
    ri.model[:] = col_major(model)
    ri.view_proj[:] = col_major(view_proj)
    ri.W, ri.H, ri.clear = W, H, int(bool(clear))
    ro = RasterOut()
    for k in ("g0", "g1", "g2", "g3", "depth"):
        setattr(ro, k, _p(out[k], f32p))
    rc = lib.orc_raster(ctypes.byref(ri), ctypes.byref(ro))
    if rc:
        raise RuntimeError(f"orc_raster failed: {rc}")
    out["sub_tris"], out["dropped"] = int(ro.sub_tris), int(ro.dropped)
    return out
