"""fdzb-b200: B200-native FDZB soft shadows (4DZB's FDZB_Soft_Shadow path).

The compute path is ``libfdzb.so`` (hand-written sm_100a CUDA behind the C ABI
declared in ``include/fdzb.h``).  This module is a thin ctypes binding:

* :class:`Context` wraps the re-entrant ``fdzb_ctx_*`` API;
* the ``FD*`` functions mirror the reference's ``namespace FD`` entry points
  (4DZB/FDZB_Soft_Shadow/api.h:10-56) on a process-wide context, with device
  tensors (or raw device pointers) in place of GL object names.

There is no CPU fallback: importing works anywhere, but every call that needs
the library raises :class:`FdzbError` if ``libfdzb.so`` is missing or no CUDA
device is present.  Build with ``python 4dzb_b200/build.py``.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfdzb.so")

FDZB_OK = 0
ERRORS = {
    -1: "FDZB_ERR_INVALID_ARG", -2: "FDZB_ERR_CUDA", -3: "FDZB_ERR_NOT_INITIALIZED",
    -4: "FDZB_ERR_NO_MEMORY", -5: "FDZB_ERR_CAPACITY", -6: "FDZB_ERR_DEVICE_TIMEOUT",
    -7: "FDZB_ERR_UNSUPPORTED", -8: "FDZB_ERR_NOT_READY",
}

ARRAYS = {
    "sample_keys": (0, np.int32), "sorted_sample_keys": (1, np.int32), "sorted_sample_ids": (2, np.int32),
    "bin_sample_start": (3, np.int32), "bin_sample_end": (4, np.int32), "bin_maxz": (5, np.float32),
    "bin_range": (6, np.float32), "tri_count": (7, np.int32), "pair_bin": (8, np.int32),
    "pair_tri": (9, np.int32), "sorted_pair_bin": (10, np.int32), "sorted_pair_tri": (11, np.int32),
    "bin_tri_start": (12, np.int32), "bin_tri_end": (13, np.int32), "tri_aabb": (14, np.float32),
    "work_counters": (15, np.uint64),
}

# Every symbol declared in include/fdzb.h.
EXPORTED = [
    "fdzb_init", "fdzb_set_backface_cull", "fdzb_add_model", "fdzb_set_sample_buffers",
    "fdzb_set_output_buffer", "fdzb_register_resources", "fdzb_unregister_resources",
    "fdzb_set_bin_num", "fdzb_set_view", "fdzb_set_scenes_esp", "fdzb_set_scene_params",
    "fdzb_set_area_light", "fdzb_launch", "fdzb_move_model", "fdzb_last_error",
    "fdzb_ctx_create", "fdzb_ctx_destroy", "fdzb_ctx_set_stream", "fdzb_ctx_set_backface_cull",
    "fdzb_ctx_add_model", "fdzb_ctx_set_sample_buffers", "fdzb_ctx_set_output_buffer",
    "fdzb_ctx_set_bin_num", "fdzb_ctx_set_view", "fdzb_ctx_set_scenes_esp",
    "fdzb_ctx_set_scene_params", "fdzb_ctx_set_area_light", "fdzb_ctx_move_model",
    "fdzb_ctx_launch", "fdzb_ctx_launch_async", "fdzb_ctx_sync", "fdzb_ctx_get_stats",
    "fdzb_ctx_export", "fdzb_ctx_set_debug", "fdzb_ctx_set_tri_order", "fdzb_light_setup",
    "fdzb_version", "fdzb_ctx_set_profiling", "fdzb_measure_alu_rate", "fdzb_check_division", "fdzb_sort_pairs_noalloc",
    "fdzb_ctx_set_graph", "fdzb_batch_create", "fdzb_batch_destroy", "fdzb_batch_set_stream",
    "fdzb_batch_set_graph", "fdzb_batch_set_profiling", "fdzb_batch_set_tri_order",
    "fdzb_batch_launch_async", "fdzb_batch_sync", "fdzb_batch_launch", "fdzb_batch_get_frame_stats",
    "fdzb_batch_get_stats", "fdzb_batch_frame_bins", "fdzb_batch_autotune",
    "fdzb_ctx_set_occlusion_schedule", "fdzb_batch_set_occlusion_schedule", "fdzb_ctx_set_pair_capacity_limit",
    "fdzb_ctx_set_model_transform", "fdzb_ctx_set_shadow_method", "fdzb_light_sample_positions", "fdzb_shade",
    "fdzb_ctx_set_depth_plane", "fdzb_batch_set_depth_plane",
    "fdzb_raster_create", "fdzb_raster_destroy", "fdzb_raster_set_stream", "fdzb_raster_draw",
    "fdzb_raster_sync", "fdzb_raster_get_stats",
    "fdzb_serve_default_config", "fdzb_serve_create", "fdzb_serve_destroy", "fdzb_serve_add_scene",
    "fdzb_serve_submit", "fdzb_serve_poll", "fdzb_serve_wait", "fdzb_serve_drain", "fdzb_serve_autotune",
    "fdzb_serve_get_stats", "fdzb_serve_reset_stats", "fdzb_serve_last_worker_error",
    "fdzb_ctx_set_launch_epoch", "fdzb_ctx_get_launch_epoch",
    "fdzb_ctx_set_occlusion_shape", "fdzb_batch_frame_shape", "fdzb_batch_set_occlusion_shape",
    "fdzb_ctx_set_open_box", "fdzb_batch_set_open_box",
]

# Open-box cull modes (include/fdzb.h).
OPEN_BOX_OFF, OPEN_BOX_ON, OPEN_BOX_AUTO = 0, 1, 2

# Occlusion shapes (staged triangles per chunk, samples per warp item).
OCC_CHUNKS = (8, 16, 32)
OCC_ITEMS = (32, 64, 128)

# Launch number at which the look-back status words are cleared (include/fdzb.h).
LOOKBACK_EPOCH_LIMIT = 0x0FFFFFFF

STAGES = ["setup", "sample_sort", "tri_pairs", "pair_sort", "occlusion"]

TRI_ORDER_REFERENCE = 0
TRI_ORDER_COVERAGE = 1
TRI_ORDER_DEPTH = TRI_ORDER_COVERAGE

SHADOW_EDGE_MASKS = 0
SHADOW_RAY_CAST = 1

OCC_LANE_PER_SAMPLE = 0
OCC_LANE_PER_PAIR = 1


class FdzbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class AreaLightDesc(ctypes.Structure):
    """Same 52-byte layout as AreaLightDes (4DZB/FDZB_Soft_Shadow/AreaLightDesc.h:3-14)."""
    _fields_ = [("rightRadius", ctypes.c_float), ("topRadius", ctypes.c_float),
                ("position", ctypes.c_float * 3), ("viewDir", ctypes.c_float * 3),
                ("upDir", ctypes.c_float * 3), ("lightResWidth", ctypes.c_int32),
                ("lightResHeight", ctypes.c_int32)]

    @classmethod
    def from_light(cls, light) -> "AreaLightDesc":
        d = cls()
        d.rightRadius = light.right_radius
        d.topRadius = light.top_radius
        d.position[:] = list(light.position)
        d.viewDir[:] = list(light.view_dir)
        d.upDir[:] = list(light.up_dir)
        d.lightResWidth = light.n
        d.lightResHeight = light.nh if getattr(light, "nh", 0) else light.n
        return d


class FrameStats(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("valid_samples", ctypes.c_int32),
                ("valid_triangles", ctypes.c_int32), ("num_pairs", ctypes.c_int32),
                ("num_bins", ctypes.c_int32), ("pair_capacity", ctypes.c_int32),
                ("pair_tests", ctypes.c_int64), ("f", ctypes.c_float), ("sub", ctypes.c_float * 2),
                ("lp_begin", ctypes.c_float * 3), ("lp_end", ctypes.c_float * 3),
                ("lp_factor", ctypes.c_float * 2), ("sample_aabb", ctypes.c_float * 6),
                ("model_aabb", ctypes.c_float * 6), ("replans", ctypes.c_int32),
                ("quirk_key_range", ctypes.c_int32), ("kernel_launches", ctypes.c_int32),
                ("triangle_passes", ctypes.c_int32), ("rows_evaluated", ctypes.c_int64),
                ("partial_masks", ctypes.c_int64), ("stage_ms", ctypes.c_float * 5),
                ("pad1", ctypes.c_float)]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class FrameDesc(ctypes.Structure):
    """fdzb_frame_desc: one frame of a batch."""
    _fields_ = [("d_pos", ctypes.c_void_p), ("d_nrm", ctypes.c_void_p), ("W", ctypes.c_int32),
                ("H", ctypes.c_int32), ("d_vtx", ctypes.c_void_p), ("n_vtx", ctypes.c_size_t),
                ("vtx_stride_bytes", ctypes.c_size_t), ("d_idx", ctypes.c_void_p), ("n_tri", ctypes.c_size_t),
                ("light", AreaLightDesc), ("bins", ctypes.c_int32), ("cull", ctypes.c_int32),
                ("esp", ctypes.c_float), ("d_shadow", ctypes.c_void_p), ("d_masks", ctypes.c_void_p),
                ("model_transform", ctypes.POINTER(ctypes.c_float))]


class BatchStats(ctypes.Structure):
    _fields_ = [("totals", FrameStats), ("frames", ctypes.c_int32), ("from_graph", ctypes.c_int32),
                ("graph_captures", ctypes.c_int64), ("graph_replays", ctypes.c_int64),
                ("tuned_classes", ctypes.c_int32), ("pad0", ctypes.c_int32), ("tune_launches", ctypes.c_int64),
                ("ms", ctypes.c_float), ("pad1", ctypes.c_float)]

    def as_dict(self) -> dict:
        out = {n: getattr(self, n) for n, _ in self._fields_ if n != "totals"}
        out["totals"] = self.totals.as_dict()
        return out


class ServeConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("slots", ctypes.c_int32), ("max_batch_frames", ctypes.c_int32),
                ("use_graphs", ctypes.c_int32), ("max_batch_samples", ctypes.c_int64),
                ("memory_budget_bytes", ctypes.c_uint64), ("max_batch_triangles", ctypes.c_int64)]


class Request(ctypes.Structure):
    _fields_ = [("scene_id", ctypes.c_int32), ("W", ctypes.c_int32), ("H", ctypes.c_int32),
                ("bins", ctypes.c_int32), ("d_pos", ctypes.c_void_p), ("d_nrm", ctypes.c_void_p),
                ("light", AreaLightDesc), ("pad0", ctypes.c_int32), ("d_shadow", ctypes.c_void_p),
                ("d_masks", ctypes.c_void_p), ("model_transform", ctypes.POINTER(ctypes.c_float))]


class RequestResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("batch_frames", ctypes.c_int32), ("latency_ms", ctypes.c_double),
                ("queue_ms", ctypes.c_double), ("stats", FrameStats)]

    def as_dict(self) -> dict:
        out = {n: getattr(self, n) for n, _ in self._fields_ if n != "stats"}
        out["stats"] = self.stats.as_dict()
        return out


class ServeStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("rejected", ctypes.c_int64),
                ("failed", ctypes.c_int64), ("batches", ctypes.c_int64), ("batched_frames", ctypes.c_int64),
                ("overlapped_batches", ctypes.c_int64), ("queued", ctypes.c_int64), ("busy_slots", ctypes.c_int32),
                ("max_inflight_batches", ctypes.c_int32), ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double), ("frames_per_s", ctypes.c_double),
                ("held_bytes", ctypes.c_int64), ("peak_bytes", ctypes.c_int64), ("budget_bytes", ctypes.c_int64),
                ("tuned_classes", ctypes.c_int32), ("slots", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


class ShadeDesc(ctypes.Structure):
    """fdzb_shade_desc."""
    _fields_ = [("W", ctypes.c_int32), ("H", ctypes.c_int32), ("d_g0", ctypes.c_void_p), ("d_g1", ctypes.c_void_p),
                ("d_g2", ctypes.c_void_p), ("d_g3", ctypes.c_void_p), ("d_shadow", ctypes.c_void_p),
                ("d_rgba", ctypes.c_void_p), ("camera_pos", ctypes.c_float * 3), ("La", ctypes.c_float * 3),
                ("Ld", ctypes.c_float * 3), ("Ls", ctypes.c_float * 3), ("n_light_samples", ctypes.c_int32),
                ("d_light_samples", ctypes.c_void_p)]


class RasterDesc(ctypes.Structure):
    """fdzb_raster_desc."""
    _fields_ = [("d_vtx", ctypes.c_void_p), ("n_vtx", ctypes.c_int32), ("vtx_stride_bytes", ctypes.c_int32),
                ("pos_offset", ctypes.c_int32), ("nrm_offset", ctypes.c_int32), ("d_idx", ctypes.c_void_p),
                ("n_tri", ctypes.c_int32), ("d_tri_material", ctypes.c_void_p), ("d_materials", ctypes.c_void_p),
                ("n_materials", ctypes.c_int32), ("model", ctypes.c_float * 16), ("view_proj", ctypes.c_float * 16),
                ("W", ctypes.c_int32), ("H", ctypes.c_int32), ("clear", ctypes.c_int32), ("d_g0", ctypes.c_void_p),
                ("d_g1", ctypes.c_void_p), ("d_g2", ctypes.c_void_p), ("d_g3", ctypes.c_void_p),
                ("d_depth", ctypes.c_void_p)]


class RasterStats(ctypes.Structure):
    """fdzb_raster_stats."""
    _fields_ = [("triangles", ctypes.c_int64), ("sub_triangles", ctypes.c_int64), ("dropped", ctypes.c_int64),
                ("tile_pairs", ctypes.c_int64), ("bad_indices", ctypes.c_int64), ("bad_materials", ctypes.c_int64),
                ("tiles_x", ctypes.c_int32), ("tiles_y", ctypes.c_int32), ("ms", ctypes.c_float),
                ("pad", ctypes.c_float)]


_lib: Optional[ctypes.CDLL] = None


def lib_available() -> bool:
    return os.path.exists(LIB_PATH)


def load() -> ctypes.CDLL:
    """Load libfdzb.so (raises FdzbError if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FdzbError(-3, f"{LIB_PATH} not built (python 4dzb_b200/build.py)")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i32, sz, f32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t, ctypes.c_float
    P = ctypes.POINTER
    sig = {
        "fdzb_init": ([], i32), "fdzb_set_backface_cull": ([i32], i32),
        "fdzb_add_model": ([vp, sz, sz, vp, sz, ctypes.c_char_p], i32),
        "fdzb_set_sample_buffers": ([vp, vp], i32), "fdzb_set_output_buffer": ([vp, vp], i32),
        "fdzb_register_resources": ([], i32), "fdzb_unregister_resources": ([], i32),
        "fdzb_set_bin_num": ([sz], i32), "fdzb_set_view": ([i32, i32], i32),
        "fdzb_set_scenes_esp": ([f32], i32), "fdzb_set_scene_params": ([sz, sz], i32),
        "fdzb_set_area_light": ([P(AreaLightDesc)], i32), "fdzb_launch": ([], f32),
        "fdzb_move_model": ([P(ctypes.c_float)], i32), "fdzb_last_error": ([], ctypes.c_char_p),
        "fdzb_ctx_create": ([P(vp), i32], i32), "fdzb_ctx_destroy": ([vp], i32),
        "fdzb_ctx_set_stream": ([vp, vp], i32), "fdzb_ctx_set_backface_cull": ([vp, i32], i32),
        "fdzb_ctx_add_model": ([vp, vp, sz, sz, vp, sz, ctypes.c_char_p], i32),
        "fdzb_ctx_set_sample_buffers": ([vp, vp, vp], i32),
        "fdzb_ctx_set_output_buffer": ([vp, vp, vp], i32), "fdzb_ctx_set_bin_num": ([vp, sz], i32),
        "fdzb_ctx_set_view": ([vp, i32, i32], i32), "fdzb_ctx_set_scenes_esp": ([vp, f32], i32),
        "fdzb_ctx_set_scene_params": ([vp, sz, sz], i32),
        "fdzb_ctx_set_area_light": ([vp, P(AreaLightDesc)], i32),
        "fdzb_ctx_move_model": ([vp, P(ctypes.c_float)], i32),
        "fdzb_ctx_launch": ([vp, P(ctypes.c_float)], i32), "fdzb_ctx_launch_async": ([vp], i32),
        "fdzb_ctx_sync": ([vp], i32), "fdzb_ctx_get_stats": ([vp, P(FrameStats)], i32),
        "fdzb_ctx_export": ([vp, i32, vp, sz], i32), "fdzb_ctx_set_debug": ([vp, i32], i32),
        "fdzb_ctx_set_tri_order": ([vp, i32], i32), "fdzb_ctx_set_profiling": ([vp, i32], i32),
        "fdzb_measure_alu_rate": ([P(ctypes.c_double)], i32),
        "fdzb_check_division": ([ctypes.c_uint64, ctypes.c_uint64, P(ctypes.c_uint64), P(ctypes.c_uint64)], i32),
        "fdzb_light_setup": ([P(AreaLightDesc), P(ctypes.c_float), P(ctypes.c_float),
                              P(ctypes.c_float), P(ctypes.c_float)], i32),
        "fdzb_version": ([], ctypes.c_char_p),
        "fdzb_ctx_set_graph": ([vp, i32], i32),
        "fdzb_ctx_set_launch_epoch": ([vp, ctypes.c_uint32], i32),
        "fdzb_ctx_get_launch_epoch": ([vp, vp], i32),
        "fdzb_ctx_set_occlusion_schedule": ([vp, i32], i32),
        "fdzb_ctx_set_occlusion_shape": ([vp, i32, i32], i32),
        "fdzb_batch_frame_shape": ([vp, i32, vp, vp, vp], i32),
        "fdzb_batch_set_occlusion_shape": ([vp, i32, i32], i32),
        "fdzb_ctx_set_open_box": ([vp, i32], i32), "fdzb_batch_set_open_box": ([vp, i32], i32),
        "fdzb_ctx_set_pair_capacity_limit": ([vp, ctypes.c_int64], i32),
        "fdzb_ctx_set_model_transform": ([vp, P(ctypes.c_float)], i32),
        "fdzb_ctx_set_shadow_method": ([vp, i32], i32),
        "fdzb_ctx_set_depth_plane": ([vp, i32], i32), "fdzb_batch_set_depth_plane": ([vp, i32], i32),
        "fdzb_raster_create": ([P(vp), i32], i32), "fdzb_raster_destroy": ([vp], i32),
        "fdzb_raster_set_stream": ([vp, vp], i32), "fdzb_raster_draw": ([vp, P(RasterDesc)], i32),
        "fdzb_raster_sync": ([vp], i32), "fdzb_raster_get_stats": ([vp, P(RasterStats)], i32),
        "fdzb_light_sample_positions": ([P(AreaLightDesc), P(ctypes.c_float)], i32),
        "fdzb_shade": ([P(ShadeDesc), vp], i32), "fdzb_batch_set_occlusion_schedule": ([vp, i32], i32),
        "fdzb_batch_create": ([P(vp), i32], i32), "fdzb_batch_destroy": ([vp], i32),
        "fdzb_batch_set_stream": ([vp, vp], i32), "fdzb_batch_set_graph": ([vp, i32], i32),
        "fdzb_batch_set_profiling": ([vp, i32], i32), "fdzb_batch_set_tri_order": ([vp, i32], i32),
        "fdzb_batch_launch_async": ([vp, P(FrameDesc), i32], i32),
        "fdzb_batch_sync": ([vp, P(ctypes.c_float)], i32),
        "fdzb_batch_launch": ([vp, P(FrameDesc), i32, P(ctypes.c_float)], i32),
        "fdzb_batch_get_frame_stats": ([vp, i32, P(FrameStats)], i32),
        "fdzb_batch_get_stats": ([vp, P(BatchStats)], i32), "fdzb_batch_frame_bins": ([vp, i32], i32),
        "fdzb_batch_autotune": ([vp, P(FrameDesc), i32, vp, sz], i32),
        "fdzb_serve_default_config": ([P(ServeConfig)], None),
        "fdzb_serve_create": ([P(vp), P(ServeConfig)], i32), "fdzb_serve_destroy": ([vp], i32),
        "fdzb_serve_add_scene": ([vp, vp, sz, sz, vp, sz, i32, f32, P(ctypes.c_int32)], i32),
        "fdzb_serve_submit": ([vp, P(Request), P(ctypes.c_uint64)], i32),
        "fdzb_serve_poll": ([vp, ctypes.c_uint64, P(RequestResult)], i32),
        "fdzb_serve_wait": ([vp, ctypes.c_uint64, i32, P(RequestResult)], i32),
        "fdzb_serve_drain": ([vp, i32], i32),
        "fdzb_serve_autotune": ([vp, P(Request), i32, vp, sz], i32),
        "fdzb_serve_get_stats": ([vp, P(ServeStats)], i32), "fdzb_serve_reset_stats": ([vp], i32),
        "fdzb_serve_last_worker_error": ([vp], ctypes.c_char_p),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _check(rc: int) -> int:
    if rc != FDZB_OK:
        msg = load().fdzb_last_error().decode()
        raise FdzbError(rc, msg)
    return rc


def _ptr(x) -> Optional[int]:
    """Device pointer of a torch tensor, or an int pointer, or None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    return int(x.data_ptr())


def light_setup(light) -> dict:
    """Host light setup (FS/api.cpp:303-400) as computed by the library."""
    lib = load()
    d = AreaLightDesc.from_light(light) if not isinstance(light, AreaLightDesc) else light
    mat = (ctypes.c_float * 16)()
    rf = (ctypes.c_float * 2)()
    corners = (ctypes.c_float * 12)()
    deltas = (ctypes.c_float * 6)()
    _check(lib.fdzb_light_setup(ctypes.byref(d), mat, rf, corners, deltas))
    return dict(mat=np.array(mat, dtype=np.float32), RF=np.array(rf, dtype=np.float32),
                corners=np.array(corners, dtype=np.float32).reshape(4, 3),
                deltas=np.array(deltas, dtype=np.float32).reshape(2, 3))


def check_division(trials: int, seed: int = 1) -> tuple:
    """(mismatches, checked): the device self-check of the occlusion rows'
    quotient against the IEEE division (fdzb_check_division)."""
    m, n = ctypes.c_uint64(), ctypes.c_uint64()
    _check(load().fdzb_check_division(trials, seed, ctypes.byref(m), ctypes.byref(n)))
    return int(m.value), int(n.value)


PROFILE_OFF, PROFILE_ALL, PROFILE_STAGES = 0, 1, 2


def _profile_mode(enable) -> int:
    """True/False or one of the PROFILE_* modes."""
    if isinstance(enable, bool):
        return PROFILE_ALL if enable else PROFILE_OFF
    return int(enable)


def measure_alu_rate() -> float:
    """FP32 lane operations per second of the current device (issue-rate probe)."""
    v = ctypes.c_double()
    _check(load().fdzb_measure_alu_rate(ctypes.byref(v)))
    return float(v.value)


def mask_words(n: int, cols: Optional[int] = None) -> int:
    """uint32 words of one sample's mask for an n x cols light grid (cols
    defaults to n)."""
    return (n * (cols if cols else n) + 31) // 32


class Context:
    """One scene / view / light on one device (the fdzb_ctx_* API)."""

    def __init__(self, device: int = -1):
        self._lib = load()
        h = ctypes.c_void_p()
        _check(self._lib.fdzb_ctx_create(ctypes.byref(h), device))
        self._h = h
        self._keep = []  # tensors whose memory the context references

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fdzb_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream) -> None:
        _check(self._lib.fdzb_ctx_set_stream(self._h, ctypes.c_void_p(stream)))

    def set_backface_cull(self, enable: bool) -> None:
        _check(self._lib.fdzb_ctx_set_backface_cull(self._h, int(bool(enable))))

    def set_debug(self, flags: int) -> None:
        """flags bit 0 (DEBUG_COPIES): keep pre-sort copies of the key arrays for
        export(); bit 1 (DEBUG_SEPARATE_PAIRS): triangle/bin pairs as separate
        key and value arrays even where one word would hold a pair."""
        _check(self._lib.fdzb_ctx_set_debug(self._h, int(flags)))

    def set_profiling(self, enable) -> None:
        """Per-stage CUDA-event timing, reported in stats()['stage_ms'], and the
        occlusion kernel's work counters (True or PROFILE_ALL); PROFILE_STAGES:
        the timing alone, with the unprofiled kernels."""
        _check(self._lib.fdzb_ctx_set_profiling(self._h, _profile_mode(enable)))

    def set_tri_order(self, order: int) -> None:
        """TRI_ORDER_REFERENCE (the reference's per-bin order) or TRI_ORDER_COVERAGE."""
        _check(self._lib.fdzb_ctx_set_tri_order(self._h, int(order)))

    def set_graph(self, enable: bool) -> None:
        """Capture launches in a CUDA graph and replay it while the shape holds (default on)."""
        _check(self._lib.fdzb_ctx_set_graph(self._h, int(bool(enable))))

    def set_launch_epoch(self, value: int) -> None:
        """Testing aid: moves the launch number that tags the look-back words."""
        _check(self._lib.fdzb_ctx_set_launch_epoch(self._h, int(value)))

    def launch_epoch(self) -> int:
        """The launch number after the pending launch (testing aid)."""
        out = ctypes.c_uint32(0)
        _check(self._lib.fdzb_ctx_get_launch_epoch(self._h, ctypes.byref(out)))
        return int(out.value)

    def set_occlusion_shape(self, chunk: int, item: int) -> None:
        """Triangles staged per chunk (OCC_CHUNKS) and samples per warp item
        (OCC_ITEMS); results are identical for every shape."""
        _check(self._lib.fdzb_ctx_set_occlusion_shape(self._h, int(chunk), int(item)))

    def set_open_box(self, mode: int) -> None:
        """OPEN_BOX_OFF, OPEN_BOX_ON or OPEN_BOX_AUTO (default); results are identical."""
        _check(self._lib.fdzb_ctx_set_open_box(self._h, int(mode)))

    def set_occlusion_schedule(self, schedule: int) -> None:
        """OCC_LANE_PER_SAMPLE (default) or OCC_LANE_PER_PAIR; results are identical."""
        _check(self._lib.fdzb_ctx_set_occlusion_schedule(self._h, int(schedule)))

    def set_pair_capacity_limit(self, pairs: int) -> None:
        """Largest pair buffer; frames with more pairs run in triangle passes."""
        _check(self._lib.fdzb_ctx_set_pair_capacity_limit(self._h, int(pairs)))

    def add_model(self, vtx, n_vtx: int, stride_bytes: int, idx, n_tri: int, name: str = "") -> None:
        self._keep += [vtx, idx]
        _check(self._lib.fdzb_ctx_add_model(self._h, _ptr(vtx), n_vtx, stride_bytes, _ptr(idx), n_tri,
                                             name.encode()))

    def set_sample_buffers(self, pos, nrm) -> None:
        self._keep += [pos, nrm]
        _check(self._lib.fdzb_ctx_set_sample_buffers(self._h, _ptr(pos), _ptr(nrm)))

    def set_output_buffer(self, shadow, masks=None) -> None:
        self._keep += [shadow, masks]
        _check(self._lib.fdzb_ctx_set_output_buffer(self._h, _ptr(shadow), _ptr(masks)))

    def set_bin_num(self, n: int) -> None:
        _check(self._lib.fdzb_ctx_set_bin_num(self._h, n))

    def set_view(self, w: int, h: int) -> None:
        _check(self._lib.fdzb_ctx_set_view(self._h, w, h))

    def set_scenes_esp(self, esp: float) -> None:
        _check(self._lib.fdzb_ctx_set_scenes_esp(self._h, esp))

    def set_scene_params(self, max_tri: int, max_vert: int) -> None:
        _check(self._lib.fdzb_ctx_set_scene_params(self._h, max_tri, max_vert))

    def set_area_light(self, light) -> None:
        d = AreaLightDesc.from_light(light) if not isinstance(light, AreaLightDesc) else light
        _check(self._lib.fdzb_ctx_set_area_light(self._h, ctypes.byref(d)))

    def move_model(self, m) -> None:
        arr = (ctypes.c_float * 16)(*[float(v) for v in np.asarray(m, dtype=np.float32).reshape(16)])
        _check(self._lib.fdzb_ctx_move_model(self._h, arr))

    def set_depth_plane(self, enable: bool) -> None:
        """fdzb_ctx_set_depth_plane: also test each triangle's own plane."""
        _check(self._lib.fdzb_ctx_set_depth_plane(self._h, int(bool(enable))))

    def set_shadow_method(self, method: int) -> None:
        """SHADOW_EDGE_MASKS (default) or SHADOW_RAY_CAST (the reference's REF_CAL checker)."""
        _check(self._lib.fdzb_ctx_set_shadow_method(self._h, int(method)))

    def set_model_transform(self, m) -> None:
        """Column-major 4x4 applied to the vertices as they are read (None clears)."""
        if m is None:
            _check(self._lib.fdzb_ctx_set_model_transform(self._h, None))
            return
        arr = (ctypes.c_float * 16)(*[float(v) for v in np.asarray(m, dtype=np.float32).reshape(16)])
        _check(self._lib.fdzb_ctx_set_model_transform(self._h, arr))

    def launch(self) -> float:
        ms = ctypes.c_float()
        _check(self._lib.fdzb_ctx_launch(self._h, ctypes.byref(ms)))
        return float(ms.value)

    def launch_async(self) -> None:
        _check(self._lib.fdzb_ctx_launch_async(self._h))

    def sync(self) -> None:
        _check(self._lib.fdzb_ctx_sync(self._h))

    def stats(self) -> dict:
        st = FrameStats()
        _check(self._lib.fdzb_ctx_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def export(self, name: str, count: int) -> np.ndarray:
        what, dt = ARRAYS[name]
        out = np.empty(count, dtype=dt)
        if count:
            _check(self._lib.fdzb_ctx_export(self._h, what, out.ctypes.data, out.nbytes))
        return out


# ---- FD:: namespace mirror (process-wide context) --------------------------

_fd_keep: list = []


def FDinit() -> None:
    """FD::FDinit (FS/api.h:15)."""
    _fd_keep.clear()
    _check(load().fdzb_init())


def FDsetBackfaceCull(enable: bool) -> None:
    _check(load().fdzb_set_backface_cull(int(bool(enable))))


def FDaddModel(vtx, idx, vertex_size_bytes: int, model_name: str = "", n_vtx: Optional[int] = None,
               n_tri: Optional[int] = None) -> None:
    """FD::FDaddModel (FS/api.h:21): vtx/idx are device tensors (VBO/IBO)."""
    _fd_keep.extend([vtx, idx])
    if n_vtx is None:
        n_vtx = vtx.numel() * vtx.element_size() // vertex_size_bytes
    if n_tri is None:
        n_tri = idx.numel() // 3
    _check(load().fdzb_add_model(_ptr(vtx), n_vtx, vertex_size_bytes, _ptr(idx), n_tri, model_name.encode()))


def FDsetSampleGLTex(pos, nrm) -> None:
    """FD::FDsetSampleGLTex (FS/api.h:24): device float4 position / normal images."""
    _fd_keep.extend([pos, nrm])
    _check(load().fdzb_set_sample_buffers(_ptr(pos), _ptr(nrm)))


def FDsetOutputGLBuffer(shadow, masks=None) -> None:
    """FD::FDsetOutputGLBuffer (FS/api.h:27)."""
    _fd_keep.extend([shadow, masks])
    _check(load().fdzb_set_output_buffer(_ptr(shadow), _ptr(masks)))


def FDregisterGLres() -> None:
    _check(load().fdzb_register_resources())


def FDunregisterGLres() -> None:
    _check(load().fdzb_unregister_resources())


def FDsetBinNum(bin_num: int) -> int:
    """FD::FDsetBinNum (FS/api.h:36): 0 on success, -1 if rejected."""
    rc = load().fdzb_set_bin_num(bin_num)
    return 0 if rc == FDZB_OK else -1


def FDsetView(w: int, h: int) -> None:
    _check(load().fdzb_set_view(w, h))


def FDsetScenesEsp(esp: float) -> None:
    _check(load().fdzb_set_scenes_esp(esp))


def FDsetSceneParams(max_tri: int, max_vert: int) -> None:
    _check(load().fdzb_set_scene_params(max_tri, max_vert))


def FDsetAreaLight(light) -> None:
    d = AreaLightDesc.from_light(light) if not isinstance(light, AreaLightDesc) else light
    _check(load().fdzb_set_area_light(ctypes.byref(d)))


def FDLaunch() -> float:
    """FD::FDLaunch (FS/api.h:52): frame GPU time in ms."""
    ms = float(load().fdzb_launch())
    if ms < 0:
        _check(int(ms))
    return ms


def moveModel(m) -> None:
    arr = (ctypes.c_float * 16)(*[float(v) for v in np.asarray(m, dtype=np.float32).reshape(16)])
    _check(load().fdzb_move_model(arr))


def upload_scene(scene, device: str = "cuda"):
    """Device tensors of a scenes.Scene: (pos, nrm, vtx, idx)."""
    import torch
    pos = torch.from_numpy(scene.pos).to(device)
    nrm = torch.from_numpy(scene.nrm).to(device)
    vtx = torch.from_numpy(scene.vtx).to(device)
    idx = torch.from_numpy(scene.idx).to(device)
    return pos, nrm, vtx, idx


DEBUG_COPIES, DEBUG_SEPARATE_PAIRS = 1, 2


def context_for_scene(scene, device: str = "cuda", masks: bool = True, debug: bool = False,
                      tri_order: Optional[int] = None, separate_pairs: bool = False):
    """A Context with the scene's buffers uploaded and outputs allocated.
    Returns (ctx, tensors dict)."""
    import torch
    pos, nrm, vtx, idx = upload_scene(scene, device)
    shadow = torch.empty(scene.S, dtype=torch.float32, device=device)
    mk = (torch.empty(scene.S * mask_words(scene.light.n, scene.light.cols), dtype=torch.int32, device=device)
          if masks else None)
    ctx = Context()
    if debug or separate_pairs:
        ctx.set_debug((DEBUG_COPIES if debug else 0) | (DEBUG_SEPARATE_PAIRS if separate_pairs else 0))
    if tri_order is not None:
        ctx.set_tri_order(tri_order)
    ctx.set_view(scene.W, scene.H)
    ctx.set_bin_num(scene.bins)
    ctx.set_scenes_esp(scene.esp)
    ctx.set_backface_cull(scene.cull)
    ctx.add_model(vtx, scene.V, 16, idx, scene.T, scene.name)
    ctx.set_sample_buffers(pos, nrm)
    ctx.set_output_buffer(shadow, mk)
    ctx.set_area_light(scene.light)
    if getattr(scene, "depth_plane", False):
        ctx.set_depth_plane(True)
    return ctx, dict(pos=pos, nrm=nrm, vtx=vtx, idx=idx, shadow=shadow, masks=mk)


# ---- batches ---------------------------------------------------------------


def _mat16(m):
    if m is None:
        return None
    return (ctypes.c_float * 16)(*[float(v) for v in np.asarray(m, dtype=np.float32).reshape(16)])


def frame_desc(pos, nrm, W: int, H: int, vtx, n_vtx: int, idx, n_tri: int, light, shadow, masks=None,
               bins: int = 0, cull: bool = False, esp: float = 1e-3, stride_bytes: int = 16,
               model_transform=None) -> FrameDesc:
    """An fdzb_frame_desc from device tensors (or int pointers); bins 0 = autotuned;
    model_transform: optional column-major 4x4 applied to the vertices as read."""
    d = FrameDesc()
    d._m = _mat16(model_transform)   # keeps the array alive with the descriptor
    d.model_transform = ctypes.cast(d._m, ctypes.POINTER(ctypes.c_float)) if d._m is not None else None
    d.d_pos, d.d_nrm = _ptr(pos), _ptr(nrm)
    d.W, d.H = W, H
    d.d_vtx, d.n_vtx, d.vtx_stride_bytes = _ptr(vtx), n_vtx, stride_bytes
    d.d_idx, d.n_tri = _ptr(idx), n_tri
    d.light = AreaLightDesc.from_light(light) if not isinstance(light, AreaLightDesc) else light
    d.bins, d.cull, d.esp = bins, int(bool(cull)), esp
    d.d_shadow, d.d_masks = _ptr(shadow), _ptr(masks)
    return d


class Batch:
    """Many independent frames per launch (the fdzb_batch_* API)."""

    def __init__(self, device: int = -1):
        self._lib = load()
        h = ctypes.c_void_p()
        _check(self._lib.fdzb_batch_create(ctypes.byref(h), device))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fdzb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _array(frames):
        arr = (FrameDesc * len(frames))(*frames)
        return arr

    def set_graph(self, enable: bool) -> None:
        _check(self._lib.fdzb_batch_set_graph(self._h, int(bool(enable))))

    def set_profiling(self, enable) -> None:
        """As Context.set_profiling."""
        _check(self._lib.fdzb_batch_set_profiling(self._h, _profile_mode(enable)))

    def set_tri_order(self, order: int) -> None:
        _check(self._lib.fdzb_batch_set_tri_order(self._h, int(order)))

    def set_occlusion_schedule(self, schedule: int) -> None:
        _check(self._lib.fdzb_batch_set_occlusion_schedule(self._h, int(schedule)))

    def set_depth_plane(self, enable: bool) -> None:
        _check(self._lib.fdzb_batch_set_depth_plane(self._h, int(bool(enable))))

    def set_stream(self, stream) -> None:
        _check(self._lib.fdzb_batch_set_stream(self._h, ctypes.c_void_p(stream)))

    def launch(self, frames) -> float:
        arr = self._array(frames)
        ms = ctypes.c_float()
        _check(self._lib.fdzb_batch_launch(self._h, arr, len(frames), ctypes.byref(ms)))
        return float(ms.value)

    def launch_async(self, frames) -> None:
        self._pending = self._array(frames)
        _check(self._lib.fdzb_batch_launch_async(self._h, self._pending, len(frames)))

    def sync(self) -> float:
        ms = ctypes.c_float()
        _check(self._lib.fdzb_batch_sync(self._h, ctypes.byref(ms)))
        return float(ms.value)

    def autotune(self, frames, scratch) -> None:
        """scratch: device float tensor with at least max(W*H) elements."""
        arr = self._array(frames)
        _check(self._lib.fdzb_batch_autotune(self._h, arr, len(frames), _ptr(scratch), scratch.numel()))

    def frame_stats(self, i: int) -> dict:
        st = FrameStats()
        _check(self._lib.fdzb_batch_get_frame_stats(self._h, i, ctypes.byref(st)))
        return st.as_dict()

    def stats(self) -> dict:
        st = BatchStats()
        _check(self._lib.fdzb_batch_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def frame_shape(self, i: int) -> tuple:
        """(bins per side, staging chunk, samples per item) of frame i of the last launch."""
        b, c, it = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        _check(self._lib.fdzb_batch_frame_shape(self._h, int(i), ctypes.byref(b), ctypes.byref(c),
                                                ctypes.byref(it)))
        return b.value, c.value, it.value

    def set_occlusion_shape(self, chunk: int = 0, item: int = 0) -> None:
        """One occlusion shape for every frame of later launches (0, 0: tuned or default)."""
        _check(self._lib.fdzb_batch_set_occlusion_shape(self._h, int(chunk), int(item)))

    def set_open_box(self, mode: int) -> None:
        """OPEN_BOX_OFF, OPEN_BOX_ON or OPEN_BOX_AUTO (default) for later launches."""
        _check(self._lib.fdzb_batch_set_open_box(self._h, int(mode)))

    def frame_bins(self, i: int) -> int:
        rc = self._lib.fdzb_batch_frame_bins(self._h, i)
        if rc <= 0:
            _check(rc if rc < 0 else -1)
        return rc


# ---- serving ---------------------------------------------------------------


def request(scene_id: int, pos, nrm, W: int, H: int, light, shadow, masks=None, bins: int = 0,
            model_transform=None) -> Request:
    """An fdzb_request from device tensors (or int pointers)."""
    r = Request()
    r._m = _mat16(model_transform)
    r.model_transform = ctypes.cast(r._m, ctypes.POINTER(ctypes.c_float)) if r._m is not None else None
    r.scene_id, r.W, r.H, r.bins = scene_id, W, H, bins
    r.d_pos, r.d_nrm = _ptr(pos), _ptr(nrm)
    r.light = AreaLightDesc.from_light(light) if not isinstance(light, AreaLightDesc) else light
    r.d_shadow, r.d_masks = _ptr(shadow), _ptr(masks)
    return r


class Server:
    """Request loop with continuous batching (the fdzb_serve_* API)."""

    def __init__(self, slots: int = 2, max_batch_frames: int = 16, max_batch_samples: int = 16 << 20,
                 memory_budget_bytes: int = 150 * 10**9, use_graphs: bool = False, device: int = -1,
                 max_batch_triangles: int = 4 << 20):
        self._lib = load()
        cfg = ServeConfig()
        self._lib.fdzb_serve_default_config(ctypes.byref(cfg))
        cfg.device, cfg.slots, cfg.max_batch_frames = device, slots, max_batch_frames
        cfg.max_batch_samples, cfg.memory_budget_bytes = max_batch_samples, memory_budget_bytes
        cfg.use_graphs = int(bool(use_graphs))
        cfg.max_batch_triangles = max_batch_triangles
        h = ctypes.c_void_p()
        _check(self._lib.fdzb_serve_create(ctypes.byref(h), ctypes.byref(cfg)))
        self._h = h
        self._keep = []

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fdzb_serve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, vtx, n_vtx: int, idx, n_tri: int, cull: bool = False, esp: float = 1e-3,
                  stride_bytes: int = 16) -> int:
        self._keep += [vtx, idx]
        sid = ctypes.c_int32()
        _check(self._lib.fdzb_serve_add_scene(self._h, _ptr(vtx), n_vtx, stride_bytes, _ptr(idx), n_tri,
                                              int(bool(cull)), esp, ctypes.byref(sid)))
        return int(sid.value)

    def submit(self, req: Request) -> int:
        t = ctypes.c_uint64()
        _check(self._lib.fdzb_serve_submit(self._h, ctypes.byref(req), ctypes.byref(t)))
        return int(t.value)

    def poll(self, ticket: int):
        out = RequestResult()
        rc = self._lib.fdzb_serve_poll(self._h, ticket, ctypes.byref(out))
        if rc < 0:
            _check(rc)
        return out.as_dict() if rc == 1 else None

    def wait(self, ticket: int, timeout_ms: int = -1):
        out = RequestResult()
        rc = self._lib.fdzb_serve_wait(self._h, ticket, timeout_ms, ctypes.byref(out))
        if rc < 0:
            _check(rc)
        return out.as_dict() if rc == 1 else None

    def drain(self, timeout_ms: int = -1) -> bool:
        rc = self._lib.fdzb_serve_drain(self._h, timeout_ms)
        if rc < 0:
            _check(rc)
        return rc == 1

    def autotune(self, reqs, scratch) -> None:
        arr = (Request * len(reqs))(*reqs)
        _check(self._lib.fdzb_serve_autotune(self._h, arr, len(reqs), _ptr(scratch), scratch.numel()))

    def stats(self) -> dict:
        st = ServeStats()
        _check(self._lib.fdzb_serve_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def reset_stats(self) -> None:
        _check(self._lib.fdzb_serve_reset_stats(self._h))

    def worker_error(self) -> str:
        return self._lib.fdzb_serve_last_worker_error(self._h).decode()


# ---- shading pass -----------------------------------------------------------


def light_sample_positions(light) -> np.ndarray:
    """Light-sample positions [H*W, 3] in the reference's numbering (i*W + j)."""
    d = AreaLightDesc.from_light(light) if not isinstance(light, AreaLightDesc) else light
    out = np.zeros(3 * d.lightResWidth * d.lightResHeight, np.float32)
    _check(load().fdzb_light_sample_positions(ctypes.byref(d), out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
    return out.reshape(-1, 3)


def shade(W: int, H: int, g0, g1, g2, g3, shadow, rgba, camera_pos, La, Ld, Ls, light_samples, stream=None) -> None:
    """fdzb_shade on device tensors; light_samples: device float tensor [n, 3]."""
    d = ShadeDesc()
    d.W, d.H = W, H
    d.d_g0, d.d_g1, d.d_g2, d.d_g3 = _ptr(g0), _ptr(g1), _ptr(g2), _ptr(g3)
    d.d_shadow, d.d_rgba = _ptr(shadow), _ptr(rgba)
    d.camera_pos[:] = [float(v) for v in camera_pos]
    d.La[:] = [float(v) for v in La]
    d.Ld[:] = [float(v) for v in Ld]
    d.Ls[:] = [float(v) for v in Ls]
    d.n_light_samples = int(light_samples.shape[0])
    d.d_light_samples = _ptr(light_samples)
    _check(load().fdzb_shade(ctypes.byref(d), ctypes.c_void_p(stream)))


# ---- G-buffer rasteriser ---------------------------------------------------


def _mat16_list(m) -> list:
    return [float(v) for v in np.asarray(m, dtype=np.float32).reshape(-1, order="F")] if np.asarray(m).ndim == 2 \
        else [float(v) for v in np.asarray(m, dtype=np.float32).reshape(16)]


def raster_desc(vtx, n_vtx: int, idx, n_tri: int, materials, n_materials: int, model, view_proj, W: int, H: int,
                g0, g1, g2=None, g3=None, depth=None, clear: bool = True, tri_material=None,
                stride_bytes: int = 32, pos_offset: int = 0, nrm_offset: int = 5) -> RasterDesc:
    """fdzb_raster_desc from device tensors (or pointers).  model / view_proj:
    4x4 matrices (numpy, mathematical row/column convention; stored column-major)
    or 16 floats already column-major."""
    d = RasterDesc()
    d.d_vtx, d.n_vtx, d.vtx_stride_bytes = _ptr(vtx), int(n_vtx), int(stride_bytes)
    d.pos_offset, d.nrm_offset = int(pos_offset), int(nrm_offset)
    d.d_idx, d.n_tri = _ptr(idx), int(n_tri)
    d.d_tri_material = _ptr(tri_material)
    d.d_materials, d.n_materials = _ptr(materials), int(n_materials)
    d.model[:] = _mat16_list(model)
    d.view_proj[:] = _mat16_list(view_proj)
    d.W, d.H, d.clear = int(W), int(H), int(bool(clear))
    d.d_g0, d.d_g1, d.d_g2, d.d_g3 = _ptr(g0), _ptr(g1), _ptr(g2), _ptr(g3)
    d.d_depth = _ptr(depth)
    return d


class Raster:
    """fdzb_raster_*: the G-buffer rasteriser (the app's GL pass 0)."""

    def __init__(self, device: int = -1):
        self._lib = load()
        h = ctypes.c_void_p()
        _check(self._lib.fdzb_raster_create(ctypes.byref(h), int(device)))
        self._h = h

    def set_stream(self, stream) -> None:
        _check(self._lib.fdzb_raster_set_stream(self._h, ctypes.c_void_p(stream)))

    def draw(self, desc: RasterDesc) -> None:
        _check(self._lib.fdzb_raster_draw(self._h, ctypes.byref(desc)))

    def sync(self) -> None:
        _check(self._lib.fdzb_raster_sync(self._h))

    def stats(self) -> dict:
        st = RasterStats()
        _check(self._lib.fdzb_raster_get_stats(self._h, ctypes.byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_ if name != "pad"}

    def close(self) -> None:
        if self._h:
            self._lib.fdzb_raster_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
