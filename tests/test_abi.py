"""The C ABI: libfdzb.so loads without a GPU, exports every symbol declared in
include/fdzb.h, computes the host light setup bit-identically to the oracle,
and reports errors as status codes (no GPU work is issued here)."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "fdzb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fdzb_\w+)\s*\(", src)))


def test_every_declared_symbol_is_exported(fdzb):
    lib = fdzb.load()
    names = _declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(fdzb.EXPORTED)


def test_version_and_error_string(fdzb):
    lib = fdzb.load()
    assert b"sm_100a" in lib.fdzb_version()
    assert isinstance(lib.fdzb_last_error(), bytes)


@pytest.mark.parametrize("n", [1, 4, 8, 16, 32])
@pytest.mark.parametrize("radius", [0.5, 1.0, 2.0])
def test_light_setup_matches_oracle(fdzb, scenes, n, radius):
    light = scenes.Light(right_radius=radius, top_radius=radius * 0.75, n=n,
                         position=(0.3, -0.2, 6.0), view_dir=(0.05, 0.02, -1.0), up_dir=(0.0, 1.0, 0.1))
    a = fdzb.light_setup(light)
    b = oracle.light_setup(light)
    assert np.array_equal(a["mat"].view(np.uint32), np.array(b.mat, np.float32).view(np.uint32))
    assert np.array_equal(a["RF"].view(np.uint32), np.array(b.RF, np.float32).view(np.uint32))
    corners = np.array([b.upRight, b.upLeft, b.downLeft, b.downRight], np.float32)
    assert np.array_equal(a["corners"], corners)
    assert np.array_equal(a["deltas"], np.array([b.x_delt, b.y_delt], np.float32))


@pytest.mark.parametrize("w,h", [(8, 16), (64, 3), (33, 64), (1, 7)])
def test_rectangular_light_setup_matches_oracle(fdzb, scenes, w, h):
    light = scenes.Light(right_radius=1.5, top_radius=0.5, n=w, nh=h, position=(0.1, 0.4, 6.0))
    a = fdzb.light_setup(light)
    b = oracle.light_setup(light)
    assert b.resW == w and b.resH == h
    assert b.fullRows == (1 << w) - 1 and b.fullCols == (1 << h) - 1 or w == 64 or h == 64
    assert np.array_equal(a["mat"].view(np.uint32), np.array(b.mat, np.float32).view(np.uint32))
    assert np.array_equal(a["deltas"], np.array([b.x_delt, b.y_delt], np.float32))
    corners = np.array([b.upRight, b.upLeft, b.downLeft, b.downRight], np.float32)
    assert np.array_equal(a["corners"], corners)


def test_light_setup_canonical_values(fdzb, scenes):
    """Light at (0,0,6) facing -z, up +y, 2x2, N=8: right=+x, top=+y, steps of
    -2r/N along each, corners at +-r(N-1)/N, perspective 1/tan(60 rad)."""
    light = scenes.Light(n=8)
    a = fdzb.light_setup(light)
    xd, yd = a["deltas"]
    assert np.allclose(xd, [-0.25, 0, 0]) and np.allclose(yd, [0, -0.25, 0])
    ur, ul, dl, dr = a["corners"]
    assert np.allclose(ur, [0.875, 0.875, 6]) and np.allclose(dl, [-0.875, -0.875, 6])
    p00 = 0.2 / (2 * np.float32(np.tan(60.0)) * np.float32(0.1))
    assert abs(a["RF"][0] - 1.0 * 2 * 0.875 * p00 * 0.5) < 1e-5
    # the projection's depth row: w = 6 - z at x = y = 0 (lookAt along -z)
    M = a["mat"]
    assert abs(M[3] * 0 + M[7] * 0 + M[11] * 1.0 + M[15] - (6 - 1.0 - 0.0)) < 1e-5


def test_projection_uses_correctly_rounded_tan(fdzb, scenes):
    """GLM 0.9.8 takes fovy in radians: range = tan(120/2 rad) * 0.1.  The light
    setup uses tan(60) correctly rounded to binary32 (0.32004037), not the C
    runtime's tanf, whose last bit differs between runtimes (glibc: 0.3200404)."""
    exact = np.tan(np.float64(60.0))
    cr = np.float32(exact)
    nb = [np.nextafter(cr, np.float32(-1)), np.nextafter(cr, np.float32(1))]
    assert all(abs(np.float64(cr) - exact) < abs(np.float64(c) - exact) for c in nb)
    rng = np.float32(cr * np.float32(0.1))
    p00 = np.float32(np.float32(0.2) / np.float32(rng + rng))
    light = scenes.Light(n=8)
    rf = np.float32(np.float32(np.float32(np.float32(1.0) * np.float32(2.0)) * np.float32(0.875)) * p00)
    rf = np.float32(rf * np.float32(0.5))
    assert fdzb.light_setup(light)["RF"][0] == rf
    assert np.float32(oracle.light_setup(light).RF[0]) == rf


def test_calls_without_context_fail_cleanly(fdzb):
    lib = fdzb.load()
    assert lib.fdzb_ctx_set_view(None, 4, 4) == -3
    assert lib.fdzb_ctx_launch(None, None) == -3
    assert lib.fdzb_ctx_export(None, 0, None, 0) == -3


def test_context_creation_without_gpu_is_an_error_not_a_crash(fdzb):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(fdzb.FdzbError):
        fdzb.Context()


def test_batch_api_rejects_null_handles(fdzb):
    lib = fdzb.load()
    assert lib.fdzb_batch_launch(None, None, 0, None) == -3
    assert lib.fdzb_batch_sync(None, None) == -3
    assert lib.fdzb_batch_get_stats(None, None) == -3
    assert lib.fdzb_batch_frame_bins(None, 0) == -3
    assert lib.fdzb_batch_autotune(None, None, 0, None, 0) == -3
    assert lib.fdzb_batch_destroy(None) == 0
    assert lib.fdzb_ctx_set_graph(None, 1) == -3


def test_batch_struct_layouts(fdzb):
    """ctypes mirrors match the C layouts (the library static_asserts the same sizes)."""
    import ctypes
    assert ctypes.sizeof(fdzb.AreaLightDesc) == 52
    assert ctypes.sizeof(fdzb.FrameStats) == 184
    assert ctypes.sizeof(fdzb.FrameDesc) == 152
    assert ctypes.sizeof(fdzb.BatchStats) == 232
    assert ctypes.sizeof(fdzb.RasterDesc) == 240
    assert ctypes.sizeof(fdzb.RasterStats) == 64
    assert fdzb.FrameDesc.light.offset == 64 and fdzb.FrameDesc.d_shadow.offset == 128


def test_noalloc_sort_rejects_overlapping_buffers(fdzb):
    """The allocation-free sort refuses outputs that share bytes with an input,
    the other output or the status word; the check runs before any CUDA call,
    so plain addresses suffice here."""
    lib = fdzb.load()
    fn = lib.fdzb_sort_pairs_noalloc
    fn.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    n = 16                       # 64 bytes per array
    ki, vi, ko, vo = 0x100000, 0x200000, 0x300000, 0x400000
    bad = [(ki, vi, ki + 32, vo, None),          # keys_out overlaps keys_in
           (ki, vi, vi, vo, None),               # keys_out == vals_in
           (ki, vi, ko, ki, None),               # vals_out == keys_in
           (ki, vi, ko, vi + 60, None),          # vals_out overlaps the end of vals_in
           (ki, vi, ko, ko + 4, None),           # outputs overlap each other
           (ki, vi, ko, vo, vo + 8)]             # status word inside vals_out
    for a, b, c, d, st in bad:
        assert fn(a, b, c, d, n, 64, None, st) == -1
        assert b"overlap" in lib.fdzb_last_error()


def test_occlusion_shape_arguments_are_checked(fdzb):
    """Shapes outside {8, 16, 32} x {32, 64, 128} are refused before any GPU work."""
    lib = fdzb.load()
    assert lib.fdzb_ctx_set_occlusion_shape(None, 32, 32) == -3        # no context
    assert lib.fdzb_batch_set_occlusion_shape(None, 16, 64) == -3


def test_open_box_mode_arguments_are_checked(fdzb):
    lib = fdzb.load()
    assert lib.fdzb_ctx_set_open_box(None, fdzb.OPEN_BOX_AUTO) == -3
    assert lib.fdzb_batch_set_open_box(None, fdzb.OPEN_BOX_ON) == -3
