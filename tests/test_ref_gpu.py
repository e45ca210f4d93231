"""The reference's own GPU code, run on the same B200, against the product.

oracle/_ref/libref4dzb_gpu*.so is 4DZB's soft-shadow sources (FS/api.cpp and
K/*.inl) compiled for sm_100a with --fmad=false by
oracle/ref_gpu/build_ref_gpu.py, at the reference's own 16 x 16 bins and with
its compile-time bin constant set to 32 x 32 and 128 x 128; FDLaunch runs its
own kernels, Thrust sorts and host sequencing.  At the same bins the product's
shadows must equal the reference's bit for bit, and the light-plane setup and
the binning counts must agree; the reference's per-sample kernel also hands
out its final light rows (a harness dump after its shadow store), which must
equal the product's masks for every binned sample -- in the reference's
per-bin triangle order and in the coverage order the product runs by default
(the small frame at its 32 x 32 bins, the HD frame at its 128 x 128).  Every scene passes the CPU preflight (keys inside
the bin grid, pairs inside the reference's pair buffers) before it reaches
the GPU.  The --fmad=true build (the reference project's default) is run too:
its shadows differ from the exact ones only where a fused multiply-add moved a
light-grid edge test across zero.
"""
import dataclasses

import numpy as np
import pytest

from oracle import ref_gpu

pytestmark = pytest.mark.gpu

needs_lib = pytest.mark.skipif(not ref_gpu.available(), reason="reference GPU harness not built (oracle/_ref)")


def _product(fdzb, scene, bins=ref_gpu.REF_BINS, tri_order=0):
    sb = dataclasses.replace(scene, bins=bins)
    ctx, t = fdzb.context_for_scene(sb, masks=True, tri_order=tri_order)
    ctx.launch()
    st = ctx.stats()
    sh = t["shadow"].cpu().numpy().copy()
    mk = t["masks"].cpu().numpy().view(np.uint32).reshape(scene.S, -1).copy()
    ctx.close()
    return sh, mk, st


def _rows_of(words, n):
    """Light rows of packed masks (bit r*n + c is row r, column c) as uint32[S, n]."""
    w = np.concatenate([words, np.zeros((words.shape[0], 1), np.uint32)], axis=1).astype(np.uint64)
    rows = np.empty((words.shape[0], n), np.uint32)
    full = np.uint64((1 << n) - 1)
    for r in range(n):
        b = r * n
        v = (w[:, b >> 5] | (w[:, (b >> 5) + 1] << np.uint64(32))) >> np.uint64(b & 31)
        rows[:, r] = (v & full).astype(np.uint32)
    return rows


def _check(fdzb, scene, ref, bins=ref_gpu.REF_BINS, tri_order=0):
    sh, mk, st = _product(fdzb, scene, bins, tri_order)
    assert ref["rows_beyond_n"] == 0
    # no pair written past its triangle's count (else the reference's own lists race)
    assert ref["q2_events"] == 0
    bad = np.flatnonzero(sh.view(np.uint32) != ref["shadow"].view(np.uint32))
    assert bad.size == 0, f"{bad.size} of {scene.S} shadows differ, first {bad[:5].tolist()}"
    # masks: the reference's per-sample kernel ran for every binned sample;
    # its rows (all 32 bits) equal the product's packed rows
    n = scene.light.n
    wr = ref["mask_written"]
    assert int(wr.sum()) == ref["valid_samples"] == st["valid_samples"]
    got = _rows_of(mk[wr], n)
    exp = ref["mask_rows"][wr]
    badm = np.flatnonzero((got != exp).any(axis=1))
    assert badm.size == 0, f"{badm.size} of {int(wr.sum())} sample masks differ, first {np.flatnonzero(wr)[badm[:5]].tolist()}"
    assert st["valid_samples"] == ref["valid_samples"]
    assert st["valid_triangles"] == ref["valid_tris"]
    assert st["num_pairs"] == ref["num_pairs"]
    f32 = np.float32
    assert np.array_equal(f32(st["sub"]), f32(ref["sub"]))
    assert np.array_equal(f32(st["lp_begin"]), f32(ref["lp_begin"]))
    assert np.array_equal(f32(st["lp_end"]), f32(ref["lp_end"]))
    assert np.array_equal(f32(st["lp_factor"]), f32(ref["lp_factor"]))
    sa, ma = ref["sample_aabb"], ref["model_aabb"]
    assert np.array_equal(f32(st["sample_aabb"]), f32(np.r_[sa[0:3], sa[4:7]]))
    assert np.array_equal(f32(st["model_aabb"]), f32(np.r_[ma[0:3], ma[4:7]]))
    return sh


@needs_lib
@pytest.mark.parametrize("cull", [False, True])
def test_small_frame_equals_reference_on_gpu(cuda_ok, fdzb, scenes, cull):
    scene = scenes.preset("small", cull=cull)
    ref = ref_gpu.run(scene, fmad=False, masks=True)
    _check(fdzb, scene, ref)


@needs_lib
def test_odd_sizes_equal_reference_on_gpu(cuda_ok, fdzb, scenes):
    # non-power-of-two width (the reference's padded output rows), N = 5 and 32
    for W, H, T, n, seed in ((301, 77, 700, 5, 11), (200, 150, 1500, 32, 12)):
        scene = scenes.make_scene(W, H, T, n=n, bins=16, seed=seed, cull=True)
        ref = ref_gpu.run(scene, fmad=False, masks=True)
        _check(fdzb, scene, ref)


@needs_lib
def test_hd_frame_equals_reference_on_gpu(cuda_ok, fdzb, scenes):
    scene = scenes.preset("hd")
    ref = ref_gpu.run(scene, fmad=False, masks=True)
    sh = _check(fdzb, scene, ref)
    assert 0.0 < float(sh.mean()) <= 1.0


@needs_lib
def test_large_frame_equals_reference_on_gpu(cuda_ok, fdzb, scenes):
    # 3840 x 2160 samples, 2M triangles, 32 x 32 light (full 32-bit rows)
    scene = scenes.preset("large")
    ref_gpu.preflight(scene, occ_stride=256)
    ref = ref_gpu.run(scene, fmad=False, checked=True, masks=True)
    _check(fdzb, scene, ref)


def _needs(bins, fmad=False):
    if not ref_gpu.available(fmad=fmad, bins=bins):
        pytest.skip(f"reference GPU harness at {bins} x {bins} bins not built (oracle/_ref)")


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("cull", [False, True])
def test_small_frame_at_32_bins_equals_reference(cuda_ok, fdzb, scenes, cull, order):
    """The small workload at its own 32 x 32 bins, both triangle orders."""
    _needs(32)
    scene = scenes.preset("small", cull=cull)
    assert scene.bins == 32
    ref = ref_gpu.run(scene, fmad=False, masks=True, bins=32)
    assert ref["bins"] == 32 and ref["num_bins"] == 32 * 32
    _check(fdzb, scene, ref, bins=32, tri_order=order)


@pytest.mark.parametrize("bins", [32, 128])
def test_odd_sizes_at_other_bins_equal_reference(cuda_ok, fdzb, scenes, bins):
    """Odd views at 32^2 and 128^2 bins.  Where the reference's write kernel
    puts a pair past its triangle's counted slots (its count and write kernels
    test different AABBs, K/Step4_RasterizeTriangleToBin.inl:74-94 vs :177-193;
    it happens when a bin's only sample defines the light plane's edge, which
    fine grids over small views make likely), the reference's lists depend on
    which of two racing writes lands; the product uses the counting test for
    both and must then equal the oracle, bit for bit."""
    import oracle
    _needs(bins)
    raced = 0
    for W, H, T, n, seed in ((301, 77, 700, 5, 11), (200, 150, 1500, 32, 12), (640, 360, 20000, 16, 13)):
        scene = scenes.make_scene(W, H, T, n=n, bins=bins, seed=seed, cull=False, sigma=0.1)
        ref = ref_gpu.run(scene, fmad=False, masks=True, bins=bins)
        if ref["q2_events"] == 0:
            _check(fdzb, scene, ref, bins=bins, tri_order=1)
            continue
        raced += 1
        sh, mk, st = _product(fdzb, scene, bins, tri_order=1)
        o = oracle.frame(scene)
        assert np.array_equal(sh.view(np.uint32), o.arrays["shadow"].astype(np.float32).view(np.uint32))
        assert np.array_equal(mk, o.arrays["masks"].reshape(scene.S, -1).astype(np.uint32))
        assert st["num_pairs"] == ref["num_pairs"]
    assert raced < 3


def test_hd_frame_at_128_bins_equals_reference_every_mask(cuda_ok, fdzb, scenes):
    """The headline configuration -- 1920 x 1080 samples, 200k triangles, a
    16 x 16 light, 128 x 128 bins, coverage order -- against the reference's
    own kernels built at 128 x 128 bins: every shadow and every binned
    sample's 16 light rows bit for bit, and the same light plane, valid counts
    and triangle/bin pair count."""
    _needs(128)
    scene = scenes.preset("hd")
    assert scene.bins == 128
    ref = ref_gpu.run(scene, fmad=False, masks=True, bins=128)
    assert ref["bins"] == 128
    sh = _check(fdzb, scene, ref, bins=128, tri_order=1)
    assert 0.0 < float(sh.mean()) <= 1.0


def test_reference_stage_times_cover_the_frame(cuda_ok, scenes):
    """The harness's per-stage events (around the five stage drivers FDLaunch
    calls) are recorded for every timed frame and add up to at most the frame."""
    _needs(32, fmad=True)
    scene = scenes.preset("small")
    r = ref_gpu.run(scene, fmad=True, bins=32, warmup=1, reps=3)
    st = r["stage_ms"]
    assert st.shape == (3, 5) and (st >= 0).all()
    assert (st.sum(axis=1) <= r["launch_ms"] * 1.001 + 1e-3).all()


# The stated rule for builds that fuse multiply-adds: at most 1e-5 of the mask
# bits may differ from the exact masks, and every differing light sample lies
# within 1e-5 light-plane units of a projected triangle edge (the FP64
# exhaustive oracle measures the distance).
FLIP_FRACTION = 1e-5
FLIP_DISTANCE = 1e-5


def _fmad_within_rule(fdzb, scene, bins):
    import oracle
    fused = ref_gpu.run(scene, fmad=True, masks=True, bins=bins)
    assert fused["rows_beyond_n"] == 0
    sh, mk, st = _product(fdzb, scene, bins, tri_order=1)
    n = scene.light.n
    wr = fused["mask_written"]
    assert int(wr.sum()) == st["valid_samples"]
    got = _rows_of(mk[wr], n)
    exp = fused["mask_rows"][wr]
    diff = got ^ exp
    flips = int(np.unpackbits(diff.view(np.uint8)).sum())
    frac = flips / (int(wr.sum()) * n * n)
    assert frac <= FLIP_FRACTION, frac
    far = 0.0
    rows = np.flatnonzero(diff.any(axis=1))
    if rows.size:
        ids = np.flatnonzero(wr)[rows].astype(np.int32)
        fr = oracle.frame(scene, setup_only=True)      # light plane only (no bins involved)
        _, dist = oracle.exhaustive_fp64(scene, fr, ids)
        bit = (diff[rows][:, :, None] >> np.arange(n, dtype=np.uint32)[None, None, :]) & 1
        flip = bit.reshape(rows.size, n * n).astype(bool)        # bit r * n + c
        far = float(dist[flip].max())
        assert far <= FLIP_DISTANCE, far
    return flips, frac, far


@needs_lib
def test_fmad_build_within_the_stated_rule_small(cuda_ok, fdzb, scenes):
    """The reference's --fmad=true build (its project's own setting) against the
    exact product at the small workload's 16 x 16 and 32 x 32 bins."""
    for bins in (16, 32):
        _needs(bins, fmad=True)
        _fmad_within_rule(fdzb, scenes.preset("small"), bins)


def test_fmad_build_within_the_stated_rule_hd(cuda_ok, fdzb, scenes):
    """The same rule on every binned sample of the HD frame at 128 x 128 bins."""
    _needs(128, fmad=True)
    _fmad_within_rule(fdzb, scenes.preset("hd"), 128)
