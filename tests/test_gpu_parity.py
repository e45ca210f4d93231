"""GPU parity: every stage of the CUDA pipeline bit-exact against the CPU oracle.

Bar: bin keys, sorted sample order, per-bin segments and statistics, triangle
footprints, per-triangle bin counts, triangle/bin pairs (before and after the
sort), per-bin triangle segments, N^2-bit masks and shadow values all equal the
FP32 restatement bit for bit (both sides compute with unfused IEEE binary32
operations in the reference's order).  In coverage order the per-bin triangle
lists are a permutation of the reference's (checked as sets); masks and shadows
must still match bit for bit.
"""
import numpy as np
import pytest

import oracle
from tests import parity

pytestmark = pytest.mark.gpu

ORDERS = [0, 1]


def _check(scene, tri_order=0, occ_stride=1, schedule=0, separate_pairs=False):
    orc = oracle.frame(scene, occ_stride=occ_stride)
    errs = parity.compare(scene, gpu=parity.run_gpu(scene, tri_order=tri_order, schedule=schedule,
                                                    separate_pairs=separate_pairs), orc=orc)
    assert not errs, "\n".join(errs)


@pytest.mark.parametrize("cull", [False, True])
@pytest.mark.parametrize("order", ORDERS)
def test_small_preset(cuda_ok, scenes, cull, order):
    _check(scenes.preset("small", cull=cull), order)


# Pairs as one word (bin << triangle bits | triangle, where they fit 32 bits:
# every scene above) and as separate key and value arrays: the same lists.
@pytest.mark.parametrize("order", ORDERS)
def test_separate_pair_arrays(cuda_ok, scenes, order):
    _check(scenes.preset("small"), order, separate_pairs=True)
    _check(scenes.make_scene(300, 170, 2000, n=16, bins=64, seed=11, sigma=0.1), order, separate_pairs=True)


@pytest.mark.parametrize("n,bins", [(8, 16), (16, 32), (32, 64), (4, 8), (12, 32), (1, 16), (2, 1)])
def test_light_grid_and_bins(cuda_ok, scenes, n, bins):
    _check(scenes.make_scene(160, 128, 700, n=n, bins=bins, seed=7, name=f"n{n}b{bins}"), 1)


@pytest.mark.parametrize("order", ORDERS)
def test_non_power_of_two_view(cuda_ok, scenes, order):
    # 1920-wide views hit the reference's padded output index (y<<ceil(log2 W)|x);
    # the library writes y*W+x.
    _check(scenes.make_scene(300, 170, 2000, n=16, bins=64, seed=11, sigma=0.1), order)


def test_background_samples(cuda_ok, scenes):
    s = scenes.make_scene(200, 150, 1500, n=8, bins=32, seed=5)
    rng = np.random.default_rng(0)
    bg = rng.random(s.S) < 0.3
    s.pos[bg, 0] = np.nan
    _check(s, 1)


def test_backfacing_samples(cuda_ok, scenes):
    s = scenes.make_scene(128, 128, 800, n=8, bins=16, seed=9)
    s.nrm[: s.S // 3, :3] *= -1.0   # a third of the receiver faces away from the light
    _check(s, 1)


@pytest.mark.parametrize("order", ORDERS)
def test_medium_scene(cuda_ok, scenes, order):
    _check(scenes.make_scene(640, 480, 20000, n=16, bins=64, seed=21, sigma=0.1), order)


def test_hd_preset_sampled(cuda_ok, scenes):
    """1920x1080 x 200k triangles x 16x16 light, 128^2 bins: every stage exact;
    masks checked on every 97th binned sample."""
    _check(scenes.preset("hd"), 1, occ_stride=97)


@pytest.mark.parametrize("schedule", [1])
@pytest.mark.parametrize("n,bins", [(1, 4), (4, 8), (8, 16), (16, 32), (32, 16)])
@pytest.mark.parametrize("order", ORDERS)
def test_other_occlusion_schedules(cuda_ok, scenes, n, bins, order, schedule):
    """The lane-per-pair occlusion schedule: same masks and shadows, bit for bit."""
    _check(scenes.make_scene(200, 150, 3000, n=n, bins=bins, seed=80 + n, sigma=0.12), order, schedule=schedule)


@pytest.mark.parametrize("schedule", [1])
def test_other_occlusion_schedules_medium(cuda_ok, scenes, schedule):
    _check(scenes.make_scene(640, 480, 20000, n=16, bins=64, seed=21, sigma=0.1), 1, schedule=schedule)


@pytest.mark.parametrize("masks", [True, False])
@pytest.mark.parametrize("schedule", [0, 1])
def test_triangle_passes_match_oracle(cuda_ok, fdzb, scenes, masks, schedule):
    """A pair-capacity limit far below the frame's pairs: the frame runs in
    passes over triangle ranges (overflowing ranges split again) and still
    matches the oracle bit for bit."""
    s = scenes.make_scene(320, 240, 6000, n=8, bins=32, seed=91, sigma=0.12)
    orc = oracle.frame(s)
    ctx, t = fdzb.context_for_scene(s, masks=masks)
    ctx.set_occlusion_schedule(schedule)
    ctx.set_pair_capacity_limit(20000)
    ctx.launch()
    st = ctx.stats()
    assert st["triangle_passes"] > 2, st["triangle_passes"]
    assert st["num_pairs"] == orc.scalars["num_pairs"]
    assert st["valid_triangles"] == orc.scalars["valid_tris"]
    sh = t["shadow"].cpu().numpy()
    assert np.array_equal(sh.view(np.uint32), orc.arrays["shadow"].astype(np.float32).view(np.uint32))
    if masks:
        mk = t["masks"].cpu().numpy().view(np.uint32)
        assert np.array_equal(mk, orc.arrays["masks"].reshape(-1).astype(np.uint32)[: mk.size])
    # a second launch reuses the limit and gives the same result
    ctx.launch()
    assert np.array_equal(t["shadow"].cpu().numpy(), sh)
    ctx.close()


@pytest.mark.parametrize("scene_args", [
    ("small", None),
    ("make", (640, 360, 20000, 16, 128, 31, 0.1)),     # penumbra-rich: the auto probe turns the cull off
    ("make", (480, 270, 30000, 8, 64, 32, 0.1)),
])
def test_open_box_modes_give_the_oracle_masks(cuda_ok, fdzb, scenes, scene_args):
    """The open-box cull skips only pairs that cannot set an unset bit: with it
    forced off, forced on and in auto mode (whose first launch probes it and
    may switch it off for the next), masks and shadows equal the oracle's."""
    kind, a = scene_args
    if kind == "small":
        s = scenes.preset("small")
    else:
        W, H, T, n, bins, seed, sigma = a
        s = scenes.make_scene(W, H, T, n=n, bins=bins, seed=seed, sigma=sigma)
    orc = oracle.frame(s)
    for mode in (fdzb.OPEN_BOX_OFF, fdzb.OPEN_BOX_ON, fdzb.OPEN_BOX_AUTO):
        ctx, t = fdzb.context_for_scene(s, masks=True, tri_order=1)
        ctx.set_open_box(mode)
        for _ in range(2):
            t["masks"].zero_()
            t["shadow"].fill_(-1.0)
            ctx.launch()
            errs = parity.compare(s, gpu=parity.collect(ctx, t, s, tri_order=1, intermediates=False), orc=orc)
            assert not errs, (mode, errs)
        wc = ctx.export("work_counters", 7)
        if mode == fdzb.OPEN_BOX_OFF:
            assert wc[6] == 0           # no pair skipped by the cull
        ctx.close()
