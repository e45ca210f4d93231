"""GPU parity: every stage of the CUDA pipeline bit-exact against the CPU oracle.

Bar: bin keys, sorted sample order, per-bin segments and statistics, triangle
footprints, per-triangle bin counts, triangle/bin pairs (before and after the
sort), per-bin triangle segments, N^2-bit masks and shadow values all equal the
FP32 restatement bit for bit (both sides compute with unfused IEEE binary32
operations in the reference's order).
"""
import numpy as np
import pytest

from tests import parity

pytestmark = pytest.mark.gpu


def _check(scene):
    errs = parity.compare(scene)
    assert not errs, "\n".join(errs)


@pytest.mark.parametrize("cull", [False, True])
def test_small_preset(cuda_ok, scenes, cull):
    _check(scenes.preset("small", cull=cull))


@pytest.mark.parametrize("n,bins", [(8, 16), (16, 32), (32, 64), (4, 8), (12, 32), (1, 16)])
def test_light_grid_and_bins(cuda_ok, scenes, n, bins):
    _check(scenes.make_scene(160, 128, 700, n=n, bins=bins, seed=7, name=f"n{n}b{bins}"))


def test_non_power_of_two_view(cuda_ok, scenes):
    # 1920-wide views hit the reference's padded output index (y<<ceil(log2 W)|x);
    # the library writes y*W+x.
    _check(scenes.make_scene(300, 170, 2000, n=16, bins=64, seed=11, sigma=0.1))


def test_background_samples(cuda_ok, scenes):
    s = scenes.make_scene(200, 150, 1500, n=8, bins=32, seed=5)
    rng = np.random.default_rng(0)
    bg = rng.random(s.S) < 0.3
    s.pos[bg, 0] = np.nan
    _check(s)


def test_backfacing_samples(cuda_ok, scenes):
    s = scenes.make_scene(128, 128, 800, n=8, bins=16, seed=9)
    s.nrm[: s.S // 3, :3] *= -1.0   # a third of the receiver faces away from the light
    _check(s)


def test_medium_scene(cuda_ok, scenes):
    _check(scenes.make_scene(640, 480, 20000, n=16, bins=64, seed=21, sigma=0.1))
