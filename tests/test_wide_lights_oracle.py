"""CPU tests of the oracle's rectangular and wide light grids and of the depth plane.

The reference's per-sample kernel runs square grids up to 32 x 32 only
(K/Step5_2_shadowCalPerSample.inl:249-254).  The same closed-form arithmetic on
64-bit row words covers any width x height up to 64 x 64 (rows along x_delt,
columns along y_delt); these tests pin that generalisation with two independent
checks: the FP64 per-light-sample oracle (O3) and the ray-cast method, whose
light samples are placed explicitly at upRight + x_delt*j + y_delt*i, so a
transposed or mis-sized grid would disagree with it at once.  The optional
depth plane (the triangle's own plane, as in the reference's per-bin kernel)
is checked the same way on a scene with occluders beside and behind the light.
"""
import dataclasses

import numpy as np
import pytest

import oracle

GRIDS = [(8, 16), (24, 5), (40, 40), (64, 64), (64, 8), (1, 7), (33, 2)]


def _bits(masks, rows, cols):
    return np.unpackbits(masks.view(np.uint8), bitorder="little").reshape(masks.shape[0], -1)[:, :rows * cols]


def _scene(scenes, rows, cols, seed=21, W=96, H=72, T=500, **kw):
    s = scenes.make_scene(W, H, T, n=rows, bins=8, seed=seed, sigma=0.3, **kw)
    s.light = dataclasses.replace(s.light, n=rows, nh=cols)
    return s


@pytest.mark.parametrize("rows,cols", GRIDS)
def test_rectangular_grid_within_tolerance_of_fp64(scenes, rows, cols):
    s = _scene(scenes, rows, cols)
    fr = oracle.frame(s)
    assert fr.scalars["state"] == 2
    ids = np.arange(s.S, dtype=np.int32)[::3].copy()
    m64, dist = oracle.exhaustive_fp64(s, fr, ids)
    m32 = fr.arrays["masks"].reshape(s.S, -1)[ids]
    assert m32.shape[1] == oracle.mask_words(rows, cols)
    b32, b64 = _bits(m32, rows, cols), _bits(m64, rows, cols)
    flip = b32 != b64
    assert flip.mean() <= 1e-4, flip.mean()
    if flip.any():
        assert dist[flip].max() <= 1e-3
    assert b32.any(), "the scene must cast some shadow"
    # shadow = set bits / (rows * cols)
    sh = fr.arrays["shadow"][ids]
    assert np.array_equal(sh, (b32.sum(axis=1) / np.float32(rows * cols)).astype(np.float32))


@pytest.mark.parametrize("rows,cols", [(8, 16), (24, 5), (40, 40)])
def test_rectangular_grid_agrees_with_ray_cast(scenes, rows, cols):
    """The edge-function rows run along x_delt and the columns along y_delt: the
    ray-cast method, which places each light sample explicitly, agrees except at
    light samples next to a projected edge."""
    s = _scene(scenes, rows, cols)
    edge = oracle.frame(s)
    ray = oracle.frame(s, shadow_method=1)
    be = _bits(edge.arrays["masks"].reshape(s.S, -1), rows, cols)
    br = _bits(ray.arrays["masks"].reshape(s.S, -1), rows, cols)
    assert be.any()
    assert (be != br).mean() < 2e-3, (be != br).mean()


def test_square_grid_explicit_height_is_the_square_grid(scenes):
    s = scenes.preset("small")
    a = oracle.frame(s)
    t = dataclasses.replace(s, light=dataclasses.replace(s.light, nh=s.light.n))
    b = oracle.frame(t)
    assert np.array_equal(a.arrays["masks"], b.arrays["masks"])
    assert np.array_equal(a.arrays["shadow"], b.arrays["shadow"])


def test_depth_plane_changes_nothing_when_occluders_are_between(scenes):
    """Every triangle of the standard scene lies between its receivers and the
    light, so the plane is never needed and the result is the same bit for bit."""
    s = scenes.preset("small")
    a = oracle.frame(s)
    b = oracle.frame(dataclasses.replace(s, depth_plane=True))
    assert np.array_equal(a.arrays["masks"], b.arrays["masks"])


def _behind_the_light(scenes, rows=16, cols=16, zlo=6.5, sigma=0.5):
    """The small scene plus 200 triangles at or above the light's plane (the
    light sits at z = 6 facing down): occluders the per-sample kernel, which
    has no triangle-plane test, wrongly lets shadow the receivers."""
    s = scenes.make_scene(96, 72, 300, n=rows, bins=8, seed=33, sigma=0.3)
    ev, ei = scenes.occluders(200, 77, sigma, zlo, zlo + 1.0)
    s = dataclasses.replace(s, vtx=np.concatenate([s.vtx, ev]), idx=np.concatenate([s.idx, ei + s.V]))
    s.light = dataclasses.replace(s.light, n=rows, nh=cols)
    return s


@pytest.mark.parametrize("rows,cols,zlo,sigma", [(16, 16, 6.5, 0.5), (12, 40, 5.9, 0.4), (16, 16, 7.0, 1.0)])
def test_depth_plane_follows_the_ray_cast(scenes, rows, cols, zlo, sigma):
    s = _behind_the_light(scenes, rows, cols, zlo=zlo, sigma=sigma)
    ray = _bits(oracle.frame(s, shadow_method=1).arrays["masks"].reshape(s.S, -1), rows, cols)
    plain = _bits(oracle.frame(s).arrays["masks"].reshape(s.S, -1), rows, cols)
    depth = _bits(oracle.frame(dataclasses.replace(s, depth_plane=True)).arrays["masks"].reshape(s.S, -1),
                  rows, cols)
    d_plain = (plain != ray).mean()
    d_depth = (depth != ray).mean()
    assert d_plain > 1e-3, "the scene must need the depth plane"
    assert d_depth < 1e-5, (d_depth, d_plain)


def test_depth_plane_within_tolerance_of_fp64(scenes):
    s = dataclasses.replace(_behind_the_light(scenes), depth_plane=True)
    fr = oracle.frame(s)
    ids = np.arange(s.S, dtype=np.int32)[::2].copy()
    m64, dist = oracle.exhaustive_fp64(s, fr, ids)
    N = s.light.n
    b32 = _bits(fr.arrays["masks"].reshape(s.S, -1)[ids], N, N)
    b64 = _bits(m64, N, N)
    flip = b32 != b64
    assert flip.mean() <= 1e-4, flip.mean()
    if flip.any():
        assert dist[flip].max() <= 1e-3
