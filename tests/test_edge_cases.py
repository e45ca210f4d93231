"""Edge cases of the shadow path on the GPU, each against the oracle stage by stage.

Empty inputs (no triangles, every sample background, no light plane),
degenerate views (1 x 1, single rows and columns, odd sizes), the bin grid's
extremes (1 and 512 per side), degenerate and repeated triangles (zero area,
collinear, duplicates: equal sort keys), triangles crossing the light's plane
(the reference has no depth test there and the oracle reproduces that),
receivers that are themselves triangle vertices (the coplanar self-skip), and
the self-skip distance at 0 and large.  Both triangle orders.
"""
import dataclasses

import numpy as np
import pytest

import oracle
from tests import parity

pytestmark = pytest.mark.gpu

ORDERS = [0, 1]


def _check(scene, order=1):
    orc = oracle.frame(scene)
    errs = parity.compare(scene, gpu=parity.run_gpu(scene, tri_order=order), orc=orc)
    assert not errs, "\n".join(errs)
    return orc


def _base(scenes, **kw):
    a = dict(W=64, H=48, T=300, n=8, bins=16, seed=3)
    a.update(kw)
    return scenes.make_scene(**a)


@pytest.mark.parametrize("order", ORDERS)
def test_no_triangles(cuda_ok, scenes, order):
    b = _base(scenes)
    s = dataclasses.replace(b, vtx=b.vtx[:0].copy(), idx=b.idx[:0].copy())
    o = _check(s, order)
    assert o.scalars["state"] == 0


def test_every_sample_background(cuda_ok, scenes):
    b = _base(scenes)
    s = dataclasses.replace(b, pos=b.pos.copy())
    s.pos[:, 0] = np.nan
    o = _check(s)
    assert o.scalars["state"] == 0


def test_triangles_beside_the_light_plane(cuda_ok, scenes):
    b = _base(scenes)
    s = dataclasses.replace(b, vtx=b.vtx.copy())
    s.vtx[:, 0] += 100.0
    o = _check(s)
    assert o.scalars["state"] == 1


@pytest.mark.parametrize("W,H", [(1, 1), (1, 7), (7, 1), (33, 17), (129, 3)])
def test_degenerate_views(cuda_ok, scenes, W, H):
    _check(scenes.make_scene(W, H, 300, n=8, bins=16, seed=4))


@pytest.mark.parametrize("bins", [1, 2, 512])
@pytest.mark.parametrize("order", ORDERS)
def test_bin_grid_extremes(cuda_ok, scenes, bins, order):
    _check(scenes.make_scene(96, 64, 400, n=8, bins=bins, seed=5), order)


def _with_degenerate_triangles(scenes, seed=6):
    b = _base(scenes, T=400, seed=seed, W=96, H=72)
    rng = np.random.default_rng(seed)
    v, i = [b.vtx], [b.idx]
    nv = b.V
    # duplicates of existing triangles (same vertex indices), in a shuffled order
    dup = b.idx[rng.permutation(b.T)[:120]]
    i.append(dup)
    # zero-area: three copies of one point; collinear: three points on a line
    pts = b.vtx[rng.integers(0, b.V, 60), :3]
    zero = np.repeat(pts[:30], 3, axis=0)
    d = rng.normal(0, 0.05, (30, 3)).astype(np.float32)
    col = np.stack([pts[30:], pts[30:] + d, pts[30:] + 2.5 * d], axis=1).reshape(-1, 3)
    # tiny triangles (edges ~1e-6)
    tiny = (pts[:30, None, :] + rng.normal(0, 1e-6, (30, 3, 3))).reshape(-1, 3)
    for blk in (zero, col, tiny):
        q = np.c_[blk, np.ones(len(blk))].astype(np.float32)
        v.append(q)
        i.append((nv + np.arange(len(blk))).reshape(-1, 3).astype(b.idx.dtype))
        nv += len(blk)
    return dataclasses.replace(b, vtx=np.concatenate(v), idx=np.concatenate(i))


@pytest.mark.parametrize("order", ORDERS)
@pytest.mark.parametrize("cull", [False, True])
def test_degenerate_and_repeated_triangles(cuda_ok, scenes, order, cull):
    s = dataclasses.replace(_with_degenerate_triangles(scenes), cull=cull)
    o = _check(s, order)
    assert o.scalars["state"] == 2 and o.scalars["num_pairs"] > 0


def test_triangles_crossing_the_light_plane(cuda_ok, scenes):
    """Occluders from below the receivers' highest point up past the light
    (the light sits at z = 6): no depth test, as in the reference."""
    b = _base(scenes, T=200, W=80, H=60, seed=8)
    ev, ei = scenes.occluders(150, 81, 0.8, 4.0, 8.0)
    s = dataclasses.replace(b, vtx=np.concatenate([b.vtx, ev]), idx=np.concatenate([b.idx, ei + b.V]))
    _check(s)


def _receiver_triangles(s, step=3):
    """Triangles whose vertices are receiver samples: cells (x, y), (x+1, y),
    (x, y+1) of the sample grid, every `step`-th cell."""
    W, H = s.W, s.H
    ys, xs = np.meshgrid(np.arange(0, H - 1, step), np.arange(0, W - 1, step), indexing="ij")
    a = (ys * W + xs).ravel()
    tri = np.stack([a, a + 1, a + W], axis=1)
    v = s.pos[tri.ravel()].copy()
    v[:, 3] = 1.0
    return v.astype(np.float32), np.arange(len(v), dtype=s.idx.dtype).reshape(-1, 3)


@pytest.mark.parametrize("esp", [1e-3, 0.0, 0.05])
def test_receivers_on_triangles_self_skip(cuda_ok, scenes, esp):
    b = _base(scenes, T=300, W=72, H=54, seed=9)
    rv, ri = _receiver_triangles(b)
    s = dataclasses.replace(b, vtx=np.concatenate([b.vtx, rv]), idx=np.concatenate([b.idx, ri + b.V]), esp=esp)
    _check(s)
