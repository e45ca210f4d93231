"""CPU tests of the G-buffer rasteriser oracle (oracle/fdzb_raster_oracle.c).

The oracle fixes the rules GL leaves to the implementation (see the file's
header); these tests check that the rules do what GL requires of them:
perspective-correct attributes (each pixel's world position projects back to
its pixel centre), shared edges drawn exactly once, GL_LESS with the earlier
triangle winning ties, near-plane clipping, and draws that compose.
"""
import importlib

import numpy as np
import pytest

from oracle import orc

scenes = importlib.import_module("4dzb_b200.scenes")


def _draw(ms, **kw):
    return orc.raster(ms.vtx, ms.idx, ms.materials, ms.model, ms.view_proj, ms.W, ms.H,
                      tri_material=ms.tri_material, **kw)


def _reproject(vp, P, W, H):
    c = np.c_[P.astype(np.float64), np.ones(len(P))] @ vp.T
    ndc = c[:, :3] / c[:, 3:4]
    return (ndc[:, 0] + 1) * W / 2, (ndc[:, 1] + 1) * H / 2, ndc[:, 2] * 0.5 + 0.5


@pytest.mark.parametrize("eye", [(0.0, -13.0, 11.0), (3.0, -6.0, 2.5), (0.0, -1.0, 20.0)])
def test_world_positions_project_back_to_their_pixel_centres(eye):
    ms = scenes.mesh_scene(160, 120, eye=eye)
    o = _draw(ms)
    cov = ~np.isnan(o["g0"][:, 0])
    assert cov.mean() > 0.2
    p = np.flatnonzero(cov)
    xw, yw, zw = _reproject(ms.view_proj, o["g0"][p, :3], ms.W, ms.H)
    # vertices snap to 1/16 pixel: a position may sit up to 1/32 pixel off
    assert np.abs(xw - (p % ms.W + 0.5)).max() < 0.04
    assert np.abs(yw - (p // ms.W + 0.5)).max() < 0.04
    assert np.abs(zw - o["depth"][p]).max() < 1e-5
    # G-buffer packing of the gatherData shader
    assert set(np.unique(o["g3"][p, 3])) <= set(ms.materials[:, 9])


def _quad(W, H):
    # a W x H window filled by two triangles whose diagonal runs through pixel
    # centres (x + 0.5, y + 0.5) for a square window; identity camera (NDC)
    vtx = np.zeros((4, 8), np.float32)
    vtx[:, :3] = [[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]]
    vtx[:, 7] = 1.0
    idx = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    return vtx, idx


def test_shared_edges_are_drawn_exactly_once():
    W = H = 32
    vtx, idx = _quad(W, H)
    mats = np.zeros((1, 10), np.float32)
    I = np.eye(4)
    a = orc.raster(vtx, idx[:1], mats, I, I, W, H)
    b = orc.raster(vtx, idx[1:], mats, I, I, W, H)
    ca, cb = ~np.isnan(a["g0"][:, 0]), ~np.isnan(b["g0"][:, 0])
    assert not (ca & cb).any(), "a pixel centre on the shared diagonal was drawn twice"
    assert (ca | cb).all(), "a pixel centre was drawn by neither triangle"
    # the diagonal's centres exist and went to exactly one side
    diag = np.arange(W) * W + np.arange(W)
    assert ca[diag].all() or cb[diag].all()


def test_earlier_triangle_wins_equal_depth_and_nearer_wins_otherwise():
    W = H = 16
    vtx = np.zeros((6, 8), np.float32)
    tri = [[-1, -1, 0.2], [3, -1, 0.2], [-1, 3, 0.2]]
    vtx[:3, :3] = tri
    vtx[3:, :3] = tri
    idx = np.array([[0, 1, 2], [3, 4, 5]], np.uint32)
    mats = np.zeros((2, 10), np.float32)
    mats[1, 9] = 7.0
    I = np.eye(4)
    o = orc.raster(vtx, idx, mats, I, I, W, H, tri_material=np.array([0, 1], np.int32))
    assert np.all(o["g3"][:, 3] == 0.0), "the first of two equal-depth triangles must win"
    vtx[3:, 2] = 0.1   # the second triangle is now nearer
    o = orc.raster(vtx, idx, mats, I, I, W, H, tri_material=np.array([0, 1], np.int32))
    assert np.all(o["g3"][:, 3] == 7.0)


def test_near_plane_clipping_splits_and_keeps_geometry():
    # camera just above the receiver, looking along it: many triangles cross
    # the near plane and are cut into a triangle or a quad
    ms = scenes.mesh_scene(160, 120, eye=(0.0, -7.5, 0.6), center=(0.0, 8.0, 0.0), near=0.5)
    o = _draw(ms)
    assert o["sub_tris"] > ms.T * 0.9
    cov = np.flatnonzero(~np.isnan(o["g0"][:, 0]))
    xw, yw, _ = _reproject(ms.view_proj, o["g0"][cov, :3], ms.W, ms.H)
    assert np.abs(xw - (cov % ms.W + 0.5)).max() < 0.04
    assert np.abs(yw - (cov // ms.W + 0.5)).max() < 0.04
    # nothing drawn is behind the near plane
    c = np.c_[o["g0"][cov, :3].astype(np.float64), np.ones(len(cov))] @ ms.view_proj.T
    assert (c[:, 2] >= -c[:, 3] - 1e-4).all()


def test_draws_compose_like_one_draw():
    ms = scenes.mesh_scene(128, 96)
    whole = _draw(ms)
    k = ms.n_receiver
    first = orc.raster(ms.vtx, ms.idx[:k], ms.materials, ms.model, ms.view_proj, ms.W, ms.H,
                       tri_material=ms.tri_material[:k])
    both = orc.raster(ms.vtx, ms.idx[k:], ms.materials, ms.model, ms.view_proj, ms.W, ms.H,
                      tri_material=ms.tri_material[k:], clear=False, prev=first)
    for key in ("g0", "g1", "g2", "g3", "depth"):
        assert np.array_equal(whole[key].view(np.uint32), both[key].view(np.uint32)), key
