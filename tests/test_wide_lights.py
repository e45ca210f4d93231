"""Rectangular and wide light grids (up to 64 x 64) and the depth plane on the GPU.

The reference's per-sample kernel runs square grids up to 32 x 32; this
library takes any width x height up to 64 each (64-bit row words past 32) and,
optionally, tests each triangle's own plane (occluders beside or behind the
light).  Every case equals the oracle's restatement of the same arithmetic
bit for bit -- stage by stage where the parity harness exports them -- and the
oracle itself is pinned to the FP64 per-light-sample check and to the
ray-cast method on the CPU (tests/test_wide_lights_oracle.py).
"""
import dataclasses

import numpy as np
import pytest

import oracle
from tests import parity

pytestmark = pytest.mark.gpu

GRIDS = [(8, 16), (24, 5), (40, 40), (64, 64), (64, 8), (33, 2), (1, 7), (32, 33)]


def _scene(scenes, rows, cols, seed=21, W=96, H=72, T=500, **kw):
    s = scenes.make_scene(W, H, T, n=rows, bins=8, seed=seed, sigma=0.3, **kw)
    s.light = dataclasses.replace(s.light, n=rows, nh=cols)
    return s


def _behind_the_light(scenes, rows, cols, zlo, sigma):
    s = scenes.make_scene(96, 72, 300, n=rows, bins=8, seed=33, sigma=0.3)
    ev, ei = scenes.occluders(200, 77, sigma, zlo, zlo + 1.0)
    s = dataclasses.replace(s, vtx=np.concatenate([s.vtx, ev]), idx=np.concatenate([s.idx, ei + s.V]))
    s.light = dataclasses.replace(s.light, n=rows, nh=cols)
    return s


@pytest.mark.parametrize("rows,cols", GRIDS)
@pytest.mark.parametrize("order", [0, 1])
def test_rectangular_grid_matches_oracle(cuda_ok, scenes, rows, cols, order):
    s = _scene(scenes, rows, cols)
    errs = parity.compare(s, gpu=parity.run_gpu(s, tri_order=order))
    assert not errs, "\n".join(errs)


@pytest.mark.parametrize("rows,cols", [(24, 5), (64, 8)])
def test_lane_per_pair_request_falls_back_for_other_grids(cuda_ok, scenes, rows, cols):
    s = _scene(scenes, rows, cols, seed=22)
    errs = parity.compare(s, gpu=parity.run_gpu(s, schedule=1))
    assert not errs, "\n".join(errs)


@pytest.mark.parametrize("rows,cols,zlo,sigma", [(16, 16, 6.5, 0.5), (12, 40, 5.9, 0.4), (64, 48, 7.0, 1.0)])
@pytest.mark.parametrize("schedule", [0, 1])
def test_depth_plane_matches_oracle(cuda_ok, scenes, rows, cols, zlo, sigma, schedule):
    s = dataclasses.replace(_behind_the_light(scenes, rows, cols, zlo, sigma), depth_plane=True)
    errs = parity.compare(s, gpu=parity.run_gpu(s, schedule=schedule))
    assert not errs, "\n".join(errs)


def test_depth_plane_is_a_no_op_with_occluders_between(cuda_ok, fdzb, scenes):
    s = scenes.make_scene(160, 120, 1500, n=16, bins=16, seed=41, sigma=0.12)
    out = []
    for dp in (False, True):
        ctx, t = fdzb.context_for_scene(dataclasses.replace(s, depth_plane=dp), masks=True)
        ctx.launch()
        out.append(t["masks"].cpu().numpy().copy())
        ctx.close()
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("rows,cols", [(40, 40), (64, 8), (8, 16)])
def test_ray_cast_on_wide_grids_matches_oracle(cuda_ok, fdzb, scenes, rows, cols):
    s = _scene(scenes, rows, cols, seed=23)
    ctx, t = fdzb.context_for_scene(s, masks=True)
    ctx.set_shadow_method(fdzb.SHADOW_RAY_CAST)
    ctx.launch()
    sh, mk = t["shadow"].cpu().numpy(), t["masks"].cpu().numpy().view(np.uint32)
    ctx.close()
    o = oracle.frame(s, shadow_method=1)
    assert np.array_equal(sh.view(np.uint32), o.arrays["shadow"].astype(np.float32).view(np.uint32))
    assert np.array_equal(mk, o.arrays["masks"].reshape(-1).astype(np.uint32)[: mk.size])


@pytest.mark.parametrize("masks", [True, False])
def test_triangle_passes_with_wide_grid(cuda_ok, fdzb, scenes, masks):
    """Passes over triangle ranges re-load each sample's 64-bit rows from the
    packed masks of the earlier passes."""
    s = scenes.make_scene(200, 150, 3000, n=40, bins=16, seed=92, sigma=0.15)
    s.light = dataclasses.replace(s.light, n=40, nh=36)
    orc = oracle.frame(s)
    ctx, t = fdzb.context_for_scene(s, masks=masks)
    ctx.set_pair_capacity_limit(4000)
    ctx.launch()
    st = ctx.stats()
    assert st["triangle_passes"] > 2, st["triangle_passes"]
    sh = t["shadow"].cpu().numpy()
    assert np.array_equal(sh.view(np.uint32), orc.arrays["shadow"].astype(np.float32).view(np.uint32))
    if masks:
        mk = t["masks"].cpu().numpy().view(np.uint32)
        assert np.array_equal(mk, orc.arrays["masks"].reshape(-1).astype(np.uint32)[: mk.size])
    ctx.close()


def test_batch_mixing_square_and_wide_frames(cuda_ok, fdzb, scenes):
    """One launch runs every frame on 64-bit row words when one frame needs
    them; each frame still equals its own plain launch and the oracle."""
    import torch
    fr = [_scene(scenes, 16, 16, seed=60), _scene(scenes, 64, 8, seed=61), _scene(scenes, 5, 30, seed=62),
          _scene(scenes, 32, 32, seed=63)]
    tens, descs = [], []
    for s in fr:
        pos, nrm, vtx, idx = fdzb.upload_scene(s)
        sh = torch.full((s.S,), -1.0, dtype=torch.float32, device="cuda")
        mk = torch.zeros(s.S * fdzb.mask_words(s.light.n, s.light.cols), dtype=torch.int32, device="cuda")
        tens.append(dict(pos=pos, nrm=nrm, vtx=vtx, idx=idx, shadow=sh, masks=mk))
        descs.append(fdzb.frame_desc(pos, nrm, s.W, s.H, vtx, s.V, idx, s.T, s.light, sh, mk, bins=s.bins,
                                     cull=s.cull, esp=s.esp))
    b = fdzb.Batch()
    b.launch(descs)
    for s, t in zip(fr, tens):
        o = oracle.frame(s)
        assert np.array_equal(t["shadow"].cpu().numpy().view(np.uint32),
                              o.arrays["shadow"].astype(np.float32).view(np.uint32))
        mk = t["masks"].cpu().numpy().view(np.uint32)
        assert np.array_equal(mk, o.arrays["masks"].reshape(-1).astype(np.uint32)[: mk.size])
    b.close()


def test_grid_limits_are_checked(cuda_ok, fdzb, scenes):
    s = _scene(scenes, 8, 8)
    ctx, _ = fdzb.context_for_scene(s)
    for w, h in ((65, 8), (8, 65), (0, 4)):
        with pytest.raises(fdzb.FdzbError):
            ctx.set_area_light(dataclasses.replace(s.light, n=w, nh=h))
    ctx.close()
