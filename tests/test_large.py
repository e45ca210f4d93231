"""The large workload (3840x2160 samples, 2M triangles, 32x32 light = 1024-bit
masks, 256^2 bins).

* parity against the oracle on a central crop of the view (480x270 samples,
  the first 250k triangles, same light and bin grid): every stage bit for bit,
  masks on every 13th binned sample;
* on the full frame, size-independent properties: every shadow value equals
  popcount(mask)/N^2, lies in [0, 1], the two triangle orders and the two
  occlusion schedules give identical masks, and a repeated launch (a CUDA graph
  replay) reproduces them.
"""
import dataclasses
import importlib

import numpy as np
import pytest

import oracle
from tests import parity

pytestmark = pytest.mark.gpu


def _crop(scene, W, H):
    x0, y0 = (scene.W - W) // 2, (scene.H - H) // 2
    idx = (np.arange(y0, y0 + H)[:, None] * scene.W + np.arange(x0, x0 + W)[None, :]).ravel()
    return dataclasses.replace(scene, W=W, H=H, pos=scene.pos[idx].copy(), nrm=scene.nrm[idx].copy(),
                               name=scene.name + "-crop")


@pytest.fixture(scope="module")
def large(scenes):
    return scenes.preset("large")


def test_large_crop_parity(cuda_ok, large):
    crop = _crop(large, 480, 270)
    crop = dataclasses.replace(crop, idx=crop.idx[:250_000].copy())
    orc = oracle.frame(crop, occ_stride=13)
    errs = parity.compare(crop, gpu=parity.run_gpu(crop, tri_order=1), orc=orc)
    assert not errs, "\n".join(errs)


def test_large_full_frame_properties(cuda_ok, fdzb, large):
    import torch
    ctx, t = fdzb.context_for_scene(large, masks=True)
    ctx.launch()
    st = ctx.stats()
    assert st["state"] == 2
    # ~10^10 triangle/bin pairs: the frame runs in triangle passes
    assert st["triangle_passes"] > 1
    mk = t["masks"].clone()
    sh = t["shadow"].clone()
    N = large.light.n
    words = fdzb.mask_words(N)
    m = mk.view(-1, words)
    pop = torch.zeros(m.shape[0], dtype=torch.int64, device="cuda")
    for w in range(words):
        x = m[:, w].to(torch.int64) & 0xFFFFFFFF
        for b in range(32):
            pop += (x >> b) & 1
    assert torch.equal((pop.to(torch.float32) / float(N * N)), sh)
    assert float(sh.min()) >= 0.0 and float(sh.max()) <= 1.0
    # graph replay
    t["masks"].zero_()
    ctx.launch()
    assert torch.equal(t["masks"], mk)
    # reference triangle order, lane-per-pair schedule
    ctx.set_tri_order(fdzb.TRI_ORDER_REFERENCE)
    t["masks"].zero_()
    ctx.launch()
    assert torch.equal(t["masks"], mk)
    ctx.set_tri_order(fdzb.TRI_ORDER_COVERAGE)
    ctx.set_occlusion_schedule(fdzb.OCC_LANE_PER_PAIR)
    t["masks"].zero_()
    ctx.launch()
    assert torch.equal(t["masks"], mk)
    ctx.close()
