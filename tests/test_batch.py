"""Batched launches (fdzb_batch_*): many independent frames per launch.

* every frame of a batch gets exactly what a separate fdzb_ctx_launch of the same
  inputs gets (shadows, masks, per-frame statistics), and what the oracle gets;
* frames that stop early (all background, no triangles, only back-facing
  samples) do not disturb their neighbours;
* CUDA-graph replays see new input data in the same buffers;
* the autotuner picks a power-of-two grid per size class and the results match
  a plain launch with that grid.
"""
import importlib

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _frames(scenes, n=6, seed_base=5000):
    fr = [scenes.batch_frame(k, s_range=(40 * 40, 180 * 120), t_range=(200, 3000), ns=(4, 8, 16),
                             seed_base=seed_base) for k in range(n)]
    grids = [8, 16, 32, 16, 4, 64, 8, 32]
    for i, f in enumerate(fr):
        f.bins = grids[i % len(grids)]
    return fr


def _upload(fdzb, scene, masks=True):
    import torch
    pos, nrm, vtx, idx = fdzb.upload_scene(scene)
    sh = torch.full((scene.S,), -1.0, dtype=torch.float32, device="cuda")
    mk = torch.zeros(scene.S * fdzb.mask_words(scene.light.n), dtype=torch.int32, device="cuda") if masks else None
    return dict(pos=pos, nrm=nrm, vtx=vtx, idx=idx, shadow=sh, masks=mk)


def _desc(fdzb, scene, t, bins=None):
    return fdzb.frame_desc(t["pos"], t["nrm"], scene.W, scene.H, t["vtx"], scene.V, t["idx"], scene.T,
                           scene.light, t["shadow"], t["masks"], bins=scene.bins if bins is None else bins,
                           cull=scene.cull, esp=scene.esp)


def _plain(fdzb, scene, bins=None):
    import dataclasses
    s = dataclasses.replace(scene, bins=scene.bins if bins is None else bins)
    ctx, t = fdzb.context_for_scene(s, masks=True)
    ctx.launch()
    st = ctx.stats()
    out = t["shadow"].cpu().numpy(), t["masks"].cpu().numpy().view(np.uint32)
    ctx.close()
    return out, st


def _check_same(a, b, what):
    assert a.shape == b.shape, what
    bad = np.flatnonzero(a.view(np.uint32) != b.view(np.uint32))
    assert bad.size == 0, f"{what}: {bad.size} differ, first {bad[:5].tolist()}"


def test_batch_matches_plain_and_oracle(cuda_ok, fdzb, scenes):
    fr = _frames(scenes, 6)
    tens = [_upload(fdzb, s) for s in fr]
    b = fdzb.Batch()
    b.launch([_desc(fdzb, s, t) for s, t in zip(fr, tens)])
    bst = b.stats()
    assert bst["frames"] == len(fr)
    for i, (s, t) in enumerate(zip(fr, tens)):
        (sh, mk), st = _plain(fdzb, s)
        _check_same(t["shadow"].cpu().numpy(), sh, f"frame {i} shadow")
        _check_same(t["masks"].cpu().numpy().view(np.uint32), mk, f"frame {i} masks")
        fs = b.frame_stats(i)
        for k in ("state", "valid_samples", "valid_triangles", "num_bins"):
            assert fs[k] == st[k], (i, k)
        for k in ("f", "sub", "lp_begin", "lp_end", "lp_factor"):
            assert np.array_equal(np.float32(fs[k]), np.float32(st[k])), (i, k)
        o = oracle.frame(s)
        _check_same(t["shadow"].cpu().numpy(), o.arrays["shadow"].astype(np.float32), f"frame {i} vs oracle")
    b.close()


def test_batch_early_exit_frames_do_not_disturb_neighbours(cuda_ok, fdzb, scenes):
    fr = _frames(scenes, 5, seed_base=5100)
    fr[1].pos[:, 0] = np.nan                        # all background: state 0
    fr[3].nrm[:, :3] *= -1.0                        # only back-facing samples: state 1
    tens = [_upload(fdzb, s) for s in fr]
    empty = scenes.batch_frame(9, s_range=(32 * 32, 32 * 32), t_range=(200, 200), seed_base=5100)
    empty.bins = 8
    te = _upload(fdzb, empty)
    d = [_desc(fdzb, s, t) for s, t in zip(fr, tens)]
    de = _desc(fdzb, empty, te)
    de.n_tri = 0                                    # no triangles: state 1
    d.insert(2, de)
    b = fdzb.Batch()
    b.launch(d)
    states = [b.frame_stats(i)["state"] for i in range(len(d))]
    assert states[1] == 0 and states[2] == 1 and states[4] == 1, states
    for i, (s, t) in enumerate(zip(fr, tens)):
        (sh, mk), _ = _plain(fdzb, s)
        _check_same(t["shadow"].cpu().numpy(), sh, f"frame {i} shadow")
        _check_same(t["masks"].cpu().numpy().view(np.uint32), mk, f"frame {i} masks")
    assert np.all(te["shadow"].cpu().numpy() == 0.0)
    b.close()


def test_graph_replay_sees_new_inputs(cuda_ok, fdzb, scenes):
    import torch
    fr = _frames(scenes, 4, seed_base=5200)
    tens = [_upload(fdzb, s) for s in fr]
    b = fdzb.Batch()
    d = [_desc(fdzb, s, t) for s, t in zip(fr, tens)]
    b.launch(d)
    b.launch(d)    # the open-box probe of the first launch may pick the other kernel: settled now
    first = [t["shadow"].clone() for t in tens]
    for t in tens:
        t["shadow"].fill_(-1.0)
    b.launch(d)
    st = b.stats()
    assert st["from_graph"] == 1 and st["graph_replays"] >= 1
    for i, t in enumerate(tens):
        assert torch.equal(t["shadow"], first[i]), i
    # new receiver samples of the same size in the same buffers
    s0 = fr[0]
    alt = scenes.make_scene(s0.W, s0.H, s0.T, n=s0.light.n, bins=s0.bins, seed=777, sigma=0.1)
    alt.light = s0.light
    alt.vtx, alt.idx = s0.vtx, s0.idx
    tens[0]["pos"].copy_(torch.from_numpy(alt.pos))
    tens[0]["nrm"].copy_(torch.from_numpy(alt.nrm))
    b.launch(d)
    assert b.stats()["graph_replays"] >= 2
    (sh, mk), _ = _plain(fdzb, alt)
    _check_same(tens[0]["shadow"].cpu().numpy(), sh, "replayed frame with new samples")
    b.close()


def test_graph_on_off_identical_for_context(cuda_ok, fdzb, scenes):
    s = scenes.make_scene(160, 120, 2000, n=8, bins=16, seed=41)
    ctx, t = fdzb.context_for_scene(s, masks=True)
    ctx.launch()
    a = t["masks"].cpu().numpy().copy()
    ctx.launch()
    b = t["masks"].cpu().numpy().copy()
    ctx.set_graph(False)
    t["masks"].zero_()
    ctx.launch()
    c = t["masks"].cpu().numpy().copy()
    assert np.array_equal(a, b) and np.array_equal(a, c)
    ctx.close()


def test_autotune_picks_power_of_two_grids(cuda_ok, fdzb, scenes):
    import torch
    fr = _frames(scenes, 4, seed_base=5300)
    tens = [_upload(fdzb, s) for s in fr]
    d = [_desc(fdzb, s, t, bins=0) for s, t in zip(fr, tens)]
    scratch = torch.empty(max(s.S for s in fr) * 8, dtype=torch.float32, device="cuda")
    b = fdzb.Batch()
    b.autotune(d, scratch)
    st0 = b.stats()
    assert st0["tuned_classes"] >= 1 and st0["tune_launches"] >= 2
    b.launch(d)
    for i, s in enumerate(fr):
        g = b.frame_bins(i)
        assert g >= 4 and (g & (g - 1)) == 0
        (sh, mk), _ = _plain(fdzb, s, bins=g)
        _check_same(tens[i]["shadow"].cpu().numpy(), sh, f"frame {i} shadow (bins {g})")
        _check_same(tens[i]["masks"].cpu().numpy().view(np.uint32), mk, f"frame {i} masks (bins {g})")
    b.close()


def test_batch_reference_and_depth_order_same_masks(cuda_ok, fdzb, scenes):
    fr = _frames(scenes, 3, seed_base=5400)
    tens = [_upload(fdzb, s) for s in fr]
    d = [_desc(fdzb, s, t) for s, t in zip(fr, tens)]
    b = fdzb.Batch()
    b.launch(d)
    depth = [t["masks"].cpu().numpy().copy() for t in tens]
    b.set_tri_order(fdzb.TRI_ORDER_REFERENCE)
    b.launch(d)
    for i, t in enumerate(tens):
        assert np.array_equal(t["masks"].cpu().numpy(), depth[i]), i
    b.close()


@pytest.mark.parametrize("chunk", [8, 16, 32])
@pytest.mark.parametrize("item", [32, 64, 128])
def test_every_occlusion_shape_gives_the_same_masks(cuda_ok, fdzb, scenes, chunk, item):
    """Staging chunk and samples per warp item (the shapes the autotuner picks
    from) change the schedule only: masks and shadows equal the default shape's
    and the oracle's, in a batch and in a context."""
    fr = _frames(scenes, 4, seed_base=5500)
    tens = [_upload(fdzb, s) for s in fr]
    d = [_desc(fdzb, s, t) for s, t in zip(fr, tens)]
    b = fdzb.Batch()
    b.launch(d)
    base = [(t["shadow"].cpu().numpy().copy(), t["masks"].cpu().numpy().copy()) for t in tens]
    for t in tens:
        t["shadow"].fill_(-1.0)
        t["masks"].zero_()
    b.set_occlusion_shape(chunk, item)
    b.launch(d)
    for i, t in enumerate(tens):
        assert b.frame_shape(i) == (fr[i].bins, chunk, item)
        _check_same(t["shadow"].cpu().numpy(), base[i][0], f"frame {i} shadow, shape {chunk}x{item}")
        _check_same(t["masks"].cpu().numpy().view(np.uint32), base[i][1].view(np.uint32), f"frame {i} masks")
    b.close()
    s = scenes.make_scene(300, 200, 4000, n=16, bins=32, seed=61, sigma=0.1)
    ctx, t = fdzb.context_for_scene(s, masks=True)
    ctx.set_occlusion_shape(chunk, item)
    ctx.launch()
    o = oracle.frame(s)
    _check_same(t["shadow"].cpu().numpy(), o.arrays["shadow"].astype(np.float32), "context shadow vs oracle")
    _check_same(t["masks"].cpu().numpy().view(np.uint32), o.arrays["masks"].astype(np.uint32), "context masks")
    ctx.close()


def test_autotuner_reports_a_shape_per_frame(cuda_ok, fdzb, scenes):
    import torch
    fr = _frames(scenes, 4, seed_base=5600)
    tens = [_upload(fdzb, s) for s in fr]
    d = [_desc(fdzb, s, t, bins=0) for s, t in zip(fr, tens)]
    scratch = torch.empty(max(s.S for s in fr) * 8, dtype=torch.float32, device="cuda")
    b = fdzb.Batch()
    b.autotune(d, scratch)
    b.launch(d)
    for i, s in enumerate(fr):
        g, chunk, item = b.frame_shape(i)
        assert g == b.frame_bins(i) and chunk in fdzb.OCC_CHUNKS and item in fdzb.OCC_ITEMS
        import dataclasses
        ctx, t = fdzb.context_for_scene(dataclasses.replace(s, bins=g), masks=True)
        ctx.launch()
        _check_same(tens[i]["masks"].cpu().numpy().view(np.uint32), t["masks"].cpu().numpy().view(np.uint32),
                    f"frame {i} masks, tuned shape {(g, chunk, item)}")
        ctx.close()
    b.close()
