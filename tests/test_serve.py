"""The request server (fdzb_serve_*): continuous batching over resident scenes.

* each request's shadows and masks are the same alone (one request on the
  server at a time), in a burst that the server batches and overlaps across
  slots, and in a plain single-frame launch of the same inputs;
* admission by memory budget: a tight budget serialises batches and never
  holds more than the budget; a request that cannot fit alone is rejected;
* bad requests fail at submission.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _world(fdzb, scenes, nscenes=3, nviews=4, seed=6000):
    import torch
    sc = [scenes.make_scene(16, 16, [1500, 400, 3000][k % 3], n=8, bins=8, seed=seed + k, sigma=0.12)
          for k in range(nscenes)]
    geo = []
    for s in sc:
        geo.append((torch.from_numpy(s.vtx).cuda(), torch.from_numpy(s.idx).cuda(), s.V, s.T))
    views = []
    sizes = [(96, 64), (128, 128), (200, 120), (64, 48), (160, 90), (144, 144)]
    for v in range(nviews):
        W, H = sizes[v % len(sizes)]
        r = scenes.make_scene(W, H, 1, n=8, bins=8, seed=seed + 100 + v)
        views.append((W, H, torch.from_numpy(r.pos).cuda(), torch.from_numpy(r.nrm).cuda()))
    return sc, geo, views


def _requests(fdzb, scenes, nreq, nscenes, nviews):
    import torch
    reqs = []
    for i in range(nreq):
        n = [4, 8, 16][i % 3]
        light = scenes.Light(right_radius=0.5 + 0.25 * (i % 4), top_radius=0.5 + 0.25 * (i % 4), n=n)
        reqs.append(dict(scene=i % nscenes, view=(i * 7) % nviews, light=light, bins=[8, 16, 32, 0][i % 4]))
    return reqs


def _outputs(fdzb, views, r):
    import torch
    W, H = views[r["view"]][:2]
    sh = torch.full((W * H,), -1.0, dtype=torch.float32, device="cuda")
    mk = torch.zeros(W * H * fdzb.mask_words(r["light"].n), dtype=torch.int32, device="cuda")
    return sh, mk


def _req(fdzb, views, r, sh, mk):
    W, H, pos, nrm = views[r["view"]]
    return fdzb.request(r["scene"], pos, nrm, W, H, r["light"], sh, mk, bins=r["bins"])


def test_results_same_alone_and_in_the_mix(cuda_ok, fdzb, scenes):
    import torch
    sc, geo, views = _world(fdzb, scenes)
    reqs = _requests(fdzb, scenes, 18, len(sc), len(views))
    srv = fdzb.Server(slots=2, max_batch_frames=5)
    for vtx, idx, V, T in geo:
        srv.add_scene(vtx, V, idx, T, cull=False, esp=1e-3)
    # alone: one request on the server at a time
    alone = []
    for r in reqs:
        sh, mk = _outputs(fdzb, views, r)
        res = srv.wait(srv.submit(_req(fdzb, views, r, sh, mk)))
        assert res["status"] == 0 and res["batch_frames"] == 1
        alone.append((sh.cpu().numpy(), mk.cpu().numpy(), res["stats"]["num_bins"]))
    # in the mix: a burst, batched and overlapped
    outs = [_outputs(fdzb, views, r) for r in reqs]
    srv.reset_stats()
    tickets = [srv.submit(_req(fdzb, views, r, *o)) for r, o in zip(reqs, outs)]
    res = [srv.wait(t) for t in tickets]
    st = srv.stats()
    assert all(x["status"] == 0 for x in res)
    assert max(x["batch_frames"] for x in res) > 1, "burst was not batched"
    assert st["completed"] == len(reqs) and st["batches"] < len(reqs)
    for i, (o, a) in enumerate(zip(outs, alone)):
        assert np.array_equal(o[0].cpu().numpy().view(np.uint32), a[0].view(np.uint32)), f"request {i} shadow"
        assert np.array_equal(o[1].cpu().numpy(), a[1]), f"request {i} masks"
    # and a plain single-frame launch of the same inputs
    for i in (0, 5, 11):
        r = reqs[i]
        s = sc[r["scene"]]
        W, H, pos, nrm = views[r["view"]]
        ctx = fdzb.Context()
        sh = torch.empty(W * H, dtype=torch.float32, device="cuda")
        mk = torch.empty(W * H * fdzb.mask_words(r["light"].n), dtype=torch.int32, device="cuda")
        ctx.set_view(W, H)
        ctx.set_bin_num(alone[i][2] and int(round(alone[i][2] ** 0.5)))
        ctx.set_scenes_esp(1e-3)
        ctx.set_backface_cull(False)
        vtx, idx, V, T = geo[r["scene"]]
        ctx.add_model(vtx, V, 16, idx, T)
        ctx.set_sample_buffers(pos, nrm)
        ctx.set_output_buffer(sh, mk)
        ctx.set_area_light(r["light"])
        ctx.launch()
        assert np.array_equal(sh.cpu().numpy().view(np.uint32), alone[i][0].view(np.uint32)), f"plain {i}"
        assert np.array_equal(mk.cpu().numpy(), alone[i][1]), f"plain masks {i}"
        ctx.close()
    srv.close()


def test_overlap_across_slots(cuda_ok, fdzb, scenes):
    sc, geo, views = _world(fdzb, scenes, seed=6100)
    reqs = _requests(fdzb, scenes, 24, len(sc), len(views))
    srv = fdzb.Server(slots=3, max_batch_frames=2)
    for vtx, idx, V, T in geo:
        srv.add_scene(vtx, V, idx, T)
    outs = [_outputs(fdzb, views, r) for r in reqs]
    tickets = [srv.submit(_req(fdzb, views, r, *o)) for r, o in zip(reqs, outs)]
    for t in tickets:
        assert srv.wait(t)["status"] == 0
    st = srv.stats()
    assert st["max_inflight_batches"] >= 2 and st["overlapped_batches"] >= 1, st
    assert st["p99_ms"] >= st["p50_ms"] > 0
    srv.close()


def test_memory_budget_admission_and_rejection(cuda_ok, fdzb, scenes):
    sc, geo, views = _world(fdzb, scenes, seed=6200)
    reqs = _requests(fdzb, scenes, 8, len(sc), len(views))
    # first find what one request needs, then allow a little more than one
    probe = fdzb.Server(slots=1, max_batch_frames=1)
    for vtx, idx, V, T in geo:
        probe.add_scene(vtx, V, idx, T)
    for r in reqs:
        o = _outputs(fdzb, views, r)
        assert probe.wait(probe.submit(_req(fdzb, views, r, *o)))["status"] == 0
    one = probe.stats()["peak_bytes"]
    probe.close()
    budget = int(one * 1.5)
    srv = fdzb.Server(slots=2, max_batch_frames=8, memory_budget_bytes=budget)
    for vtx, idx, V, T in geo:
        srv.add_scene(vtx, V, idx, T)
    outs = [_outputs(fdzb, views, r) for r in reqs]
    tickets = [srv.submit(_req(fdzb, views, r, *o)) for r, o in zip(reqs, outs)]
    res = [srv.wait(t) for t in tickets]
    st = srv.stats()
    assert all(x["status"] == 0 for x in res)
    assert st["peak_bytes"] <= budget, st
    # a budget below one request's needs: rejected, not hung
    tiny = fdzb.Server(slots=1, memory_budget_bytes=1 << 20)
    for vtx, idx, V, T in geo:
        tiny.add_scene(vtx, V, idx, T)
    o = _outputs(fdzb, views, reqs[0])
    r = tiny.wait(tiny.submit(_req(fdzb, views, reqs[0], *o)), timeout_ms=20000)
    assert r is not None and r["status"] == -4
    assert tiny.stats()["rejected"] == 1
    tiny.close()
    srv.close()


def test_bad_requests_fail_at_submission(cuda_ok, fdzb, scenes):
    sc, geo, views = _world(fdzb, scenes, nscenes=1, nviews=1, seed=6300)
    srv = fdzb.Server(slots=1)
    vtx, idx, V, T = geo[0]
    srv.add_scene(vtx, V, idx, T)
    r = _requests(fdzb, scenes, 1, 1, 1)[0]
    sh, mk = _outputs(fdzb, views, r)
    bad = _req(fdzb, views, r, sh, mk)
    bad.scene_id = 7
    with pytest.raises(fdzb.FdzbError):
        srv.submit(bad)
    bad = _req(fdzb, views, r, sh, mk)
    bad.bins = 12
    with pytest.raises(fdzb.FdzbError):
        srv.submit(bad)
    bad = _req(fdzb, views, r, sh, mk)
    bad.light.lightResWidth = 65       # grids are limited to 64 x 64
    bad.light.lightResHeight = 8
    with pytest.raises(fdzb.FdzbError):
        srv.submit(bad)
    srv.close()


def test_rectangular_and_wide_lights_are_served(cuda_ok, fdzb, scenes):
    """Requests with rectangular and 64-bit-row light grids, batched with a
    square one, equal their plain single-frame launches bit for bit."""
    import torch
    sc, geo, views = _world(fdzb, scenes, nscenes=1, nviews=3, seed=6400)
    srv = fdzb.Server(slots=1, max_batch_frames=4)
    vtx, idx, V, T = geo[0]
    srv.add_scene(vtx, V, idx, T, cull=False, esp=1e-3)
    lights = [scenes.Light(n=8), scenes.Light(n=12, nh=40), scenes.Light(n=24, nh=5)]
    outs, tickets = [], []
    for v, light in enumerate(lights):
        W, H, pos, nrm = views[v]
        sh = torch.full((W * H,), -1.0, dtype=torch.float32, device="cuda")
        mk = torch.zeros(W * H * fdzb.mask_words(light.n, light.cols), dtype=torch.int32, device="cuda")
        outs.append((sh, mk))
        tickets.append(srv.submit(fdzb.request(0, pos, nrm, W, H, light, sh, mk, bins=16)))
    for t in tickets:
        assert srv.wait(t)["status"] == 0
    for v, light in enumerate(lights):
        W, H, pos, nrm = views[v]
        ctx = fdzb.Context()
        sh = torch.empty(W * H, dtype=torch.float32, device="cuda")
        mk = torch.empty(W * H * fdzb.mask_words(light.n, light.cols), dtype=torch.int32, device="cuda")
        ctx.set_view(W, H)
        ctx.set_bin_num(16)
        ctx.set_scenes_esp(1e-3)
        ctx.set_backface_cull(False)
        ctx.add_model(vtx, V, 16, idx, T)
        ctx.set_sample_buffers(pos, nrm)
        ctx.set_output_buffer(sh, mk)
        ctx.set_area_light(light)
        ctx.launch()
        assert torch.equal(sh, outs[v][0]), f"light {v} shadow"
        assert torch.equal(mk, outs[v][1]), f"light {v} masks"
        assert float(sh.max()) > 0.0
        ctx.close()
    srv.close()
