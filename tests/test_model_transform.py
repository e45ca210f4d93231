"""Model transform applied as the vertices are read (fdzb_ctx_set_model_transform,
fdzb_frame_desc.model_transform, fdzb_request.model_transform).

The reference animates a scene by rewriting its vertex buffer in place
(FD::moveModel, K/moveModel.inl).  Reading the vertices through the same
transform must give the same floats, so a launch with the transform equals, bit
for bit, moveModel on a copy of the buffer followed by a launch -- and the
oracle run on the moved vertices.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _matrix(angle=0.3, t=(0.4, -0.25, 0.15), s=1.05):
    c, si = np.cos(angle), np.sin(angle)
    m = np.eye(4, dtype=np.float32)
    m[:3, :3] = s * np.array([[c, -si, 0.0], [si, c, 0.0], [0.0, 0.0, 1.0]], np.float32)
    m[:3, 3] = t
    return m.T.reshape(16).copy()        # column-major, as moveModel takes it


def _moved_vertices(vtx, m):
    """The reference's in-place transform, as the oracle restates it (float32,
    each component summed left to right)."""
    M = np.asarray(m, np.float32)
    out = vtx.copy()
    x, y, z = vtx[:, 0], vtx[:, 1], vtx[:, 2]
    one = np.float32(1.0)
    for r in range(3):
        acc = (M[r] * x).astype(np.float32)
        acc = (acc + (M[4 + r] * y).astype(np.float32)).astype(np.float32)
        acc = (acc + (M[8 + r] * z).astype(np.float32)).astype(np.float32)
        out[:, r] = (acc + (M[12 + r] * one).astype(np.float32)).astype(np.float32)
    return out


def test_context_transform_equals_move_model(cuda_ok, fdzb, scenes):
    import dataclasses
    s = scenes.make_scene(200, 150, 3000, n=8, bins=16, seed=301, sigma=0.12)
    m = _matrix()
    ctx, t = fdzb.context_for_scene(s, masks=True)
    ctx.set_model_transform(m)
    ctx.launch()
    a_sh, a_mk = t["shadow"].cpu().numpy().copy(), t["masks"].cpu().numpy().copy()
    # second launch (graph replay) with the same transform
    ctx.launch()
    assert np.array_equal(t["masks"].cpu().numpy(), a_mk)
    ctx.close()
    ctx2, t2 = fdzb.context_for_scene(s, masks=True)
    ctx2.move_model(m)                      # in place, like the reference
    ctx2.launch()
    assert np.array_equal(t2["shadow"].cpu().numpy().view(np.uint32), a_sh.view(np.uint32))
    assert np.array_equal(t2["masks"].cpu().numpy(), a_mk)
    ctx2.close()
    moved = dataclasses.replace(s, vtx=_moved_vertices(s.vtx, m))
    o = oracle.frame(moved)
    assert np.array_equal(a_sh.view(np.uint32), o.arrays["shadow"].astype(np.float32).view(np.uint32))


def test_transform_changes_per_launch_and_clears(cuda_ok, fdzb, scenes):
    s = scenes.make_scene(160, 120, 2000, n=8, bins=16, seed=302, sigma=0.12)
    ctx, t = fdzb.context_for_scene(s, masks=True)
    ctx.launch()
    plain = t["masks"].cpu().numpy().copy()
    outs = []
    for k in range(3):
        ctx.set_model_transform(_matrix(angle=0.1 * (k + 1), t=(0.1 * k, 0.0, 0.0)))
        ctx.launch()
        outs.append(t["masks"].cpu().numpy().copy())
    assert not np.array_equal(outs[0], outs[1])
    ctx.set_model_transform(None)
    ctx.launch()
    assert np.array_equal(t["masks"].cpu().numpy(), plain)
    ctx.close()


def test_batch_and_request_transforms(cuda_ok, fdzb, scenes):
    import torch
    s = scenes.make_scene(128, 96, 1500, n=8, bins=16, seed=303, sigma=0.12)
    m = _matrix(angle=-0.2)
    ctx, t = fdzb.context_for_scene(s, masks=True)
    ctx.set_model_transform(m)
    ctx.launch()
    want = t["masks"].cpu().numpy().copy()
    ctx.close()
    pos, nrm, vtx, idx = fdzb.upload_scene(s)
    sh = torch.empty(s.S, dtype=torch.float32, device="cuda")
    mk = torch.empty(s.S * fdzb.mask_words(8), dtype=torch.int32, device="cuda")
    b = fdzb.Batch()
    d = fdzb.frame_desc(pos, nrm, s.W, s.H, vtx, s.V, idx, s.T, s.light, sh, mk, bins=16, esp=s.esp,
                        model_transform=m)
    b.launch([d])
    assert np.array_equal(mk.cpu().numpy(), want)
    b.close()
    srv = fdzb.Server(slots=1)
    sid = srv.add_scene(vtx, s.V, idx, s.T, cull=False, esp=s.esp)
    mk.zero_()
    r = srv.wait(srv.submit(fdzb.request(sid, pos, nrm, s.W, s.H, s.light, sh, mk, bins=16, model_transform=m)))
    assert r["status"] == 0
    assert np.array_equal(mk.cpu().numpy(), want)
    srv.close()
