"""The G-buffer rasteriser on the GPU (fdzb_raster_*), against its oracle.

Every G-buffer target and the depth buffer equal the oracle's
(oracle/fdzb_raster_oracle.c) bit for bit: cameras above, beside and inside
the scene (near-plane clipping), views that are not multiples of the 16-pixel
tile, draws on top of earlier draws.  End to end, the rasterised view feeds the
shadow pipeline (g0 and g1 are its sample buffers) and the shading pass: the
shadows equal the shadow oracle's on the oracle's own G-buffer.
"""
import dataclasses
import importlib

import numpy as np
import pytest

import oracle
from oracle import orc

pytestmark = pytest.mark.gpu
scenes = importlib.import_module("4dzb_b200.scenes")


def _dev(fdzb, ms, rows=None):
    import torch
    rows = slice(None) if rows is None else rows
    return dict(vtx=torch.from_numpy(ms.vtx).cuda(),
                idx=torch.from_numpy(np.ascontiguousarray(ms.idx[rows]).view(np.int32)).cuda(),
                tm=torch.from_numpy(np.ascontiguousarray(ms.tri_material[rows])).cuda(),
                mats=torch.from_numpy(ms.materials).cuda())


def _targets(ms, with23=True):
    import torch
    S = ms.W * ms.H
    t = {k: torch.empty((S, 4), dtype=torch.float32, device="cuda") for k in ("g0", "g1")}
    t["g2"] = torch.empty((S, 4), dtype=torch.float32, device="cuda") if with23 else None
    t["g3"] = torch.empty((S, 4), dtype=torch.float32, device="cuda") if with23 else None
    t["depth"] = torch.empty(S, dtype=torch.float32, device="cuda")
    return t


def _draw(fdzb, r, ms, t, dev, n_tri, clear=True):
    d = fdzb.raster_desc(dev["vtx"], ms.vtx.shape[0], dev["idx"], n_tri, dev["mats"], ms.materials.shape[0],
                         ms.model, ms.view_proj, ms.W, ms.H, t["g0"], t["g1"], t["g2"], t["g3"], t["depth"],
                         clear=clear, tri_material=dev["tm"])
    r.draw(d)
    r.sync()


def _same(gpu, cpu, what):
    a = gpu.cpu().numpy().view(np.uint32)
    b = np.ascontiguousarray(cpu, np.float32).reshape(a.shape).view(np.uint32)
    bad = np.flatnonzero(a != b)
    assert bad.size == 0, f"{what}: {bad.size} words differ, first {bad[:5].tolist()}"


@pytest.mark.parametrize("W,H,eye,center", [
    (160, 120, (0.0, -13.0, 11.0), (0.0, 0.0, 0.0)),
    (333, 177, (3.0, -6.0, 2.5), (0.0, 0.0, 0.0)),
    (200, 150, (0.0, -7.5, 0.6), (0.0, 8.0, 0.0)),     # inside the scene: near-plane clipping
    (64, 64, (0.0, -1.0, 20.0), (0.0, 0.0, 0.0)),
])
@pytest.mark.parametrize("with23", [True, False])
def test_raster_matches_oracle(cuda_ok, fdzb, W, H, eye, center, with23):
    ms = scenes.mesh_scene(W, H, eye=eye, center=center)
    dev, t = _dev(fdzb, ms), _targets(ms, with23)
    r = fdzb.Raster()
    _draw(fdzb, r, ms, t, dev, ms.T)
    st = r.stats()
    o = orc.raster(ms.vtx, ms.idx, ms.materials, ms.model, ms.view_proj, W, H, tri_material=ms.tri_material)
    assert st["sub_triangles"] == o["sub_tris"] and st["dropped"] == o["dropped"]
    assert st["bad_indices"] == 0 and st["bad_materials"] == 0
    for k in ("g0", "g1", "depth") + (("g2", "g3") if with23 else ()):
        _same(t[k], o[k], k)
    r.close()


def test_draw_on_top_of_an_earlier_draw(cuda_ok, fdzb):
    ms = scenes.mesh_scene(150, 110)
    k = ms.n_receiver
    t = _targets(ms)
    r = fdzb.Raster()
    _draw(fdzb, r, ms, t, _dev(fdzb, ms, slice(0, k)), k)
    _draw(fdzb, r, ms, t, _dev(fdzb, ms, slice(k, None)), ms.T - k, clear=False)
    whole = orc.raster(ms.vtx, ms.idx, ms.materials, ms.model, ms.view_proj, ms.W, ms.H,
                       tri_material=ms.tri_material)
    for key in ("g0", "g1", "g2", "g3", "depth"):
        _same(t[key], whole[key], key)
    r.close()


def test_bad_inputs_are_rejected(cuda_ok, fdzb):
    ms = scenes.mesh_scene(32, 32, T=10)
    dev, t = _dev(fdzb, ms), _targets(ms)
    r = fdzb.Raster()
    d = fdzb.raster_desc(dev["vtx"], ms.vtx.shape[0], dev["idx"], ms.T, dev["mats"], 2, ms.model, ms.view_proj,
                         32, 32, t["g0"], t["g1"], clear=False)
    with pytest.raises(fdzb.FdzbError):   # no depth buffer to draw on top of
        r.draw(d)
    d = fdzb.raster_desc(dev["vtx"], ms.vtx.shape[0], dev["idx"], ms.T, dev["mats"], 2, ms.model, ms.view_proj,
                         32, 32, t["g0"], t["g1"], nrm_offset=6)
    with pytest.raises(fdzb.FdzbError):   # normal runs past the 8-float vertex
        r.draw(d)
    r.close()


def test_rasterised_view_through_shadows_and_shading(cuda_ok, fdzb):
    """The app's frame without GL: pass 0 (G-buffer), FDLaunch (shadows) and
    pass 1 (shading).  The shadows equal the shadow oracle's on the oracle's
    G-buffer, bit for bit."""
    import torch
    ms = scenes.mesh_scene(256, 192, T=2000)
    dev, t = _dev(fdzb, ms), _targets(ms)
    r = fdzb.Raster()
    _draw(fdzb, r, ms, t, dev, ms.T)
    o = orc.raster(ms.vtx, ms.idx, ms.materials, ms.model, ms.view_proj, ms.W, ms.H, tri_material=ms.tri_material)
    sc = scenes.shadow_scene(ms, o["g0"], o["g1"], bins=32)
    ctx, tt = fdzb.context_for_scene(sc, masks=True)
    ctx.set_sample_buffers(t["g0"], t["g1"])      # the rasteriser's own output, on the device
    ctx.launch()
    sh = tt["shadow"]
    ref = oracle.frame(sc)
    _same(sh, ref.arrays["shadow"], "shadow")
    assert 0.01 < float(ref.arrays["shadow"][~np.isnan(o["g0"][:, 0])].mean()) < 0.99
    # pass 1: Phong with the visibility, one light sample at the light's centre
    rgba = torch.empty((ms.W * ms.H, 4), dtype=torch.float32, device="cuda")
    lights = torch.tensor([list(ms.light.position)], dtype=torch.float32, device="cuda")
    fdzb.shade(ms.W, ms.H, t["g0"], t["g1"], t["g2"], t["g3"], sh, rgba, ms.eye, (0.2, 0.2, 0.2),
               (0.8, 0.8, 0.8), (0.5, 0.5, 0.5), lights)
    torch.cuda.synchronize()
    out = rgba.cpu().numpy()
    cov = ~np.isnan(o["g0"][:, 0])
    assert np.isfinite(out[cov]).all()
    ctx.close()
    r.close()
