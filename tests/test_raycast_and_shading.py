"""The reference's ray-cast cross-check (REF_CAL, K/Step5_2_calRef.inl) and the
shading pass that consumes the shadow buffer (phoneShading.shf).

* ray cast on the GPU equals the oracle's FP32 restatement bit for bit (masks and
  shadows), in both triangle orders;
* ray cast and edge-function masks agree except for light samples next to a
  projected edge (at most 1e-3 of the set bits differ here);
* shading matches a float64 restatement of the shader within 1e-4 relative,
  and leaves pixels with a NaN shadow untouched.
"""
import dataclasses

import numpy as np
import pytest

import oracle


def test_light_sample_positions_formula(fdzb, scenes):
    L = scenes.Light(right_radius=1.5, top_radius=0.75, n=4, position=(0.2, -0.1, 6.0))
    p = fdzb.light_sample_positions(L)
    s = fdzb.light_setup(L)
    ur, (xd, yd) = s["corners"][0], s["deltas"]
    for i in range(4):
        for j in range(4):
            want = (ur + xd * np.float32(j)).astype(np.float32) + (yd * np.float32(i)).astype(np.float32)
            assert np.array_equal(p[i * 4 + j], want.astype(np.float32))


def _gpu_raycast(fdzb, scene, order):
    ctx, t = fdzb.context_for_scene(scene, masks=True, tri_order=order)
    ctx.set_shadow_method(fdzb.SHADOW_RAY_CAST)
    ctx.launch()
    out = t["shadow"].cpu().numpy(), t["masks"].cpu().numpy().view(np.uint32)
    ctx.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("n,bins", [(4, 8), (8, 16), (16, 16)])
@pytest.mark.parametrize("order", [0, 1])
def test_raycast_matches_oracle(cuda_ok, fdzb, scenes, n, bins, order):
    s = scenes.make_scene(160, 120, 1500, n=n, bins=bins, seed=400 + n, sigma=0.12)
    sh, mk = _gpu_raycast(fdzb, s, order)
    o = oracle.frame(s, shadow_method=1)
    assert np.array_equal(sh.view(np.uint32), o.arrays["shadow"].astype(np.float32).view(np.uint32))
    assert np.array_equal(mk, o.arrays["masks"].astype(np.uint32)[: mk.size])


@pytest.mark.gpu
def test_raycast_cross_checks_edge_masks(cuda_ok, fdzb, scenes):
    s = scenes.make_scene(320, 240, 8000, n=16, bins=32, seed=410, sigma=0.1)
    sh_r, mk_r = _gpu_raycast(fdzb, s, 1)
    ctx, t = fdzb.context_for_scene(s, masks=True)
    ctx.launch()
    mk_e = t["masks"].cpu().numpy().view(np.uint32)
    ctx.close()
    set_bits = int(np.unpackbits(mk_e.view(np.uint8)).sum())
    diff = int(np.unpackbits((mk_e ^ mk_r).view(np.uint8)).sum())
    assert set_bits > 10000
    assert diff <= 1e-3 * set_bits, (diff, set_bits)


def _shade_ref(g0, g1, g2, g3, shadow, cam, La, Ld, Ls, lights):
    g0, g1, g2, g3 = (x.astype(np.float64) for x in (g0, g1, g2, g3))
    I = 1.0 - shadow.astype(np.float64)
    wp, N = g0[:, :3], g1[:, :3] / np.linalg.norm(g1[:, :3], axis=1, keepdims=True)
    ka, kd, ks, sh = g2[:, :3], g3[:, :3], np.stack([g0[:, 3], g1[:, 3], g2[:, 3]], 1), g3[:, 3:4]
    V = np.asarray(cam, np.float64) - wp
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    acc = np.zeros_like(wp)
    for lp in lights.astype(np.float64):
        L = lp - wp
        L /= np.linalg.norm(L, axis=1, keepdims=True)
        ldn = np.sum(L * N, 1, keepdims=True)
        R = 2 * ldn * N - L
        spec = np.power(np.maximum(np.sum(R * V, 1, keepdims=True), 0.0), sh)
        acc += np.asarray(La) * ka + (np.asarray(Ld) * kd * np.maximum(ldn, 0) + np.asarray(Ls) * ks * spec) * I[:, None]
    return acc / len(lights)


@pytest.mark.gpu
@pytest.mark.parametrize("nl", [1, 16])
def test_shading_matches_float64_restatement(cuda_ok, fdzb, scenes, nl):
    import torch
    s = scenes.make_scene(128, 96, 1500, n=4, bins=16, seed=420, sigma=0.12)
    ctx, t = fdzb.context_for_scene(s, masks=False)
    ctx.launch()
    shadow = t["shadow"].clone()
    shadow[:7] = float("nan")                       # discarded pixels
    ctx.close()
    rng = np.random.default_rng(421)
    S = s.S
    g0 = np.concatenate([s.pos[:, :3], rng.uniform(0, 1, (S, 1))], 1).astype(np.float32)
    g1 = np.concatenate([s.nrm[:, :3], rng.uniform(0, 1, (S, 1))], 1).astype(np.float32)
    g2 = rng.uniform(0, 0.3, (S, 4)).astype(np.float32)
    g3 = np.concatenate([rng.uniform(0, 1, (S, 3)), rng.uniform(1, 40, (S, 1))], 1).astype(np.float32)
    lights = fdzb.light_sample_positions(dataclasses.replace(s.light, n=4))[:nl].copy()
    cam, La, Ld, Ls = (0.5, -3.0, 9.0), (0.2, 0.2, 0.25), (0.8, 0.7, 0.6), (0.5, 0.5, 0.5)
    dev = lambda a: torch.from_numpy(a).cuda()
    rgba = torch.full((S, 4), -7.0, dtype=torch.float32, device="cuda")
    fdzb.shade(s.W, s.H, dev(g0), dev(g1), dev(g2), dev(g3), shadow, rgba, cam, La, Ld, Ls, dev(lights))
    torch.cuda.synchronize()
    out = rgba.cpu().numpy()
    assert np.all(out[:7] == -7.0)                  # untouched
    want = _shade_ref(g0[7:], g1[7:], g2[7:], g3[7:], shadow.cpu().numpy()[7:], cam, La, Ld, Ls, lights)
    np.testing.assert_allclose(out[7:, :3], want, rtol=1e-4, atol=1e-5)
    assert np.all(out[7:, 3] == 1.0)
