"""Scenes at extreme coordinate scales: the row quotient's slow path.

The pair test takes the rows' quotient from a hoisted reciprocal only where the
pair's edge coefficients lie in the ranges that make that exact (|A|, |C| in
[2^-38, 2^40], |B| in [2^-100, 2^39]); elsewhere it divides.  The coefficients
are products of three coordinate differences, so the small scene scaled by
2^16 (coordinates near 5e5) puts nearly every pair above the range and scaled
by 2^-16 below it.  Both frames must still equal the oracle bit for bit, as
every in-range frame does.  Scaling by a power of two changes no rounding of
the scene's own data, so the scaled frames are valid inputs of the same kind.
"""
import dataclasses

import numpy as np
import pytest

import oracle
from tests import parity

pytestmark = pytest.mark.gpu


def scaled(scene, k):
    f = np.float32(2.0 ** k)
    pos = scene.pos.copy()
    vtx = scene.vtx.copy()
    pos[:, :3] *= f
    vtx[:, :3] *= f
    li = scene.light
    light = dataclasses.replace(li, right_radius=li.right_radius * float(f), top_radius=li.top_radius * float(f),
                                position=tuple(float(np.float32(p) * f) for p in li.position))
    return dataclasses.replace(scene, pos=pos, vtx=vtx, light=light, esp=float(np.float32(scene.esp) * f),
                               name=f"{scene.name}x2^{k}")


@pytest.mark.parametrize("k", [16, -16])
@pytest.mark.parametrize("order", [0, 1])
def test_scaled_scene_equals_oracle(cuda_ok, fdzb, scenes, k, order):
    s = scaled(scenes.preset("small"), k)
    orc = oracle.frame(s)
    ctx, t = fdzb.context_for_scene(s, masks=True, tri_order=order)
    ctx.launch()
    errs = parity.compare(s, gpu=parity.collect(ctx, t, s, tri_order=order, intermediates=False), orc=orc)
    ctx.close()
    assert not errs, "\n".join(errs)
    assert (orc.arrays["shadow"] > 0).any()     # the frame has shadows to compare
