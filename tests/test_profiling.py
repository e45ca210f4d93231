"""Profiling modes and the two forms of the occlusion kernel.

The occlusion kernel runs in a form that accumulates the work counters (pair
tests, light rows, partial row masks) only when profiling asks for them; every
other launch runs the form without them.  Both forms must give the same masks
and shadows, the counters must be filled exactly in the counting mode, and the
stage-timing mode must time the stages without counting.
"""
import numpy as np
import pytest

import oracle
from tests import parity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", ["small", "odd"])
def test_counting_and_plain_kernels_agree(cuda_ok, fdzb, scenes, which):
    if which == "small":
        scene = scenes.preset("small")
    else:
        scene = scenes.make_scene(301, 77, 4000, n=16, bins=16, seed=9, sigma=0.1)
    orc = oracle.frame(scene)
    ctx, t = fdzb.context_for_scene(scene, masks=True)
    seen = {}
    for mode in (fdzb.PROFILE_OFF, fdzb.PROFILE_ALL, fdzb.PROFILE_STAGES, fdzb.PROFILE_OFF):
        ctx.set_profiling(mode)
        t["masks"].zero_()
        t["shadow"].fill_(-1.0)
        ctx.launch()
        st = ctx.stats()
        errs = parity.compare(scene, gpu=parity.collect(ctx, t, scene, intermediates=False), orc=orc)
        assert not errs, (mode, errs)
        seen.setdefault(mode, []).append((t["masks"].cpu().numpy().copy(), st))
        if mode == fdzb.PROFILE_ALL:
            assert st["pair_tests"] > 0 and st["rows_evaluated"] > 0 and st["partial_masks"] > 0
            assert all(x > 0 for x in st["stage_ms"])
        elif mode == fdzb.PROFILE_STAGES:
            assert st["pair_tests"] == 0 and st["rows_evaluated"] == 0
            assert all(x > 0 for x in st["stage_ms"])
        else:
            assert st["pair_tests"] == 0 and st["rows_evaluated"] == 0
    ref = seen[fdzb.PROFILE_ALL][0][0]
    for mode, runs in seen.items():
        for masks, _ in runs:
            assert np.array_equal(masks, ref), mode
    ctx.close()


def test_profiling_mode_out_of_range(cuda_ok, fdzb, scenes):
    ctx, _ = fdzb.context_for_scene(scenes.preset("small"))
    with pytest.raises(RuntimeError):
        ctx.set_profiling(3)
    ctx.close()
