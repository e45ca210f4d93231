"""Look-back tags across the clearing point of the launch number.

The radix sorts and the pair scan find their tiles' offsets by a decoupled
look-back whose status words carry the context's launch number and are never
cleared between launches.  Before the number could wrap round (a tag equal to a
stale word's), the library clears the words and restarts the number.  These
tests move the number to just below that point, launch across it, and require
every launch to give the oracle's sorted lists, masks and shadows.
"""
import numpy as np
import pytest
import torch

import oracle
from tests import parity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("graph", [True, False])
def test_launches_across_the_epoch_limit(cuda_ok, fdzb, scenes, graph):
    scene = scenes.preset("small")
    orc = oracle.frame(scene)
    # debug capture (the exported intermediates) turns graphs off: the graph
    # run compares masks and shadows, the other one every stage
    ctx, t = fdzb.context_for_scene(scene, debug=not graph, tri_order=fdzb.TRI_ORDER_REFERENCE)
    ctx.set_graph(graph)
    ctx.launch()
    first = parity.collect(ctx, t, scene, intermediates=not graph)
    errs = parity.compare(scene, gpu=first, orc=orc)
    assert not errs, "\n".join(errs)

    limit = fdzb.LOOKBACK_EPOCH_LIMIT
    ctx.set_launch_epoch(limit - 2)
    seen = []
    for _ in range(5):
        t["masks"].fill_(-1)
        t["shadow"].fill_(-1.0)
        ctx.launch()
        seen.append(ctx.launch_epoch())
        again = parity.collect(ctx, t, scene, intermediates=not graph)
        errs = parity.compare(scene, gpu=again, orc=orc)
        assert not errs, "\n".join(errs)
    # limit - 1, limit, then cleared and restarted at 1
    assert seen == [limit - 1, limit, 1, 2, 3]
    ctx.close()


def test_epoch_setter_checks_its_argument(cuda_ok, fdzb, scenes):
    scene = scenes.make_scene(64, 48, 50, n=4, bins=8, seed=3)
    ctx, _ = fdzb.context_for_scene(scene)
    with pytest.raises(fdzb.FdzbError):
        ctx.set_launch_epoch(5)          # no launch yet: no arena
    ctx.launch()
    with pytest.raises(fdzb.FdzbError):
        ctx.set_launch_epoch(fdzb.LOOKBACK_EPOCH_LIMIT)
    ctx.close()
    torch.cuda.synchronize()
