"""fdzb_sort_pairs_noalloc: the sort for callers that cannot allocate device memory.

Some callers may not call cudaMalloc/cudaFree (a host-owned allocator or pool,
a plugin inside another process's memory budget, a real-time loop that must not
synchronise for cudaFree).  This entry point sorts with a fixed scratch area
built into the library.  Its results must equal the frame pipeline's own sort,
read back through fdzb_ctx_export, on two calls in a row (the calls share the
scratch area and the second must not see the first one's leftovers).

This file is named to be collected last: if it fails, a run that stops at the
first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(lib, keys, vals, key_range):
    import torch
    n = keys.size
    kin = torch.from_numpy(keys.astype(np.int32)).cuda()
    vin = torch.from_numpy(vals.astype(np.int32)).cuda()
    kout = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    vout = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.fdzb_sort_pairs_noalloc(kin.data_ptr(), vin.data_ptr(), kout.data_ptr(), vout.data_ptr(),
                                     n, key_range, ctypes.c_void_p(stream), status.data_ptr())
    assert rc == 0, lib.fdzb_last_error().decode()
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return kout.cpu().numpy()[:n], vout.cpu().numpy()[:n], (kin.cpu().numpy(), vin.cpu().numpy())


def test_noalloc_sort_matches_pipeline_sort_twice(cuda_ok, fdzb, scenes):
    lib = fdzb.load()
    lib.fdzb_sort_pairs_noalloc.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int32, ctypes.c_uint32,
                                                                    ctypes.c_void_p, ctypes.c_void_p]
    lib.fdzb_sort_pairs_noalloc.restype = ctypes.c_int
    scene = scenes.preset("small")
    ctx, _ = fdzb.context_for_scene(scene, debug=True, tri_order=fdzb.TRI_ORDER_REFERENCE)
    ctx.launch()
    st = ctx.stats()
    S, NB, P = scene.S, scene.bins * scene.bins, st["num_pairs"]
    assert st["state"] == 2 and P > 0

    # call 1: (bin key, sample position) pairs of the frame, S = 65,536
    keys = ctx.export("sample_keys", S)
    k1, v1, inputs = _noalloc(lib, keys, np.arange(S, dtype=np.int32), NB + 1)
    assert np.array_equal(k1, ctx.export("sorted_sample_keys", S))
    assert np.array_equal(v1, ctx.export("sorted_sample_ids", S))
    assert np.array_equal(inputs[0], keys)              # inputs untouched

    # call 2, same scratch: (bin, triangle) pairs in triangle order
    pk = ctx.export("pair_bin", P)
    pt = ctx.export("pair_tri", P)
    k2, v2, _ = _noalloc(lib, pk, pt, NB)
    assert np.array_equal(k2, ctx.export("sorted_pair_bin", P))
    assert np.array_equal(v2, ctx.export("sorted_pair_tri", P))
    ctx.close()


def test_noalloc_sort_rejects_more_than_its_scratch_holds(cuda_ok, fdzb):
    lib = fdzb.load()
    lib.fdzb_sort_pairs_noalloc.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int32, ctypes.c_uint32,
                                                                    ctypes.c_void_p, ctypes.c_void_p]
    lib.fdzb_sort_pairs_noalloc.restype = ctypes.c_int
    big = (1 << 20) + 1
    rc = lib.fdzb_sort_pairs_noalloc(None, None, None, None, big, 16, None, None)
    assert rc == -1
    assert b"1048576" in lib.fdzb_last_error()
