"""fdzb_sort_pairs_noalloc: the sort for callers that cannot allocate device memory.

Some callers may not call cudaMalloc/cudaFree (a host-owned allocator or pool,
a plugin inside another process's memory budget, a real-time loop that must not
synchronise for cudaFree).  This entry point sorts with a fixed scratch area
built into the library.  Its results must equal the frame pipeline's own sort,
read back through fdzb_ctx_export, on two calls in a row (the calls share the
scratch area and the second must not see the first one's leftovers), and a
stable argsort for every pass count (1 to 4 digit passes), ragged last tiles,
the largest size and n = 0.

This file is named to be collected last: if it fails, a run that stops at the
first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_PAIRS = 1 << 20


def _bind(lib):
    lib.fdzb_sort_pairs_noalloc.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int32, ctypes.c_uint32,
                                                                    ctypes.c_void_p, ctypes.c_void_p]
    lib.fdzb_sort_pairs_noalloc.restype = ctypes.c_int
    return lib


def _noalloc(lib, keys, vals, key_range):
    import torch
    n = keys.size
    kin = torch.from_numpy(keys.astype(np.uint32).view(np.int32)).cuda()
    vin = torch.from_numpy(vals.astype(np.uint32).view(np.int32)).cuda()
    kout = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    vout = torch.full((max(n, 1),), -1, dtype=torch.int32, device="cuda")
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.fdzb_sort_pairs_noalloc(kin.data_ptr(), vin.data_ptr(), kout.data_ptr(), vout.data_ptr(),
                                     n, key_range, ctypes.c_void_p(stream), status.data_ptr())
    assert rc == 0, lib.fdzb_last_error().decode()
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    inputs = (kin.cpu().numpy().view(np.uint32), vin.cpu().numpy().view(np.uint32))
    return kout.cpu().numpy().view(np.uint32)[:n], vout.cpu().numpy().view(np.uint32)[:n], inputs


def test_noalloc_sort_matches_pipeline_sort_twice(cuda_ok, fdzb, scenes):
    lib = _bind(fdzb.load())
    scene = scenes.preset("small")
    ctx, _ = fdzb.context_for_scene(scene, debug=True, tri_order=fdzb.TRI_ORDER_REFERENCE)
    ctx.launch()
    st = ctx.stats()
    S, NB, P = scene.S, scene.bins * scene.bins, st["num_pairs"]
    assert st["state"] == 2 and P > 0

    # call 1: (bin key, sample position) pairs of the frame, S = 65,536
    keys = ctx.export("sample_keys", S)
    k1, v1, inputs = _noalloc(lib, keys, np.arange(S, dtype=np.int32), NB + 1)
    assert np.array_equal(k1, ctx.export("sorted_sample_keys", S).view(np.uint32))
    assert np.array_equal(v1, ctx.export("sorted_sample_ids", S).view(np.uint32))
    assert np.array_equal(inputs[0], keys.view(np.uint32))              # inputs untouched

    # call 2, same scratch: (bin, triangle) pairs in triangle order
    pk = ctx.export("pair_bin", P)
    pt = ctx.export("pair_tri", P)
    k2, v2, _ = _noalloc(lib, pk, pt, NB)
    assert np.array_equal(k2, ctx.export("sorted_pair_bin", P).view(np.uint32))
    assert np.array_equal(v2, ctx.export("sorted_pair_tri", P).view(np.uint32))
    ctx.close()


# (n, key_range): 1, 2, 3 and 4 digit passes (an odd pass count goes out ->
# scratch -> out), tiles of 4096 keys with a ragged last tile, the largest n.
CASES = [(4097, 200), (65536, 1 << 16), (100003, (1 << 17) + 1), (1048575, 0xFFFFFFFF),
         (MAX_PAIRS, (1 << 24) + 7), (1, 5), (0, 16)]


@pytest.mark.parametrize("n,key_range", CASES)
def test_noalloc_sort_equals_stable_argsort(cuda_ok, fdzb, n, key_range):
    lib = _bind(fdzb.load())
    rng = np.random.default_rng(n + key_range)
    # many repeated keys, so that stability is visible
    distinct = rng.integers(0, key_range, size=max(1, min(n // 8 + 1, 1 << 16)), dtype=np.uint64)
    keys = distinct[rng.integers(0, distinct.size, size=n)].astype(np.uint32)
    if n:
        keys[0] = key_range - 1
    vals = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    order = np.argsort(keys, kind="stable")
    for _ in range(2):   # two calls in a row on the shared scratch
        k, v, (kin, vin) = _noalloc(lib, keys, vals, key_range)
        assert np.array_equal(k, keys[order])
        assert np.array_equal(v, vals[order])
        assert np.array_equal(kin, keys) and np.array_equal(vin, vals)


def test_noalloc_sort_rejects_more_than_its_scratch_holds(cuda_ok, fdzb):
    lib = _bind(fdzb.load())
    big = MAX_PAIRS + 1
    rc = lib.fdzb_sort_pairs_noalloc(None, None, None, None, big, 16, None, None)
    assert rc == -1
    assert b"1048576" in lib.fdzb_last_error()
