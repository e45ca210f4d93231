"""Golden fixtures produced by the reference's own sources (tests/golden/make_golden.py,
4DZB's kernels and FD:: host code compiled for the CPU by oracle/ref_emu).

* the oracle reproduces every stored stage bit for bit (CPU);
* the CUDA pipeline reproduces every stored stage bit for bit (GPU), in the
  reference's triangle order and, for masks and shadows, in coverage order;
* where the reference sources are present, the harness rebuilt here
  reproduces the fixtures (pins the fixtures to the sources).
"""
import glob
import importlib
import os

import numpy as np
import pytest

import oracle
from oracle.refpath import reference_present

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
STAGES = ["sorted_keys", "sorted_vals", "bin_sample_start", "bin_sample_end", "bin_maxz", "bin_range",
          "tri_aabb", "tri_count", "sorted_pair_bin", "sorted_pair_tri", "bin_tri_start", "bin_tri_end",
          "shadow"]


def _scene(z):
    scenes = importlib.import_module("4dzb_b200.scenes")
    L = z["light"]
    light = scenes.Light(right_radius=float(L[0]), top_radius=float(L[1]), position=tuple(L[2:5]),
                         view_dir=tuple(L[5:8]), up_dir=tuple(L[8:11]), n=int(z["N"]))
    return scenes.Scene(W=int(z["W"]), H=int(z["H"]), pos=z["pos"], nrm=z["nrm"], vtx=z["vtx"], idx=z["idx"],
                        light=light, bins=int(z["bins"]), esp=float(z["esp"]), cull=bool(z["cull"]),
                        name=os.path.basename(str(z.fid.name)) if hasattr(z, "fid") else "golden")


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind == "f":
        return np.array_equal(a.view(np.uint32), b.astype(np.float32).view(np.uint32)) or \
            np.array_equal(a, b, equal_nan=True)
    return np.array_equal(a, b)


def test_fixtures_exist():
    assert len(FIXTURES) >= 5


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_oracle_matches_reference_fixture(path):
    z = np.load(path)
    s = _scene(z)
    fr = oracle.frame(s)
    assert fr.scalars["state"] == 2
    for k in STAGES:
        assert _same(fr.arrays[k], z["ref_" + k]), k
    assert fr.scalars["num_pairs"] == int(z["ref_num_pairs"])
    assert fr.scalars["valid_samples"] == int(z["ref_valid_samples"])
    assert fr.scalars["valid_tris"] == int(z["ref_valid_tris"])
    L = oracle.light_setup(s.light)
    assert _same(np.array(L.mat, np.float32), z["ref_mat"])
    assert _same(np.array(L.RF, np.float32), z["ref_RF"])
    assert _same(np.array(fr.scalars["sub"], np.float32), z["ref_sub"])
    assert _same(np.array(fr.scalars["lp_begin"], np.float32), z["ref_lp_begin"])
    assert _same(np.array(fr.scalars["lp_end"], np.float32), z["ref_lp_end"])
    assert _same(np.array(fr.scalars["lp_factor"], np.float32), z["ref_lp_factor"])


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_library_light_setup_matches_reference_fixture(fdzb, path):
    z = np.load(path)
    s = _scene(z)
    L = fdzb.light_setup(s.light)
    assert _same(L["mat"], z["ref_mat"]) and _same(L["RF"], z["ref_RF"])
    assert _same(L["corners"].ravel(), z["ref_corners"]) and _same(L["deltas"].ravel(), z["ref_deltas"])


@pytest.mark.skipif(not reference_present(), reason="reference sources not present")
def test_reference_harness_reproduces_fixtures():
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref not built")
    for path in FIXTURES:
        z = np.load(path)
        r = ref.run(_scene(z))
        assert r["errors"] == 0
        for k in STAGES:
            assert _same(r[k], z["ref_" + k]), (path, k)


@pytest.mark.gpu
@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_cuda_pipeline_matches_reference_fixture(cuda_ok, path, order):
    from tests import parity
    z = np.load(path)
    s = _scene(z)
    out, st, ex = parity.run_gpu(s, tri_order=order)
    assert st["state"] == 2
    assert st["num_pairs"] == int(z["ref_num_pairs"])
    assert st["valid_samples"] == int(z["ref_valid_samples"])
    assert st["valid_triangles"] == int(z["ref_valid_tris"])
    W, l2 = s.W, int(z["ref_view_log2up"])
    sv = z["ref_sorted_vals"]
    assert _same(ex["sorted_sample_keys"], z["ref_sorted_keys"])
    assert _same(ex["sorted_sample_ids"], (sv >> l2) * W + (sv & ((1 << l2) - 1)))
    for k in ("bin_sample_start", "bin_sample_end", "bin_maxz", "bin_range", "tri_aabb", "tri_count",
              "sorted_pair_bin", "bin_tri_start", "bin_tri_end"):
        assert _same(ex[k], z["ref_" + k]), k
    if order == 0:
        assert _same(ex["sorted_pair_tri"], z["ref_sorted_pair_tri"])
    else:
        o = np.lexsort((ex["sorted_pair_tri"], ex["sorted_pair_bin"]))
        assert _same(ex["sorted_pair_tri"][o], z["ref_sorted_pair_tri"])
    assert _same(out["shadow"], z["ref_shadow"])
    assert _same(np.float32(st["sub"]), z["ref_sub"])
    assert _same(np.float32(st["lp_begin"]), z["ref_lp_begin"])
