#!/usr/bin/env python3
"""Generate the golden fixtures of the FDZB soft-shadow path from the reference
itself: 4DZB's own kernel and host sources compiled for the CPU
(oracle/ref_emu/build_ref.py -> oracle/_ref/libref4dzb.so, which needs the
reference sources; run this where they are present).

Each fixture stores the frame's inputs (view samples, triangle soup, light,
knobs) and the reference's outputs after FD::FDLaunch: light projection,
sub-constant and light plane, sorted (bin, sample) pairs, per-bin segments and
statistics, per-triangle AABBs and bin counts, sorted (bin, triangle) pairs,
per-bin triangle segments and the shadow buffer.  The reference's bin grid is
its compile-time 16 x 16 (FS/constants.h:13).

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))

# name: (W, H, T, N, seed, cull, esp, background fraction, back-facing fraction)
FIXTURES = {
    "g0_n8": (128, 128, 512, 8, 101, False, 1e-3, 0.0, 0.0),
    "g1_n8_cull": (128, 128, 512, 8, 102, True, 1e-3, 0.0, 0.0),
    "g2_n16_w160": (160, 96, 600, 16, 103, False, 1e-3, 0.0, 0.0),
    "g3_n32": (128, 64, 400, 32, 104, False, 1e-3, 0.0, 0.0),
    "g4_n4_mixed": (128, 128, 512, 4, 105, True, 1e-6, 0.25, 0.2),
}

ARRAYS = ["shadow", "sorted_keys", "sorted_vals", "bin_sample_start", "bin_sample_end", "bin_maxz", "bin_range",
          "tri_aabb", "tri_count", "tri_prefix", "sorted_pair_bin", "sorted_pair_tri", "bin_tri_start",
          "bin_tri_end"]
SCALARS = ["num_bins", "valid_samples", "valid_tris", "num_pairs", "view_log2up", "mat", "RF", "corners",
           "deltas", "sub", "lp_begin", "lp_end", "lp_factor"]


def scene_for(name):
    scenes = importlib.import_module("4dzb_b200.scenes")
    W, H, T, N, seed, cull, esp, bg, back = FIXTURES[name]
    s = scenes.make_scene(W, H, T, n=N, bins=16, seed=seed, esp=esp, cull=cull, name=name)
    rng = np.random.default_rng(seed)
    if bg > 0:
        s.pos[rng.random(s.S) < bg, 0] = np.nan
    if back > 0:
        flip = rng.random(s.S) < back
        s.nrm[flip, :3] *= -1.0
    return s


def make(name: str) -> str:
    ref = importlib.import_module("oracle.ref")
    s = scene_for(name)
    r = ref.run(s)
    if r["errors"]:
        raise RuntimeError(f"{name}: reference harness reported {r['errors']} errors")
    W, H, T, N, seed, cull, esp, bg, back = FIXTURES[name]
    d = dict(W=W, H=H, T=T, N=N, seed=seed, cull=int(cull), esp=np.float32(esp), bins=16,
             pos=s.pos, nrm=s.nrm, vtx=s.vtx, idx=s.idx,
             light=np.array([s.light.right_radius, s.light.top_radius, *s.light.position, *s.light.view_dir,
                             *s.light.up_dir], np.float32))
    for k in ARRAYS:
        d["ref_" + k] = r[k]
    for k in SCALARS:
        d["ref_" + k] = np.asarray(r[k])
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **d)
    return path


if __name__ == "__main__":
    for n in FIXTURES:
        print(make(n), os.path.getsize(os.path.join(HERE, n + ".npz")))
