"""Stage-by-stage comparison of the CUDA pipeline with the CPU oracle.

Used by the gpu-marked tests and by __graft_entry__.smoke() (as the checker).
"""
from __future__ import annotations

import importlib

import numpy as np

import oracle


def run_gpu(scene, masks: bool = True, tri_order: int = 0, schedule: int = 0, separate_pairs: bool = False):
    """One frame through the library's public Context API; returns
    (outputs dict, stats dict, exported intermediates dict).  tri_order 0 is the
    reference's per-bin triangle order, 1 the coverage order; schedule selects the
    occlusion kernel's warp schedule; separate_pairs keeps the triangle/bin
    pairs as key and value arrays where one word would hold them."""
    fdzb = importlib.import_module("4dzb_b200")
    ctx, t = fdzb.context_for_scene(scene, masks=masks, debug=True, tri_order=tri_order,
                                    separate_pairs=separate_pairs)
    ctx.set_occlusion_schedule(schedule)
    ms = ctx.launch()
    res = collect(ctx, t, scene, ms=ms, tri_order=tri_order)
    ctx.close()
    return res


def collect(ctx, t, scene, ms=None, tri_order: int = 0, intermediates: bool = True):
    """(outputs dict, stats dict, exported intermediates dict) of the last launch
    of a Context made by context_for_scene (t: its tensors); intermediates need
    a debug Context."""
    st = ctx.stats()
    S, T, NB = scene.S, scene.T, scene.bins * scene.bins
    P = st["num_pairs"] if st["state"] == 2 else 0
    ex = {}
    if st["state"] == 2 and intermediates:
        for name, n in (("sample_keys", S), ("sorted_sample_keys", S), ("sorted_sample_ids", S),
                        ("bin_sample_start", NB + 1), ("bin_sample_end", NB + 1), ("bin_maxz", NB),
                        ("bin_range", 4 * NB), ("tri_count", T), ("pair_bin", P), ("pair_tri", P),
                        ("sorted_pair_bin", P), ("sorted_pair_tri", P), ("bin_tri_start", NB),
                        ("bin_tri_end", NB), ("tri_aabb", 8 * T)):
            ex[name] = ctx.export(name, n)
    out = dict(shadow=t["shadow"].cpu().numpy(), ms=ms, tri_order=tri_order)
    if t.get("masks") is not None:
        out["masks"] = t["masks"].cpu().numpy().view(np.uint32).reshape(S, -1)
    return out, st, ex


def _per_bin_sorted(keys, vals):
    """(bin, triangle) pairs ordered by bin, then triangle id."""
    o = np.lexsort((vals, keys))
    return keys[o], vals[o]


def _eq(name, a, b, errs, atol=None):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        errs.append(f"{name}: shape {a.shape} vs {b.shape}")
        return
    if a.dtype.kind == "f":
        bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    else:
        bad = a != b
    n = int(bad.sum())
    if n:
        i = np.flatnonzero(bad)[:5]
        errs.append(f"{name}: {n}/{a.size} differ, first at {i.tolist()}: gpu {a.ravel()[i].tolist()} "
                    f"oracle {b.ravel()[i].tolist()}")


def compare(scene, gpu=None, orc=None, check_intermediates: bool = True) -> list[str]:
    """Return a list of mismatch descriptions (empty = bit-exact parity)."""
    if gpu is None:
        gpu = run_gpu(scene)
    if orc is None:
        orc = oracle.frame(scene)
    out, st, ex = gpu
    o = orc.arrays
    s = orc.scalars
    errs: list[str] = []
    if st["state"] != s["state"]:
        errs.append(f"state: gpu {st['state']} oracle {s['state']}")
    if s["state"] >= 1:
        for k in ("f",):
            if np.float32(st[k]) != np.float32(s[k]):
                errs.append(f"{k}: gpu {st[k]!r} oracle {s[k]!r}")
        _eq("sub", np.float32(st["sub"]), np.float32(s["sub"]), errs)
    if s["state"] == 2:
        _eq("sample_aabb", np.float32(st["sample_aabb"]), np.float32(s["sample_aabb"]), errs)
        _eq("model_aabb", np.float32(st["model_aabb"]), np.float32(s["model_aabb"]), errs)
        _eq("lp_begin", np.float32(st["lp_begin"]), np.float32(s["lp_begin"]), errs)
        _eq("lp_end", np.float32(st["lp_end"]), np.float32(s["lp_end"]), errs)
        _eq("lp_factor", np.float32(st["lp_factor"]), np.float32(s["lp_factor"]), errs)
        if st["valid_samples"] != s["valid_samples"]:
            errs.append(f"valid_samples: gpu {st['valid_samples']} oracle {s['valid_samples']}")
        if st["valid_triangles"] != s["valid_tris"]:
            errs.append(f"valid_triangles: gpu {st['valid_triangles']} oracle {s['valid_tris']}")
        if st["num_pairs"] != s["num_pairs"]:
            errs.append(f"num_pairs: gpu {st['num_pairs']} oracle {s['num_pairs']}")
        if check_intermediates and ex:
            W, l2 = scene.W, s["view_log2up"]
            sv = o["sorted_vals"]
            sv_pos = (sv >> l2) * W + (sv & ((1 << l2) - 1))
            _eq("sample_keys", ex["sample_keys"], o["keys"], errs)
            _eq("sorted_sample_keys", ex["sorted_sample_keys"], o["sorted_keys"], errs)
            _eq("sorted_sample_ids", ex["sorted_sample_ids"], sv_pos, errs)
            _eq("bin_sample_start", ex["bin_sample_start"], o["bin_sample_start"], errs)
            _eq("bin_sample_end", ex["bin_sample_end"], o["bin_sample_end"], errs)
            _eq("bin_maxz", ex["bin_maxz"], o["bin_maxz"], errs)
            _eq("bin_range", ex["bin_range"], o["bin_range"], errs)
            _eq("tri_aabb", ex["tri_aabb"], o["tri_aabb"], errs)
            _eq("tri_count", ex["tri_count"], o["tri_count"], errs)
            if st["num_pairs"] == s["num_pairs"]:
                if out.get("tri_order", 0) == 0:
                    _eq("pair_bin", ex["pair_bin"], o["pair_bin"], errs)
                    _eq("pair_tri", ex["pair_tri"], o["pair_tri"], errs)
                else:
                    # coverage order emits the triangles in another order; each
                    # triangle's bins still come out row-major, as in the reference
                    k = np.argsort(ex["pair_tri"], kind="stable")
                    _eq("pair_bin (per triangle)", ex["pair_bin"][k], o["pair_bin"], errs)
                    _eq("pair_tri (per triangle)", ex["pair_tri"][k], o["pair_tri"], errs)
                _eq("sorted_pair_bin", ex["sorted_pair_bin"], o["sorted_pair_bin"], errs)
                if out.get("tri_order", 0) == 0:
                    _eq("sorted_pair_tri", ex["sorted_pair_tri"], o["sorted_pair_tri"], errs)
                else:
                    # coverage order: same bins, same triangle set per bin, other order
                    kb, vt = _per_bin_sorted(ex["sorted_pair_bin"], ex["sorted_pair_tri"])
                    _eq("sorted_pair_tri (per-bin set)", vt, o["sorted_pair_tri"], errs)
            _eq("bin_tri_start", ex["bin_tri_start"], o["bin_tri_start"], errs)
            _eq("bin_tri_end", ex["bin_tri_end"], o["bin_tri_end"], errs)
    # With a sampled oracle (occ_stride > 1) only the listed binned samples carry
    # oracle masks; every unbinned sample is always final.
    keep = np.ones(scene.S, bool)
    if orc._in.occ_stride > 1 and s["state"] == 2:
        W, l2 = scene.W, s["view_log2up"]
        sv = o["sorted_vals"][: s["valid_samples"]]
        keep[(sv >> l2) * W + (sv & ((1 << l2) - 1))] = False
        keep[o["occ_samples"]] = True
    if "masks" in out:
        words = out["masks"].shape[1]
        _eq("masks", out["masks"][keep], o["masks"].reshape(-1, words)[keep], errs)
    _eq("shadow", out["shadow"][keep], o["shadow"][keep], errs)
    return errs
