"""bench.py's output contract, on the CPU.

The reference arm (`--impl reference`) times the reference's own sources on
the host cores and needs no GPU: its JSON line must carry the contract's keys
with consistent values (the GPU-only `reference_gpu` entry reports itself
unavailable here).  The roofline's DRAM traffic comes from the committed ncu
summary of the occlusion kernel.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _last_json(out: str) -> dict:
    lines = [l for l in out.splitlines() if l.startswith("{")]
    assert lines, out[-2000:]
    return json.loads(lines[-1])


def test_reference_arm_line_on_cpu():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--config", "small", "--steps", "2",
                        "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    d = _last_json(r.stdout)
    assert d["impl"] == "reference"
    assert d["metric"] == "shadow frames/s" and d["unit"] == "frames/s"
    assert d["n_gpus"] == 1 and d["steps"] == 2 and d["warmup"] >= 3
    assert d["value"] > 0 and abs(d["ms_per_step"] - 1e3 / d["value"]) < 1e-6 * d["ms_per_step"]
    assert d["higher_is_better"] is True and d["scaling"] in ("weak", "strong")
    assert d["vs_baseline"] is None
    assert d["dtype"] == "f32" and d["data"] == "synthetic"
    assert d["config"]["workload"] == "small" and d["config"]["W"] == 256 and d["config"]["triangles"] == 1024
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["unit"] == "frames/s" and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert "unavailable" in d["reference_gpu"]
    # each step is a bounded sample scaled to a full frame, and the line says so
    assert d["extrapolated"] is True and "extrapolated" in d["steps_are"]
    assert 0 < d["measured_ms_per_step"]


def test_roofline_traffic_comes_from_the_committed_profile():
    sys.path.insert(0, ROOT)
    import bench
    t = bench.profile_traffic("k_occlusion", "hd")
    assert t is not None and 5e7 < t < 5e8     # DRAM bytes of one HD launch (samples in, results out)
    assert bench.profile_traffic("k_occlusion", "no_such_workload") is None
    assert isinstance(bench.measured_peaks(), dict)
