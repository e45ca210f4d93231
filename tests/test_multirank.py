"""The N > 1 path of bench.py (replicas, one process per GPU) on the CPU: two
`gloo` ranks reduce their timings to the maximum over ranks and compute the
whole-job rate the way the benchmark does; a rank that raises leaves the other
with an error instead of a hang (short process-group timeout)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q, fail_rank):
    import datetime
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        if rank == fail_rank:
            raise RuntimeError("injected failure on the host")
        ms = [10.0, 12.5][rank] * 3          # 3 steps, rank 1 slower
        worst = bench.max_over_ranks(ms, dist, "cpu")
        q.put((rank, worst, bench.whole_job_rate(3, world, worst)))
    except RuntimeError as e:
        q.put((rank, "error", str(e)[:80]))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(fail_rank=-1):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q, fail_rank)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in ps:
        p.join(timeout=60)
    return sorted(out, key=lambda x: x[0])


def test_max_over_ranks_and_whole_job_rate():
    out = _run()
    assert out[0][1] == out[1][1] == 37.5           # max of 30 and 37.5 ms
    assert abs(out[0][2] - 2 * 3 * 1e3 / 37.5) < 1e-9


def test_failed_rank_does_not_hang_the_other():
    out = _run(fail_rank=1)
    assert out[1][1] == "error"
    assert out[0][1] == "error" or isinstance(out[0][1], float)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(5.0, None) == 5.0
    assert bench.whole_job_rate(20, 1, 1000.0) == 20.0
