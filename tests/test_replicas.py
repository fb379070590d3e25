"""The multi-GPU path is replicas only: every rank runs the whole workload on its own GPU
and the job's time is the slowest rank's.  The host side of that (the max over ranks,
the whole-job value, rank 0 alone printing the reference arm) runs here as two gloo
ranks on the CPU."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as td
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        slowest = bench.max_over_ranks(100.0 + 25.0 * rank, True, "cpu")
        out.put((rank, slowest, bench.replica_value(1e9, 4, world, slowest)))
    finally:
        td.destroy_process_group()


def test_max_over_ranks_and_whole_job_value_with_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    # both ranks agree on the slowest time (rank 1: 125 ms) and the value counts both ranks
    assert [r[1] for r in res] == [125.0, 125.0]
    assert res[0][2] == pytest.approx(2.0 * 1e9 * 4 * 2 / 0.125 / 1e9)


def test_single_process_keeps_its_own_time():
    import bench
    assert bench.max_over_ranks(42.5, False, "cpu") == 42.5
    assert bench.replica_value(5e8, 2, 1, 1000.0) == pytest.approx(2.0)


def test_reference_arm_prints_on_rank_zero_only(monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = bench.argparse.Namespace(gpus=2, steps=1, warmup=0)
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args)  # returns before any work on ranks other than 0
    assert buf.getvalue() == ""
