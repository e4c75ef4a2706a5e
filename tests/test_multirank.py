"""Multi-GPU is replicas only: every rank generates its own realizations (distinct seeds, no
data-path collective) and the benchmark reports the units of all ranks over the slowest
rank's time.  The host-side plumbing runs here as world-size-2 gloo ranks on CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(1.0 + rank, world, "cpu")  # rank 1 is the slowest
        q.put((rank, bench.replica_seed(rank), t, bench.aggregate_rate(world, 100, 4, t)))
    finally:
        dist.destroy_process_group()


def test_replicas_reduce_to_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert out[0][1] != out[1][1]                    # distinct realizations per replica
    assert out[0][2] == out[1][2] == 2.0             # max over ranks on every rank
    assert out[0][3] == out[1][3] == 2 * 100 * 4 / 2.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("RANK", "1")

    class A:
        steps, warmup, gpus = 1, 0, 2
    assert bench.run_reference(A()) is None
    assert capsys.readouterr().out == ""
