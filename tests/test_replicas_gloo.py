"""Replica plumbing of bench.py on CPU: two gloo ranks over 127.0.0.1 take the barrier, the
max over ranks of their timings and the whole-job aggregate, as the NCCL ranks do on GPUs."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_init("gloo")
    bench.barrier(w)
    t_local = 0.5 + 0.25 * r                     # the slower rank sets the job time
    t = bench.max_over_ranks(w, t_local, "cpu")
    q.put((r, w, t, bench.aggregate_rate(w, 10, t)))
    bench.barrier(w)
    dist.destroy_process_group()


def test_two_gloo_replicas():
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
    for r, w, t, rate in out:
        assert w == 2 and t == 0.75
        assert rate == pytest.approx(2 * 10 / 0.75)


def test_single_rank_is_local():
    import bench
    assert bench.max_over_ranks(1, 0.3, "cpu") == 0.3
    assert bench.aggregate_rate(1, 20, 0.5) == 40.0
