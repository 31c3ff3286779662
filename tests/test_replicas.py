"""bench.py's N > 1 path on the CPU: one process per rank over gloo
(world size 2).  The GPU run uses the same functions over NCCL; the path has
no data-path collective (replicas), only the timing and unit reductions."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import datetime
    import sys

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ws, r, local = bench.dist_env()
        ms = [10.0, 12.5][rank]  # the slower rank sets the job time
        units = [1e9, 3e9][rank]
        v = bench.whole_job_value(units, ms, ws, "cpu")
        mx = bench.reduce_scalar(ms, "max", ws, "cpu")
        sm = bench.reduce_scalar(units, "sum", ws, "cpu")
        q.put((rank, ws, r, local, v, mx, sm))
    finally:
        dist.destroy_process_group()


def test_two_rank_reductions_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ws, r, local, v, mx, sm in res:
        assert (ws, r, local) == (2, rank, rank)
        assert mx == 12.5 and sm == 4e9
        assert v == pytest.approx(4e9 / 0.0125)


def test_reference_arm_other_ranks_do_no_work(capsys, monkeypatch):
    import sys

    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        scale, edge_factor, steps, warmup, gpus = 24, 16, 1, 0, 2

    bench.run_reference(A())  # rank 1 returns at once (no graph, no output)
    assert capsys.readouterr().out == ""
