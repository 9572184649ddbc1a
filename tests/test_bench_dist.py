"""CPU check of bench.py's multi-process plumbing (world size 2, gloo): the
barrier and the max over ranks of the per-rank timings that the N-GPU run
uses (one replica per GPU, no data-path collective)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import bench
    import torch.distributed as dist
    ws, r, _ = bench.dist_setup("gloo")
    bench.barrier(ws)
    v = bench.max_over_ranks(1.0 + r, ws)
    q.put((r, ws, v))
    dist.destroy_process_group()


def test_two_rank_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=5) for _ in range(2))
    assert out == [(0, 2, 2.0), (1, 2, 2.0)]


def test_reference_arm_other_ranks_exit(monkeypatch, capsys):
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")

    class A:
        steps, warmup, cpu_iters, ref_iters = 1, 1, 1, 1
    bench.run_reference(A, (4, 4, 4, 4))
    assert capsys.readouterr().out == ""
