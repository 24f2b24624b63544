"""Multi-process plumbing of bench.py on the CPU: two ranks over gloo (the
N > 1 path runs N independent replicas; the only collectives are the barrier
and the max over ranks of the device timings)."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    import torch.distributed as dist

    ws, r, local = bench.dist_setup()
    try:
        assert (ws, r, local) == (world, rank, rank)
        m = bench.dist_max(1.5 + rank)  # each rank's step time; the job's is the slowest
        bench.dist_barrier()
        args = argparse.Namespace(config="small", steps=1, warmup=0, gpus=world)
        rc = bench.run_reference(args) if rank != 0 else 0  # non-zero ranks exit without work
        out.put((rank, m, rc))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_and_barrier():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [r[1] for r in res] == [2.5, 2.5]
    assert [r[2] for r in res] == [0, 0]
