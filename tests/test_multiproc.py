"""The benchmark's multi-rank plumbing on CPU: two gloo ranks set up the process group the way
`torchrun bench.py --gpus 2` does, meet at the barrier, and agree on the max over ranks (the
timing rule); the reference arm does its work on rank 0 only."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "CUDA_VISIBLE_DEVICES": ""})
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    r, w, _ = bench.dist_setup(world)
    bench.barrier(w)
    m = bench.max_over_ranks(10.0 * (r + 1), w)

    class A:
        steps, warmup = 1, 0

    if r != 0:  # non-zero ranks leave the reference arm without work
        bench.reference_arm(A(), r, w)
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((r, w, m))


def test_two_gloo_ranks_share_barrier_and_max():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [r[0] for r in res] == [0, 1]
    assert all(r[1] == 2 and r[2] == 20.0 for r in res)
