"""The multi-GPU bench path on CPU: two ranks over gloo (127.0.0.1).

bench.py gives every rank its own database replica (workload seed = rank,
weak scaling, no collective on the data path) and reports the whole-job
value from the maximum time over ranks.  These tests run that logic with
world_size 2 on the gloo backend without a GPU.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime

    import torch.distributed as dist
    import bench
    from comer2_b200 import synth as S
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    w, r, _ = bench._dist()
    assert (w, r) == (world, rank)
    # each rank times a different amount; every rank must see the maximum
    t = bench._max_over_ranks(10.0 + rank, world, "gloo")
    wl = S.config(1, seed=rank, scale=0.0005)
    out.put((rank, t, int(wl.db.lengths.sum()), int(wl.db.lengths[0])))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gloo_max_and_replicas():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(world))
    # max over ranks
    assert [t for _, t, _, _ in res] == [11.0, 11.0]
    # rank-seeded replicas are different databases of the same configuration
    assert res[0][2:] != res[1][2:]
