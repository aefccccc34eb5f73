"""The multi-GPU plumbing of bench.py on CPU: two gloo ranks (one process each, as torchrun
starts them), the per-rank sector split and the max/sum reductions the timing uses.  The solves
themselves are replicas with no collective, so nothing else crosses ranks."""
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
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    r, w, _ = bench.dist_setup(None, backend="gloo")
    order = bench.sector_order(r, w, 27, 6)
    total = bench.all_sum(float(len(order)), w)
    slowest = bench.all_max(1.5 + r, w)
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((r, order, total, slowest))


def test_two_gloo_ranks_split_sectors_and_reduce():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, o0, t0, m0), (r1, o1, t1, m1) = res
    assert (r0, r1) == (0, 1)
    assert not set(o0) & set(o1)                        # disjoint sectors
    assert sorted(o0 + o1) == list(range(12))           # together the first 12, once each
    assert t0 == t1 == 12.0                             # whole-job solves: the sum over ranks
    assert m0 == m1 == 2.5                              # job time: the max over ranks
