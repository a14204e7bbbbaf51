"""The N > 1 path of bench.py on CPU: two gloo ranks, one process each.

`bench.py --gpus N` runs N independent replicas (one box per rank, seed base +
rank), with no collective on the data path: only a barrier and the max over
ranks of the timed region.  This checks that plumbing with world_size 2 over
gloo on 127.0.0.1, with a rank that is slower than the other.
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


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    w, r, local, pg = bench.dist_setup(world)
    assert (w, r) == (world, rank) and pg is not None
    bench.barrier(pg)
    ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
    ms_max = bench.reduce_max(pg, ms, local)
    value = bench.aggregate_value(1000, 4, w, ms_max)
    out.put((rank, bench.replica_seed(7, rank), ms_max, value))
    bench.barrier(pg)
    pg.destroy_process_group()


def test_two_gloo_replicas_time_as_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(out.get(timeout=10) for _ in range(2))
    seeds = {g[1] for g in got}
    assert seeds == {7, 8}                       # independent realisations
    for _, _, ms_max, value in got:
        assert ms_max == 150.0                   # max over ranks
        assert value == pytest.approx(1000 * 4 * 2 / 0.150)
