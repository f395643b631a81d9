"""The N > 1 path of bench.py on CPU: two gloo ranks run the same rank bookkeeping the
NCCL ranks use on GPUs (dist_setup, Ctx.barrier / max_ms / total) and partition the
workloads as the bench does (each rank its own ensemble or request stream, no collective
on the data path; the whole job's rate is the sum of the units over the max time)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

import bench  # noqa: F401  (imported before the fork)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), MDG_DIST_BACKEND="gloo")
    import bench
    from medusa_b200 import loadgen
    from medusa_b200 import problems as P
    w, r, local, dist = bench.dist_setup()
    ctx = bench.Ctx(w, r, local, dist)
    ctx.barrier()
    ms = ctx.max_ms(10.0 + rank)                       # the slowest rank sets the time
    probs = P.ensemble_1d(64, seed=bench.ENSEMBLE_SEED + ctx.rank)
    ncell = sum(p.ncell for p in probs)
    ncell_all = ctx.total(ncell)
    reqs = loadgen.request_stream(50, seed=11 + ctx.rank)
    rate = ctx.total(1.0e9 * (rank + 1))
    out[rank] = (w, r, ms, ncell, ncell_all, [p.n[0] for p in probs[:8]], [q.ncell for q in reqs[:8]], rate)
    ctx.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_partition_and_reduce():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        # fork: the children inherit the imported modules (no CUDA context exists in this
        # CPU test), which saves a fresh torch import per rank
        mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True,
                           start_method="fork")
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r in range(world):
        w, rank, ms, ncell, ncell_all, _, _, rate = res[r]
        assert (w, rank) == (world, r)
        assert ms == 11.0                               # max over ranks
        assert ncell_all == res[0][3] + res[1][3]       # the whole job's zones
        assert rate == 3.0e9
    # each rank has its own ensemble and its own request stream
    assert res[0][5] != res[1][5]
    assert res[0][6] != res[1][6]
