"""Host side of the multi-GPU bench (independent replicas, no data-path
collective) on two CPU ranks over gloo: each rank gets its own seeded problem
of the same shape, the reported step time is the slowest rank's, and the
whole-job value counts every rank's cells."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method="env://", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        assert bench.dist_env() == (rank, world, rank)
        c = bench.workload(2000, rank)
        local_ms = 5.0 + 3.0 * rank  # rank 1 is the slower one
        ms = bench.max_over_ranks(local_ms)
        dist.barrier()
        out[rank] = (ms, bench.replica_value(2000, world, ms * 1e-3), c["positions"].shape,
                     float(c["positions"].sum()), float(c["weights"].sum()))
    finally:
        dist.destroy_process_group()


def test_two_replicas_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        codes = [p.exitcode for p in procs]
        assert codes == [0, 0], codes
        res = dict(out)
    assert res[0][0] == res[1][0] == 8.0           # max over ranks
    assert res[0][1] == pytest.approx(2 * 2000 / 8e-3)  # every rank's cells / slowest time
    assert res[0][2] == res[1][2] == (2000, 2)     # same shape
    assert res[0][3] != res[1][3]                  # a different problem per rank


def test_single_process_passthrough():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.replica_value(10, 1, 2.0) == 5.0
    assert np.isfinite(bench.replica_value(1_000_000, 8, 6e-3))
