"""The multi-GPU plumbing of bench.py on CPU: two gloo ranks.

bench.py --gpus N runs N independent replicas of the step (the single-domain
step does not shard) and reports the whole-job throughput over the slowest
rank's time.  This checks the max-over-ranks reduction, the whole-job formula
and that replicas get different seeded inputs, with the gloo backend.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank  # this rank's timed region
        worst = bench.reduce_max(ms, dist, "cpu")
        dist.barrier()
        value = bench.job_mlups(world, 100, bench.NODES, worst)
        p = type("P", (), dict(nx=8, ny=6, nz=5, dz=0.25, rho0=1600.0, voltage=1e4, lz=1.0))
        f = bench.initial_fields(p, seed=rank)
        out[rank] = (worst, value, float(f["u"][1:-1].sum()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_and_differ_in_inputs():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
    assert out[0][0] == out[1][0] == 15.0
    import sys
    sys.path.insert(0, str(ROOT))
    import bench
    expect = world * 100 * bench.NODES / 15e-3 / 1e6
    assert out[0][1] == pytest.approx(expect) and out[1][1] == pytest.approx(expect)
    assert out[0][2] != out[1][2]  # each replica its own seeded perturbation
