"""T-sweep sharding (ehd-convection-3d_b200/sweep.py) on CPU: the split of the
instances over ranks, and sweep.main's gather over two gloo ranks with a
stand-in runner in place of the GPU batch (the batch itself is covered by
tests/test_gpu_batch.py, a real share by tests/test_gpu_sweep.py)."""
import importlib.util
import os
import socket

import torch.multiprocessing as mp

from conftest import ROOT

PKG = ROOT / "ehd-convection-3d_b200"


def load_sweep():
    spec = importlib.util.spec_from_file_location("ehd_sweep", PKG / "sweep.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_instances_follow_the_sweep_definition():
    S = load_sweep()
    insts = S.make_instances(64, seed=0)
    assert len(insts) == 64 and [s["index"] for s in insts] == list(range(64))
    for s in insts:
        assert 100.0 <= s["T"] <= 400.0
        assert s["nz"] in (24, 32, 40, 48) and s["nx"] == s["ny"] == 2 * s["nz"]
    assert S.make_instances(64, seed=0) == insts  # seeded
    assert len({s["nz"] for s in insts}) > 1  # uneven sizes


def test_assignment_covers_every_instance_once_and_balances_nodes():
    S = load_sweep()
    insts = S.make_instances(64, seed=3)
    total = sum(S.nodes_of(s) for s in insts)
    for world in (1, 2, 3, 8):
        shares = S.assign(insts, world)
        assert len(shares) == world
        got = sorted(s["index"] for share in shares for s in share)
        assert got == list(range(64))
        loads = [sum(S.nodes_of(s) for s in share) for share in shares]
        assert max(loads) - min(loads) <= max(S.nodes_of(s) for s in insts)
        assert sum(loads) == total
        assert S.assign(insts, world) == shares  # every rank computes the same split


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _fake_runner(share, **kw):
    # a stand-in for the GPU batch: deterministic per-instance numbers
    return [{**s, "nu_e": 1.0 + s["T"] / 1000.0, "steps": 1000 * (1 + s["index"] % 3),
             "saturated": s["index"] % 2 == 0, "share_wall_s": 1.0} for s in share]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    S = load_sweep()
    res = S.main(["--instances", "10", "--seed", "5"], runner=_fake_runner)
    out[rank] = [(r["index"], r["nu_e"], r["steps"]) for r in res]


def test_two_gloo_ranks_gather_every_instance():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    S = load_sweep()
    expect = [(r["index"], r["nu_e"], r["steps"])
              for r in _fake_runner(S.make_instances(10, seed=5))]
    assert out[0] == expect and out[1] == expect
