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


class _FakeColumn:
    """A column whose current alternates with a period of two steps, like the
    injector's: a + b (-1)^step."""

    def __init__(self, a, b):
        self.a, self.b, self.steps = a, b, 0

    def initialize(self):
        self.steps = 0

    def diagnostics(self):
        return {"current": self.a + self.b * (-1) ** self.steps}


class _FakeBatch:
    made = []

    def __init__(self, params, precision, device=0):
        assert precision == "fp64" and all(p.nx == 1 and p.ny == 1 for p in params)
        self.cols = [_FakeColumn(p.a, p.b) for p in params]
        self.closed = False
        _FakeBatch.made.append(self)

    def __iter__(self):
        return iter(self.cols)

    def step(self, n):
        for c in self.cols:
            c.steps += n

    def close(self):
        self.closed = True


class _FakeParams:
    def __init__(self, nx, ny, a, b, dx=0.1, dy=0.1):
        self.nx, self.ny, self.a, self.b, self.dx, self.dy = nx, ny, a, b, dx, dy
        self.lx, self.ly = nx * dx, ny * dy

    def as_dict(self):
        return dict(vars(self))

    @classmethod
    def from_dict(cls, d):
        p = cls.__new__(cls)
        p.__dict__.update(d)
        return p


class _FakeEhd:
    Params = _FakeParams
    Batch = _FakeBatch


def test_hydrostatic_columns_batch_by_step_count_and_average_two_steps():
    """The columns of instances with equal step counts share a batch; I0 is
    the mean of the currents after n and n + 1 steps, scaled to the plane."""
    S = load_sweep()
    _FakeBatch.made = []
    params = [_FakeParams(8, 6, 2.0, 0.5), _FakeParams(4, 4, 3.0, 1.0),
              _FakeParams(8, 8, 5.0, 0.25)]
    batches, starts = S.hydrostatic_columns(_FakeEhd, params, [10, 20, 10])
    assert len(batches) == 2 and [len(b.cols) for b in batches] == [2, 1]
    for p, (col, i0) in zip(params, starts):
        assert col.steps in (11, 21)  # left after n + 1 steps
        assert i0 == p.a * p.nx * p.ny  # the alternation averages out
    for b in batches:
        b.close()


def test_step_sampled_takes_the_two_step_mean():
    spec = importlib.util.spec_from_file_location("ehd_binding_copy", PKG / "ehd.py")
    E = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(E)

    class Sim:
        def __init__(self):
            self.k = 0

        def step(self, n):
            self.k += n

        def diagnostics(self):
            cur = 4.0 + (1.0 if self.k % 2 else -1.0)
            return {"current": cur, "nu_e": cur / 2.0}

    s = Sim()
    d = E._sampled([s], 10, s.step)[0]
    assert s.k == 10 and d["current_mean"] == 4.0 and d["nu_e"] == 2.0
    d = E._sampled([s], 1, s.step)[0]  # one step: the single-step ratio
    assert d["current_mean"] == d["current"] and d["nu_e"] == d["current"] / 2.0
