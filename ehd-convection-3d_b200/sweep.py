"""Parameter sweeps in the electric Rayleigh number T: many instances of
uneven size run to saturated Nu_e, batched on each GPU and sharded across
GPUs.

No reference counterpart: the reference runs one instance per process with a
compile-time grid (LBM.h:34-36).  A sweep is a list of instances (T, grid,
seed).  Each rank of a torch.distributed job takes a share of them, balanced
by node count, runs its share as one ehd_batch (one CUDA graph launch per step
over all of its instances, launch shapes from the batch autotuner) from the
hydrostatic column's own state (ehd_set_state_from_column) plus seeded noise
until each instance's Nu_e saturates, and
the per-instance results are gathered on every rank.  The only exchange
between ranks is that gather (a few numbers per instance).

    python -m torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1 \\
        ehd-convection-3d_b200/sweep.py --instances 64 --precision fp16
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def make_instances(n: int = 64, seed: int = 0, nz_choices=(24, 32, 40, 48),
                   t_range=(100.0, 400.0)) -> list[dict]:
    """The sweep's instances: T uniform in t_range, nz cells drawn from
    nz_choices (NZ = nz + 1 nodes, NX = NY = 2 nz, Lz = 1, dx = 1 / nz), a
    seed per instance for its velocity noise."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nz = int(rng.choice(nz_choices))
        out.append({"index": i, "T": float(rng.uniform(*t_range)), "nz": nz, "nx": 2 * nz,
                    "ny": 2 * nz, "seed": i})
    return out


def nodes_of(inst: dict) -> int:
    return inst["nx"] * inst["ny"] * (inst["nz"] + 1)


def assign(instances: list[dict], world: int) -> list[list[dict]]:
    """Shares for `world` ranks, balanced by node count: largest instance
    first onto the least-loaded rank (ties to the lower rank), each share in
    instance order.  Deterministic, so every rank computes the same split."""
    shares = [[] for _ in range(world)]
    load = [0] * world
    for inst in sorted(instances, key=lambda s: (-nodes_of(s), s["index"])):
        r = min(range(world), key=lambda k: (load[k], k))
        shares[r].append(inst)
        load[r] += nodes_of(inst)
    return [sorted(s, key=lambda x: x["index"]) for s in shares]


def instance_params(ehd, inst: dict, M=10.0, C=10.0, Fe=4000.0, lambda_f=1.0 / 12.0,
                    lambda_g=1.0e-6):
    """ehd_params of one instance: dx = dy = dz = 1 / nz, Lz = 1."""
    nz = inst["nz"]
    dz = 1.0 / nz
    return ehd.params_from_groups(inst["nx"], inst["ny"], nz + 1, inst["nx"] * dz,
                                  inst["ny"] * dz, T=inst["T"], M=M, C=C, Fe=Fe,
                                  lambda_f=lambda_f, lambda_g=lambda_g)


def hydrostatic_steps(p, transits: float) -> int:
    """`transits` charge transit times Lz / (K V / Lz), an even number of steps."""
    n = int(round(transits * p.lz * p.lz / (p.K * p.voltage) / p.dt))
    return n + (n & 1)


def hydrostatic_profiles(ehd, params: list, nsteps: list, device=0):
    """ehd_hydrostatic_profile for many instances at once: the 1 x 1 x NZ
    columns of all instances with the same step count run as one batch (one
    graph launch per step for all of them), in FP64 from the reference's
    initial state.  A batch step is bitwise the step of a lone context, so
    the profiles and I0 equal ehd_hydrostatic_profile's."""
    out = [None] * len(params)
    by_steps = {}
    for i, n in enumerate(nsteps):
        by_steps.setdefault(int(n), []).append(i)
    for n, idx in by_steps.items():
        cols = []
        for i in idx:
            q = ehd.Params.from_dict(params[i].as_dict())
            q.nx, q.ny, q.lx, q.ly = 1, 1, params[i].dx, params[i].dy
            cols.append(q)
        with ehd.Batch(cols, "fp64", device=device) as b:
            for sim in b:
                sim.initialize()
            b.step(n)
            profs, cur = [], []
            for sim in b:
                f = sim.get_fields()
                profs.append({k: np.asarray(v).reshape(-1).copy() for k, v in f.items()})
                cur.append(sim.diagnostics()["current"])
            b.step(1)  # I0: mean of the currents after n and n + 1 steps
            for i, sim, prof, c0 in zip(idx, b, profs, cur):
                i0 = 0.5 * (c0 + sim.diagnostics()["current"]) * params[i].nx * params[i].ny
                out[i] = (prof, i0)
    return out


def hydrostatic_columns(ehd, params: list, nsteps: list, device=0):
    """ehd_hydrostatic_column for many instances at once: the 1 x 1 x NZ
    columns of all instances with the same step count run as one FP64 batch,
    left after n + 1 steps.  Returns the batches (close them when done) and,
    per instance, (column, I0) with I0 the mean of the currents after n and
    n + 1 steps, as ehd_hydrostatic_column has them."""
    out = [None] * len(params)
    batches = []
    by_steps = {}
    for i, n in enumerate(nsteps):
        by_steps.setdefault(int(n), []).append(i)
    for n, idx in by_steps.items():
        cols = []
        for i in idx:
            q = ehd.Params.from_dict(params[i].as_dict())
            q.nx, q.ny, q.lx, q.ly = 1, 1, params[i].dx, params[i].dy
            cols.append(q)
        b = ehd.Batch(cols, "fp64", device=device)
        batches.append(b)
        for sim in b:
            sim.initialize()
        b.step(n)
        cur = [sim.diagnostics()["current"] for sim in b]
        b.step(1)
        for i, sim, c0 in zip(idx, b, cur):
            i0 = 0.5 * (c0 + sim.diagnostics()["current"]) * params[i].nx * params[i].ny
            out[i] = (sim, i0)
    return batches, out


def run_share(share: list[dict], precision="fp16", device=0, amp=1.0e-3, sample_every=1000,
              tol=1e-3, hold=3, max_steps=200000, min_steps=0, autotune=True,
              hydrostatic_transits=16.0, **groups) -> list[dict]:
    """Runs one rank's share on one GPU as a batch; one result per instance.
    min_steps: steps taken before the saturation sampling starts (the
    criterion cannot tell the slow linear growth near the threshold from a
    stationary state).  `groups` overrides M, C, Fe, lambda_f, lambda_g of
    instance_params."""
    if not share:
        return []
    sys.path.insert(0, str(HERE))
    import ehd

    t0 = time.perf_counter()
    params = [instance_params(ehd, s, **groups) for s in share]
    col_batches, starts = hydrostatic_columns(
        ehd, params, [hydrostatic_steps(p, hydrostatic_transits) for p in params], device=device)
    t1 = time.perf_counter()
    batch = ehd.Batch(params, precision, device=device)
    try:
        if autotune:
            batch.autotune(trial_steps=10)
        for sim, s, (col, i0) in zip(batch, share, starts):
            sim.set_state_from_column(col, seed=s["seed"], amp=amp)
            sim.set_reference_current(i0)
        for b in col_batches:
            b.close()
        t2 = time.perf_counter()
        if min_steps > 0:
            batch.step(min_steps)
        res = batch.run_to_saturation(sample_every=sample_every, tol=tol, hold=hold,
                                      max_steps=max(0, max_steps - min_steps))
        t3 = time.perf_counter()
        out = []
        for s, r, sim in zip(share, res, batch):
            d = sim.diagnostics()
            out.append({**s, **r, "steps": r["steps"] + min_steps,
                        "kinetic_energy": d["kinetic_energy"], "nonfinite": d["nonfinite"],
                        "tuning": sim.get_tuning(), "share_wall_s": t3 - t0,
                        "hydrostatic_wall_s": t1 - t0, "run_wall_s": t3 - t2})
        return out
    finally:
        batch.close()
        for b in col_batches:
            b.close()


def gather(results: list[dict], dist=None) -> list[dict]:
    """Every rank's results on every rank, in instance order."""
    if dist is None:
        return sorted(results, key=lambda r: r["index"])
    allr = [None] * dist.get_world_size()
    dist.all_gather_object(allr, results)
    return sorted([r for part in allr for r in part], key=lambda r: r["index"])


def main(argv=None, runner=run_share):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", default="fp16", choices=["fp64", "fp32", "mixed", "fp16", "bf16"])
    ap.add_argument("--sample-every", type=int, default=1000)
    ap.add_argument("--tol", type=float, default=1e-3)
    ap.add_argument("--hold", type=int, default=3)
    ap.add_argument("--max-steps", type=int, default=200000)
    ap.add_argument("--min-steps", type=int, default=0,
                    help="steps before the saturation sampling starts")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--out", default=None, help="write the gathered results (JSON) here")
    a = ap.parse_args(argv)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600), **kw)
    try:
        insts = make_instances(a.instances, a.seed)
        share = assign(insts, world)[rank]
        res = runner(share, precision=a.precision, device=local, sample_every=a.sample_every,
                     tol=a.tol, hold=a.hold, max_steps=a.max_steps, min_steps=a.min_steps,
                     autotune=not a.no_autotune)
        allres = gather(res, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    if rank == 0:
        summary = {"instances": len(allres), "ranks": world,
                   "saturated": sum(1 for r in allres if r.get("saturated")),
                   "non_finite": sum(1 for r in allres if r.get("saturated") is None),
                   "wall_s": max((r.get("share_wall_s", 0.0) for r in allres), default=0.0)}
        print(json.dumps(summary), flush=True)
        if a.out:
            Path(a.out).write_text(json.dumps(allres, indent=1))
    return allres


if __name__ == "__main__":
    main()
