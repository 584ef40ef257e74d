"""Fine-grid warm start: the Fourier neural operator's coarse-grid prediction,
carried to a finer and wider grid, as the initial state of a run with 16-bit
population storage, beside a cold start in FP32.  No reference counterpart.

Pipeline, all on one GPU:
  1. the network is trained on coarse-grid trajectories (warmstart.py), or
     loaded from a file that --save wrote;
  2. it predicts the coarse state `horizon` coarse steps after the coarse
     hydrostatic column plus seeded noise, for one (T, M, C);
  3. the prediction is tiled periodically in x and y (the fine box is `tiles`
     coarse boxes wide) and interpolated linearly onto the fine nodes (the fine
     spacing is the coarse one over `factor`; x, y periodic, z between the
     electrode nodes); rho comes from the fine hydrostatic column, and phi and
     E from a Poisson solve of the interpolated charge;
  4. from that state the fine grid runs `steps` steps with FP16 deviation
     storage, and, for the storage error, in FP32; a cold start (the fine
     hydrostatic column's state plus seeded noise) runs the same steps in FP32.
     Diagnostics (kinetic energy, Nu_e, total charge) every `sample` steps.

Fields are in the solver's physical units (velocity, charge density and
potential do not depend on the spacing), so they carry over between grids
unchanged; the fine step is the coarse one over `factor` (dt = CFL dx), so
the prediction stands for the fine state horizon * factor fine steps after
the start.

    python ehd-convection-3d_b200/finestart.py --T 300 --coarse 64 64 33 --tiles 2 --factor 4
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

PRED_FIELDS = ("u", "v", "w", "q", "phi")


def _periodic_axis(a: np.ndarray, axis: int, factor: int) -> np.ndarray:
    """Linear interpolation along a periodic axis onto `factor` times as many
    points: fine point i sits at coarse position i / factor."""
    n = a.shape[axis]
    pos = np.arange(n * factor) / factor
    i0 = np.floor(pos).astype(np.int64)
    w = pos - i0
    i0 %= n
    i1 = (i0 + 1) % n
    shape = [1] * a.ndim
    shape[axis] = -1
    w = w.reshape(shape)
    return np.take(a, i0, axis=axis) * (1.0 - w) + np.take(a, i1, axis=axis) * w


def _bounded_axis(a: np.ndarray, axis: int, factor: int) -> np.ndarray:
    """Linear interpolation between the end nodes of an axis: (n - 1) factor
    + 1 points, the coarse nodes kept exactly."""
    n = a.shape[axis]
    m = (n - 1) * factor + 1
    pos = np.arange(m) / factor
    i0 = np.minimum(np.floor(pos).astype(np.int64), n - 2)
    w = pos - i0
    shape = [1] * a.ndim
    shape[axis] = -1
    w = w.reshape(shape)
    return np.take(a, i0, axis=axis) * (1.0 - w) + np.take(a, i0 + 1, axis=axis) * w


def upsample(field: np.ndarray, tiles: int, factor: int) -> np.ndarray:
    """A coarse field [z][y][x] on the fine grid: tiled `tiles` times in x and
    y, then linearly interpolated by `factor` in x, y (periodic) and z
    (between the electrode nodes).  (nz, ny, nx) -> ((nz - 1) factor + 1,
    ny tiles factor, nx tiles factor)."""
    f = np.tile(np.asarray(field, np.float64), (1, tiles, tiles))
    f = _periodic_axis(f, 2, factor)
    f = _periodic_axis(f, 1, factor)
    return _bounded_axis(f, 0, factor)


def fine_params(ehd, coarse_p, tiles: int, factor: int):
    """ehd_params of the fine grid: the coarse box `tiles` times wider in x
    and y, spacing and time step over `factor`, the same physics."""
    q = ehd.Params.from_dict(coarse_p.as_dict())
    q.nx, q.ny = coarse_p.nx * tiles * factor, coarse_p.ny * tiles * factor
    q.nz = (coarse_p.nz - 1) * factor + 1
    q.lx, q.ly = coarse_p.lx * tiles, coarse_p.ly * tiles
    q.dx, q.dy, q.dz = coarse_p.dx / factor, coarse_p.dy / factor, coarse_p.dz / factor
    q.dt = coarse_p.dt / factor
    return q


def save_net(path, net, mean, std):
    """The network's configuration, parameters and output standardisation."""
    c = net.cfg
    cfg = {k: int(getattr(c, k)) for k in ("nx", "ny", "nz", "in_channels", "out_channels",
                                            "width", "layers", "modes_x", "modes_y", "modes_z",
                                            "hidden", "max_batch")}
    np.savez(path, params=net.params(), mean=np.asarray(mean), std=np.asarray(std),
             config=json.dumps(cfg))


def load_net(path, device=0):
    import fno
    d = np.load(path)
    c = json.loads(str(d["config"]))
    net = fno.FNO(c["nx"], c["ny"], c["nz"], c["in_channels"], c["out_channels"],
                  width=c["width"], layers=c["layers"],
                  modes=(c["modes_x"], c["modes_y"], c["modes_z"]), hidden=c["hidden"],
                  max_batch=c["max_batch"], device=device)
    net.set_params(d["params"])
    return net, d["mean"], d["std"]


def predict(ehd, net, mean, std, group: dict, coarse_grid, transits=4.0, device=0):
    """(coarse params, predicted coarse fields) for one (T, M, C, seed)."""
    import torch

    import sweep
    import warmstart as W
    p = W.params_of(ehd, group, *coarse_grid)
    cbs, [(col, i0)] = sweep.hydrostatic_columns(ehd, [p], [sweep.hydrostatic_steps(p, transits)],
                                                 device=device)
    with ehd.Simulation(p, "fp32", device=device) as sim:
        sim.set_state_from_column(col, seed=group["seed"], amp=1e-3)
        f0 = sim.get_fields()
    for cb in cbs:
        cb.close()
    x = torch.tensor(W.channels(f0, p, group)[None], device=torch.device("cuda", device))
    # the network predicts the velocity and the change of q, phi (warmstart.py)
    u = (W.channels(f0, p, group)[..., :W.COUT].astype(np.float64) * W.RESIDUAL +
         net.forward(x).cpu().numpy()[0].astype(np.float64) * std + mean)
    pred = {"u": u[..., 0], "v": u[..., 1], "w": u[..., 2], "q": u[..., 3] * p.charge0,
            "phi": u[..., 4] * p.voltage}
    return p, pred


def warm_fields(pred: dict, fine_profile: dict, tiles: int, factor: int) -> dict:
    """Fine-grid fields from a coarse prediction: u, v, w, q, phi upsampled,
    no-slip walls, rho from the fine hydrostatic column, E zero (the caller
    solves the Poisson problem of the charge before stepping)."""
    f = {k: upsample(pred[k], tiles, factor) for k in PRED_FIELDS}
    for k in ("u", "v", "w"):
        f[k][0] = 0.0
        f[k][-1] = 0.0
    shape = f["q"].shape
    f["rho"] = np.broadcast_to(np.asarray(fine_profile["rho"])[:, None, None], shape).copy()
    for k in ("ex", "ey", "ez"):
        f[k] = np.zeros(shape)
    return {k: np.ascontiguousarray(v, np.float64) for k, v in f.items()}


def run(sim, steps: int, sample: int) -> dict:
    """Steps in chunks of `sample`, diagnostics after each (they synchronise;
    Nu_e as the two-step mean of Simulation.step_sampled); wall time of the
    whole run."""
    import torch
    hist = []
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        n = min(sample, steps - done)
        d = sim.step_sampled(n)
        done += n
        hist.append({"step": done, "kinetic_energy": d["kinetic_energy"], "nu_e": d["nu_e"],
                     "total_charge": d["total_charge"], "umax": d["umax"],
                     "nonfinite": d["nonfinite"]})
    sim.synchronize()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    return {"history": hist, "wall_s": wall}


def field_errors(a: dict, b: dict) -> dict:
    """Max-norm error of a against b over each field, relative to b's max."""
    out = {}
    for k in ("u", "v", "w", "q", "phi"):
        scale = float(np.abs(b[k]).max())
        out[k] = float(np.abs(a[k] - b[k]).max() / scale) if scale > 0 else 0.0
    return out


def compare(ehd, coarse_p, pred: dict, group: dict, tiles: int, factor: int, steps: int,
            sample: int, warm_precision="fp16", transits=4.0, device=0, log=None) -> dict:
    """The fine-grid runs of step 4 of the pipeline for one prediction."""
    import sweep
    fp = fine_params(ehd, coarse_p, tiles, factor)
    cbs, [(fcol, i0)] = sweep.hydrostatic_columns(ehd, [fp],
                                                  [sweep.hydrostatic_steps(fp, transits)],
                                                  device=device)
    fprof = {"rho": np.asarray(fcol.get_fields(("rho",))["rho"]).reshape(-1)}
    start = warm_fields(pred, fprof, tiles, factor)
    nodes = fp.nx * fp.ny * fp.nz
    res = {"fine_grid": [fp.nx, fp.ny, fp.nz], "fine_lx": fp.lx, "steps": steps,
           "sample": sample, "fine_dt": fp.dt, "reference_current": i0}
    ends = {}
    runs = [("warm_" + warm_precision, warm_precision, True)]
    if warm_precision != "fp32":
        runs.append(("warm_fp32", "fp32", True))
    runs.append(("cold_fp32", "fp32", False))
    for name, prec, warm in runs:
        with ehd.Simulation(fp, prec, device=device) as sim:
            if warm:
                sim.set_fields(start)
                sim.poisson()  # phi and E of the interpolated charge
            else:
                sim.set_state_from_column(fcol, seed=group["seed"], amp=1e-3)
            sim.set_reference_current(i0)
            d0 = sim.diagnostics()
            r = run(sim, steps, sample)
            r["initial"] = {"kinetic_energy": d0["kinetic_energy"], "nu_e": d0["nu_e"],
                            "total_charge": d0["total_charge"]}
            r["mlups"] = nodes * steps / max(r["wall_s"], 1e-12) / 1e6
            if warm:
                ends[prec] = sim.get_fields()
        res[name] = r
        if log:
            last = r["history"][-1]
            log(f"{name}: KE {r['initial']['kinetic_energy']:.3e} -> {last['kinetic_energy']:.3e}, "
                f"Nu_e {last['nu_e']:.5f}, {r['mlups']:.0f} MLUPS")
    for cb in cbs:
        cb.close()
    if warm_precision in ends and "fp32" in ends and warm_precision != "fp32":
        res["warm_storage_error"] = field_errors(ends[warm_precision], ends["fp32"])
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--T", type=float, default=300.0)
    ap.add_argument("--M", type=float, default=10.0)
    ap.add_argument("--C", type=float, default=10.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--coarse", type=int, nargs=3, default=(64, 64, 33),
                    metavar=("NX", "NY", "NZ"))
    ap.add_argument("--tiles", type=int, default=2)
    ap.add_argument("--factor", type=int, default=4)
    ap.add_argument("--steps", type=int, default=20000, help="fine steps of each run")
    ap.add_argument("--sample", type=int, default=2000)
    ap.add_argument("--precision", default="fp16", choices=["fp16", "bf16", "fp32"])
    ap.add_argument("--load", default=None, help="network file written by --save")
    ap.add_argument("--save", default=None, help="write the trained network here (.npz)")
    ap.add_argument("--train", type=int, default=128)
    ap.add_argument("--horizon", type=int, default=40000)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--width", type=int, default=32)
    ap.add_argument("--modes", type=int, default=12)
    ap.add_argument("--layers", type=int, default=4)
    ap.add_argument("--hidden", type=int, default=128)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    import torch

    import ehd
    import fno
    import warmstart as W

    def log(m):
        print(m, flush=True)

    coarse = tuple(a.coarse)
    res = {"T": a.T, "M": a.M, "C": a.C, "coarse_grid": list(coarse), "tiles": a.tiles,
           "factor": a.factor, "horizon": a.horizon, "precision": a.precision}
    t0 = time.perf_counter()
    if a.load:
        net, mean, std = load_net(a.load)
        res["network"] = a.load
        if (net.cfg.nx, net.cfg.ny, net.cfg.nz) != coarse:
            raise SystemExit(f"{a.load}: network grid {(net.cfg.nx, net.cfg.ny, net.cfg.nz)} "
                             f"is not the coarse grid {coarse}")
    else:
        groups = W.sample_groups(a.train, seed=1)
        xtr, ytr, itr = W.trajectories(ehd, groups, a.horizon, grid=coarse)
        dtr = ytr - xtr[..., :W.COUT] * W.RESIDUAL  # targets as warmstart.py
        mean = dtr.reshape(-1, W.COUT).mean(0)
        std = dtr.reshape(-1, W.COUT).std(0) + 1e-12
        dev = torch.device("cuda", 0)
        nz, ny, nx = xtr.shape[1:4]
        net = fno.FNO(nx, ny, nz, W.CIN, W.COUT, width=a.width, layers=a.layers,
                      modes=(a.modes, a.modes, min(a.modes, nz // 2)), hidden=a.hidden,
                      max_batch=a.batch, seed=7)
        hist = W.train(net, torch.tensor(xtr, device=dev),
                       torch.tensor((dtr - mean) / std, device=dev, dtype=torch.float32),
                       a.epochs, a.lr, a.batch, log=log)
        res.update(train=len(itr), loss_first=hist[0], loss_last=hist[-1])
        if a.save:
            save_net(a.save, net, mean, std)
    res["network_s"] = round(time.perf_counter() - t0, 1)
    group = {"T": a.T, "M": a.M, "C": a.C, "seed": a.seed}
    cp, pred = predict(ehd, net, mean, std, group, coarse)
    res.update(compare(ehd, cp, pred, group, a.tiles, a.factor, a.steps, a.sample,
                       warm_precision=a.precision, log=log))
    net.close()
    log(json.dumps({k: v for k, v in res.items()
                    if k not in ("warm_fp16", "warm_bf16", "warm_fp32", "cold_fp32")}))
    if a.out:
        Path(a.out).write_text(json.dumps(res, indent=1))
    return res


if __name__ == "__main__":
    main()
