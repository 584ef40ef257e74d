"""Learned warm start: the Fourier neural operator (include/ehd_fno.h) trained
on trajectories the EHD step itself generates, predicting the state after
`horizon` steps from (T, M, C) and the initial fields, so that a run can start
past the linear-growth transient.  No reference counterpart.

Pipeline, all on one GPU:
  1. trajectories: instances with T, M, C drawn uniformly, each from its
     hydrostatic column's state plus seeded noise, run `horizon` steps as batches
     (one graph launch per step for a whole batch);
  2. training: Adam on the mean-square error of the standardised u, v at the
     horizon and the standardised change of w, q and phi over it (their
     prediction is the initial state plus the predicted change);
  3. evaluation on held-out instances: the prediction against the plain
     run's state at the horizon, beside the same error of the initial state
     (what the plain method has without the network), and the Nu_e of a
     short run from the warm start against the plain run's.

Input channels per node: u, v, w, q / q0, phi / V, then T / 400, M / 20,
C / 20 and z / Lz as constant or coordinate channels.  Output channels: u, v
at the horizon and the change of w, q / q0, phi / V over it, standardised per
channel with the training set's mean and spread.

    python ehd-convection-3d_b200/warmstart.py --train 448 --test 64 --horizon 40000
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

IN_FIELDS = ("u", "v", "w", "q", "phi")
CIN, COUT = 9, 5
# Output channels predicted as the change over the horizon rather than as the
# state itself: w (the vertical velocity of the growing mode, close to its
# start over the horizon), q / q0 and phi / V (near-steady profiles), each
# carried over and corrected.  u and v are predicted as the state at the
# horizon: their seeded noise relaxes, so the start says little, pointwise,
# about them.
RESIDUAL = np.array([0.0, 0.0, 1.0, 1.0, 1.0], np.float32)


def sample_groups(n, seed, t_range=(150.0, 400.0), m_range=(5.0, 20.0), c_range=(5.0, 20.0)):
    rng = np.random.default_rng(seed)
    return [dict(T=float(rng.uniform(*t_range)), M=float(rng.uniform(*m_range)),
                 C=float(rng.uniform(*c_range)), seed=int(seed * 100003 + i)) for i in range(n)]


def params_of(ehd, g, nx=64, ny=64, nz=33, lambda_f=1.0 / 12.0, lambda_g=1.0e-6, Fe=4000.0):
    dz = 1.0 / (nz - 1)
    return ehd.params_from_groups(nx, ny, nz, nx * dz, ny * dz, T=g["T"], M=g["M"], C=g["C"],
                                  Fe=Fe, lambda_f=lambda_f, lambda_g=lambda_g)


def channels(f, p, g):
    """FNO input a[z][y][x][9] from fields f (reference layout [z][y][x])."""
    nz, ny, nx = f["q"].shape
    out = np.empty((nz, ny, nx, CIN), np.float32)
    out[..., 0] = f["u"]
    out[..., 1] = f["v"]
    out[..., 2] = f["w"]
    out[..., 3] = f["q"] / p.charge0
    out[..., 4] = f["phi"] / p.voltage
    out[..., 5] = g["T"] / 400.0
    out[..., 6] = g["M"] / 20.0
    out[..., 7] = g["C"] / 20.0
    out[..., 8] = (np.arange(nz) * p.dz / p.lz)[:, None, None]
    return out


def targets(f, p):
    return channels(f, p, dict(T=0.0, M=0.0, C=0.0))[..., :COUT]


def trajectories(ehd, groups, horizon, chunk=64, transits=4.0, precision="fp32", device=0,
                 extra=0, grid=(64, 64, 33)):
    """(inputs, targets, per-instance info) for the groups; instances whose
    fields go non-finite are dropped.  With extra > 0 the runs go on `extra`
    steps past the horizon and info records Nu_e there too."""
    import sweep
    ins, outs, info = [], [], []
    for c0 in range(0, len(groups), chunk):
        gs = groups[c0:c0 + chunk]
        ps = [params_of(ehd, g, *grid) for g in gs]
        cbs, starts = sweep.hydrostatic_columns(ehd, ps, [sweep.hydrostatic_steps(p, transits)
                                                          for p in ps], device=device)
        with ehd.Batch(ps, precision, device=device) as b:
            firsts = []
            for sim, g, (col, i0) in zip(b, gs, starts):
                sim.set_state_from_column(col, seed=g["seed"], amp=1e-3)
                sim.set_reference_current(i0)
                firsts.append(sim.get_fields())
            for cb in cbs:
                cb.close()
            keep = []
            for sim, g, p, f0, (col, i0), d in zip(b, gs, ps, firsts, starts,
                                                   b.step_sampled(horizon)):
                if d["nonfinite"]:
                    keep.append(False)
                    continue
                keep.append(True)
                f1 = sim.get_fields()
                ins.append(channels(f0, p, g))
                outs.append(targets(f1, p))
                info.append(dict(g, nu_e=d["nu_e"], kinetic_energy=d["kinetic_energy"], i0=i0))
            if extra > 0:
                k = len(info) - sum(keep)
                for d, kp in zip(b.step_sampled(extra), keep):
                    if kp:
                        info[k]["nu_e_extra"] = d["nu_e"]
                        k += 1
    return np.stack(ins), np.stack(outs), info


def train(net, a, t, epochs, lr, batch, seed=0, log=None):
    """Adam on shuffled mini-batches; a, t CUDA tensors [n, z, y, x, c]."""
    import torch
    rng = np.random.default_rng(seed)
    n = a.shape[0]
    hist = []
    for ep in range(epochs):
        order = rng.permutation(n)
        tot = 0.0
        for s in range(0, n - batch + 1, batch):
            idx = torch.as_tensor(order[s:s + batch], device=a.device)
            loss = net.backward(a[idx], t[idx])
            net.adam_step(lr=lr * (0.5 ** (ep * 3 // max(1, epochs))))
            tot += loss
        hist.append(tot / max(1, n // batch))
        if log:
            log(f"epoch {ep} loss {hist[-1]:.4e}")
    return hist


def rel_l2(x, y):
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-30))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--train", type=int, default=448)
    ap.add_argument("--test", type=int, default=64)
    ap.add_argument("--horizon", type=int, default=40000)
    ap.add_argument("--relax", type=int, default=2000, help="steps after the warm start")
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--width", type=int, default=32)
    ap.add_argument("--modes", type=int, default=12)
    ap.add_argument("--layers", type=int, default=4)
    ap.add_argument("--hidden", type=int, default=128)
    ap.add_argument("--grid", type=int, nargs=3, default=(64, 64, 33), metavar=("NX", "NY", "NZ"))
    ap.add_argument("--t-range", type=float, nargs=2, default=(150.0, 400.0), metavar=("LO", "HI"),
                    help="electric Rayleigh number T of the instances, uniform in [LO, HI]")
    ap.add_argument("--residual", type=float, nargs=COUT, default=tuple(RESIDUAL),
                    metavar=IN_FIELDS,
                    help="per output channel: 1 to predict its change over the horizon, "
                         "0 to predict its value there")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    resid = np.array(a.residual, np.float32)
    grid = tuple(a.grid)
    import torch

    import ehd
    import fno

    def log(m):
        print(m, flush=True)

    t0 = time.perf_counter()
    gtr = sample_groups(a.train, seed=1, t_range=tuple(a.t_range))
    gte = sample_groups(a.test, seed=2, t_range=tuple(a.t_range))
    xtr, ytr, itr = trajectories(ehd, gtr, a.horizon, grid=grid)
    xte, yte, ite = trajectories(ehd, gte, a.horizon, extra=a.relax, grid=grid)
    t_data = time.perf_counter() - t0
    log(f"trajectories: {len(itr)} train, {len(ite)} test, {t_data:.1f} s")
    # the network learns, per channel, the state at the horizon or its change
    # over the horizon (--residual), standardised; for the residual channels the
    # prediction is the initial state plus that change, so a channel that
    # hardly moves is carried over instead of being re-predicted
    dtr = ytr - xtr[..., :COUT] * resid
    mean = dtr.reshape(-1, COUT).mean(0)
    std = dtr.reshape(-1, COUT).std(0) + 1e-12
    dev = torch.device("cuda", 0)
    Xtr = torch.tensor(xtr, device=dev)
    Ytr = torch.tensor((dtr - mean) / std, device=dev, dtype=torch.float32)
    nz, ny, nx = xtr.shape[1:4]
    net = fno.FNO(nx, ny, nz, CIN, COUT, width=a.width, layers=a.layers,
                  modes=(a.modes, a.modes, min(a.modes, nz // 2)),
                  hidden=a.hidden, max_batch=a.batch, seed=7)
    t1 = time.perf_counter()
    hist = train(net, Xtr, Ytr, a.epochs, a.lr, a.batch, log=log)
    t_train = time.perf_counter() - t1
    # held-out: prediction against the plain run's state at the horizon
    errs, base = [], []
    errs_v, base_v = [], []  # the velocity channels alone
    errs_c = [[] for _ in range(COUT)]  # per output channel
    base_c = [[] for _ in range(COUT)]
    preds = []
    for k in range(len(ite)):
        u = (xte[k][..., :COUT] * resid +
             net.forward(torch.tensor(xte[k:k + 1], device=dev)).cpu().numpy()[0] * std + mean)
        preds.append(u)
        errs.append(rel_l2(u, yte[k]))
        base.append(rel_l2(xte[k][..., :COUT], yte[k]))
        errs_v.append(rel_l2(u[..., :3], yte[k][..., :3]))
        base_v.append(rel_l2(xte[k][..., :3], yte[k][..., :3]))
        for c in range(COUT):
            errs_c[c].append(rel_l2(u[..., c], yte[k][..., c]))
            base_c[c].append(rel_l2(xte[k][..., c], yte[k][..., c]))
    # warm start: a short run from the prediction against the plain run
    # continued by the same number of steps
    nu_warm, nu_cold, nu_none = [], [], []
    import sweep
    m = min(len(ite), 16)
    ps = [params_of(ehd, ite[k], *grid) for k in range(m)]
    cbs, starts = sweep.hydrostatic_columns(ehd, ps, [sweep.hydrostatic_steps(p, 4.0) for p in ps])
    with ehd.Batch(ps, "fp32") as bw, ehd.Batch(ps, "fp32") as bn:
        for k in range(m):
            p, (col, i0) = ps[k], starts[k]
            rho = np.asarray(col.get_fields(("rho",))["rho"]).reshape(-1)
            u = preds[k]
            shape = u.shape[:3]
            f = {"u": u[..., 0].astype(np.float64), "v": u[..., 1].astype(np.float64),
                 "w": u[..., 2].astype(np.float64), "q": u[..., 3] * p.charge0,
                 "phi": u[..., 4] * p.voltage,
                 "rho": np.broadcast_to(rho[:, None, None], shape).copy(),
                 "ex": np.zeros(shape), "ey": np.zeros(shape), "ez": np.zeros(shape)}
            for key in ("u", "v", "w"):
                f[key][0] = 0.0
                f[key][-1] = 0.0
            bw[k].set_fields({key: np.ascontiguousarray(v, np.float64) for key, v in f.items()})
            bw[k].poisson()  # phi and E consistent with the predicted charge
            bw[k].set_reference_current(i0)
            bn[k].set_state_from_column(col, seed=ite[k]["seed"], amp=1e-3)
            bn[k].set_reference_current(i0)
        for cb in cbs:
            cb.close()
        dw = bw.step_sampled(a.relax)
        dn = bn.step_sampled(a.relax)
        for k in range(m):
            nu_warm.append(dw[k]["nu_e"])
            nu_none.append(dn[k]["nu_e"])
            nu_cold.append(ite[k]["nu_e_extra"])
    res = {
        "train": len(itr), "test": len(ite), "horizon": a.horizon, "epochs": a.epochs,
        "residual": [float(x) for x in resid],
        "params": net.nparam, "data_s": round(t_data, 1), "train_s": round(t_train, 1),
        "loss_first": hist[0], "loss_last": hist[-1],
        "pred_rel_l2_mean": float(np.mean(errs)), "initial_rel_l2_mean": float(np.mean(base)),
        "gain": float(np.mean(base) / max(np.mean(errs), 1e-30)),
        "pred_rel_l2_velocity": float(np.mean(errs_v)),
        "initial_rel_l2_velocity": float(np.mean(base_v)),
        "gain_velocity": float(np.mean(base_v) / max(np.mean(errs_v), 1e-30)),
        "gain_channels": {name: float(np.mean(base_c[c]) / max(np.mean(errs_c[c]), 1e-30))
                          for c, name in enumerate(("u", "v", "w", "q", "phi"))},
        "initial_rel_l2_channels": {name: float(np.mean(base_c[c]))
                                    for c, name in enumerate(("u", "v", "w", "q", "phi"))},
        "nu_e_plain_at_horizon_plus_relax": nu_cold,
        "nu_e_warm_after_relax": nu_warm,
        "nu_e_plain_after_relax_from_start": nu_none,
        "nu_e_err_warm": float(np.mean(np.abs(np.array(nu_warm) - np.array(nu_cold)))),
        "nu_e_err_plain_short": float(np.mean(np.abs(np.array(nu_none) - np.array(nu_cold)))),
    }
    log(json.dumps({k: v for k, v in res.items() if not isinstance(v, list)}))
    if a.out:
        Path(a.out).write_text(json.dumps(res, indent=1))
    net.close()
    return res


if __name__ == "__main__":
    main()
