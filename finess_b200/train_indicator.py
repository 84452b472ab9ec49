"""Trains the troubled-cell indicator on labels the method generates itself.

Training set: faces of FINESS runs -- the isentropic vortex (200^2, periodic),
the four-quadrant Riemann problem (512^2, transmissive) and random
four-quadrant Riemann problems (256^2) at several times -- each face's label
being whether WENO5-JS weights there depart from the linear weights by more
than 10 %.  Features and labels are computed on the device (fin_face_samples),
the network is trained on the device (fin_mlp_train, tcgen05 tensor cores),
and the logit threshold is chosen on a held-out split so that at least 99.5 %
of the troubled faces are flagged.

    python -m finess_b200.train_indicator [--out PATH] [--samples 2000000]
    python -m finess_b200.train_indicator --physics mhd [--out PATH] [--samples 2000000]

The MHD network (--physics mhd) is trained the same way on faces of ideal-MHD
runs -- the Orszag-Tang vortex at 512^2, 1024^2 and 2048^2 through t = pi
and smooth random periodic MHD states at 512^2 -- with the MHD features and labels
(fin_mhd_face_samples: the WENO5-JS weights of any of the eight
characteristic fields).
"""
import argparse
import json
import math
import os
import time

import numpy as np

from . import problems as P
from ._abi import FIN_PREC_FP64, FIN_WENO_JS
from .indicator import DEFAULT_WEIGHTS, DEFAULT_MHD_WEIGHTS, MLP
from .solver import Solver


def _snapshots(p, q0, times, rng, per_snapshot):
    """Run the FP64 solver through `times`, sampling faces at each."""
    Xs, ys = [], []
    with Solver(p) as s:
        s.set_state(q0, 0.0)
        a1, a2 = s.GlobalWaveSpd(q0)
        dt = 0.4 * min((p.xhigh - p.xlow) / p.mx, (p.yhigh - p.ylow) / p.my) / max(a1, a2)
        dtv = np.array([0.0, dt, p.max_dt])
        t = 0.0
        for tt in times:
            if tt > t:
                dtv, _ = s.FinSolveRK(tt, dtv)
                t = tt
            nf = (p.mx + 1) * p.my + p.mx * (p.my + 1)
            stride = max(1, nf // per_snapshot)
            X, y = s.face_samples(offset=int(rng.integers(stride)), stride=stride)
            Xs.append(X)
            ys.append(y)
    return Xs, ys


def generate(total=2_000_000, seed=0, verbose=True):
    rng = np.random.default_rng(seed)
    Xs, ys = [], []
    runs = []
    p = P.vortex_params(n=200, weno=FIN_WENO_JS)
    runs.append((p, P.vortex_exact(p), [0.0, 2.5, 5.0, 7.5, 10.0]))
    p = P.riemann_params(n=512, weno=FIN_WENO_JS)
    runs.append((p, P.riemann_init(p), [0.0, 0.1, 0.3, 0.5, 0.8]))
    p = P.shock_entropy_params(nx=1024, ny=128, weno=FIN_WENO_JS)
    runs.append((p, P.shock_entropy_init(p), [0.1, 0.6, 1.2, 1.8]))
    for k in range(8):
        p = P.riemann_params(n=256, weno=FIN_WENO_JS)
        runs.append((p, P.random_riemann_state(p, rng), [0.0, 0.05, 0.15, 0.25]))
    per = total // sum(len(r[2]) for r in runs) + 1
    for p, q0, times in runs:
        p.precision = FIN_PREC_FP64
        t0 = time.time()
        X, y = _snapshots(p, q0, times, rng, per)
        Xs += X
        ys += y
        if verbose:
            print(f"  {p.mx}x{p.my}: {sum(len(v) for v in y)} faces, {np.mean(np.concatenate(y)):.3f} troubled, "
                  f"{time.time() - t0:.1f} s", flush=True)
    X = np.concatenate(Xs)
    y = np.concatenate(ys)
    idx = rng.permutation(len(y))[:total]
    return X[idx], y[idx]


def _mhd_snapshots(p, q0, aux0, times, rng, per_snapshot):
    """Run the FP64 MHD solver through `times`, sampling faces at each."""
    from .mhd import MhdSolver, first_dt
    Xs, ys = [], []
    with MhdSolver(p) as s:
        s.set_state(q0, aux0, 0.0)
        dtv = np.array([0.0, first_dt(p, q0), p.max_dt])
        t = 0.0
        for tt in times:
            if tt > t:
                s.FinSolveRK(tt, dtv)
                t = tt
            nf = (p.mx + 1) * p.my + p.mx * (p.my + 1)
            stride = max(1, nf // per_snapshot)
            X, y = s.face_samples(offset=int(rng.integers(stride)), stride=stride)
            Xs.append(X)
            ys.append(y)
    return Xs, ys


def generate_mhd(total=2_000_000, seed=0, verbose=True):
    from ._abi import FIN_PREC_FP32
    rng = np.random.default_rng(seed)
    runs = []
    # (grid, times, form): 2048^2 runs in the FP32 form (the labels are
    # computed in FP64 from the state either way)
    for n, times, prec in ((512, [0.0, 0.5, 1.0, 1.5, 2.0, 2.5, 3.0], FIN_PREC_FP64),
                           (1024, [0.5, 1.0, 1.5, 2.0, 2.5, math.pi], FIN_PREC_FP64),
                           (2048, [0.5, 1.0, 1.5, 2.0, 2.5, math.pi], FIN_PREC_FP32)):
        p = P.orszag_tang_params(n=n)
        p.precision = prec
        q, aux = P.orszag_tang_init(p)
        runs.append((p, q, aux, times))
    for k in range(4):
        p = P.orszag_tang_params(n=512)
        p.precision = FIN_PREC_FP64
        q, aux = P.mhd_random_state(p, rng, amp=0.3)
        runs.append((p, q, aux, [0.0, 0.3, 0.8]))
    per = total // sum(len(r[3]) for r in runs) + 1
    Xs, ys = [], []
    for p, q0, aux0, times in runs:
        t0 = time.time()
        X, y = _mhd_snapshots(p, q0, aux0, times, rng, per)
        Xs += X
        ys += y
        if verbose:
            print(f"  MHD {p.mx}x{p.my}: {sum(len(v) for v in y)} faces, {np.mean(np.concatenate(y)):.3f} troubled, "
                  f"{time.time() - t0:.1f} s", flush=True)
    X = np.concatenate(Xs)
    y = np.concatenate(ys)
    idx = rng.permutation(len(y))[:total]
    return X[idx], y[idx]


def train(X, y, epochs=10, seed=0, recall=0.995):
    n = len(y)
    nval = n // 10
    Xv, yv, Xt, yt = X[:nval], y[:nval], X[nval:], y[nval:]
    pos = max(1, int(yt.sum()))
    pos_weight = float(min(10.0, (len(yt) - pos) / pos))
    m = MLP(seed=seed)
    losses = m.train(Xt, yt, epochs=epochs, batch=4096, lr=3e-3, pos_weight=pos_weight, seed=seed)
    z = m.forward(Xv)
    zpos = np.sort(z[yv == 1])
    thr = float(zpos[int((1.0 - recall) * len(zpos))]) if len(zpos) else 0.0
    pred = z > thr
    rep = {
        "samples": int(n), "troubled_fraction": float(y.mean()), "pos_weight": pos_weight,
        "epoch_loss": [float(v) for v in losses], "z_threshold": thr,
        "val_recall": float(np.mean(pred[yv == 1])) if yv.sum() else None,
        "val_flagged_fraction": float(pred.mean()),
        "val_accuracy": float(np.mean(pred == (yv == 1))),
    }
    return m, rep


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--physics", default="euler", choices=["euler", "mhd"])
    ap.add_argument("--out", default=None)
    ap.add_argument("--samples", type=int, default=2_000_000)
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    t0 = time.time()
    out = args.out or (DEFAULT_MHD_WEIGHTS if args.physics == "mhd" else DEFAULT_WEIGHTS)
    print("generating training faces ...", flush=True)
    X, y = (generate_mhd if args.physics == "mhd" else generate)(args.samples, args.seed)
    t1 = time.time()
    print(f"training on {len(y)} faces ({y.mean():.3f} troubled) ...", flush=True)
    m, rep = train(X, y, args.epochs, args.seed)
    rep["generate_s"] = t1 - t0
    rep["train_s"] = time.time() - t1
    rep["physics"] = args.physics
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    np.savez(out, params=m.params, z_threshold=np.float32(rep["z_threshold"]), report=json.dumps(rep))
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
