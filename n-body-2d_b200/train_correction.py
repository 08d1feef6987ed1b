"""Trains the learned far-field correction on the GPU.

Residual samples (exact minus monopole, see include/nbody_b200.h
nb_mlp_samples) come from snapshots of the 16,384-body exponential disc and of
the two colliding discs at seeds 1-8, 2^24 samples in all by default; the
network is trained by the library's own BF16 tensor-core kernels
(nb_mlp_train).  The weights land in weights/correction_theta<theta>.npy with a
JSON record of the run beside them.

    python n-body-2d_b200/train_correction.py [--theta 1.0] [--bmax 0.75]
        [--band-theta 0.5] [--quad] [--samples 16777216] [--collision-n 4194304]
        [--epochs 6] [--out DIR] [--name NAME]

--bmax is the b_max acceptance ratio of the walk the network corrects
(nb_params.bmax_ratio), --band-theta the opening angle of the plain walk it
stands in for (nb_params.band_theta), and --quad trains it on top of the
quadrupole walk (targets: exact minus monopole minus quadrupole); inference
must use the same values, which the JSON record carries.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import pathlib
import sys
import time

import numpy as np

PKG = pathlib.Path(__file__).resolve().parent


def _package():
    if "nbody_b200" in sys.modules:
        return sys.modules["nbody_b200"]
    spec = importlib.util.spec_from_file_location(
        "nbody_b200", PKG / "__init__.py", submodule_search_locations=[str(PKG)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["nbody_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def collect(nb, theta, bmax, total, collision_n, eps2=1e-4, seeds=range(1, 9), band_theta=0.5,
            quad=False):
    """About total/16 samples from each of the 16 snapshots."""
    per = total // (2 * len(seeds))
    Xs, Ys, info = [], [], []
    for seed in seeds:
        for kind, n in (("disc", 16384), ("collision", collision_n)):
            m, p, v = nb.universes.make(kind, n, seed)
            cfg = nb.SimConfig(theta=theta, epsilon_squared=eps2, mode=nb.NB_MODE_SPLIT,
                               learned=True, bmax_ratio=bmax, band_theta=band_theta,
                               quadrupole=quad)
            with nb.NbContext(cfg, m, p, v) as ctx:
                # a few hundred band cells per target group
                X, Y = ctx.mlp_samples(max(64, per // 150), seed=seed, capacity=per)
            Xs.append(X)
            Ys.append(Y)
            info.append({"kind": kind, "n": n, "seed": seed, "samples": int(X.shape[0])})
    return np.concatenate(Xs), np.concatenate(Ys), info


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--theta", type=float, default=1.0)
    ap.add_argument("--bmax", type=float, default=0.75)
    ap.add_argument("--band-theta", type=float, default=0.5)
    ap.add_argument("--quad", action="store_true")
    ap.add_argument("--name", default=None, help="weights file stem (default correction_theta<theta>)")
    ap.add_argument("--samples", type=int, default=1 << 24)
    ap.add_argument("--collision-n", type=int, default=4194304)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--batch", type=int, default=2048)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=str(PKG / "weights"))
    args = ap.parse_args(argv)
    nb = _package()
    t0 = time.time()
    X, Y, info = collect(nb, args.theta, args.bmax, args.samples, args.collision_n,
                         band_theta=args.band_theta, quad=args.quad)
    t_samples = time.time() - t0
    t0 = time.time()
    params, losses = nb.mlp_train(X, Y, epochs=args.epochs, batch=args.batch, lr=args.lr, seed=0)
    t_train = time.time() - t0
    pred = nb.mlp_forward(params, X[:1 << 20]) * params[-1]
    fit = float(np.sqrt(((pred - Y[:1 << 20]) ** 2).mean() / (Y[:1 << 20] ** 2).mean()))
    out = pathlib.Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    stem = args.name or f"correction_theta{args.theta:g}"
    np.save(out / f"{stem}.npy", params.astype(np.float32))
    rec = {"theta": args.theta, "bmax_ratio": args.bmax, "band_theta": args.band_theta,
           "quadrupole": bool(args.quad), "samples": int(X.shape[0]),
           "snapshots": info,
           "epochs": args.epochs, "batch": args.batch, "lr": args.lr,
           "loss_per_epoch": [float(x) for x in losses], "relative_rms_fit": fit,
           "seconds_sampling": round(t_samples, 2), "seconds_training": round(t_train, 2)}
    (out / f"{stem}.json").write_text(json.dumps(rec, indent=1))
    print(json.dumps({k: v for k, v in rec.items() if k != "snapshots"}))


if __name__ == "__main__":
    main()
