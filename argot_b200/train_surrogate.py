"""Trains the frequency-integral surrogate on the GPU and writes
argot_b200/data/surrogate.npz (parameters + validated error envelope).

    python -m argot_b200.train_surrogate [--samples 10000000] [--epochs 30]

1. seeded samples of the exact 256-bin quadrature generated on the device;
2. training with the hand-written forward / backward / Adam kernels;
3. validation on held-out samples with the tensor-core inference path:
   the error envelope (largest error of q per output and bin of predicted
   q, times 1.5) from which the rate kernels bound each ray's error.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import surrogate as S


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--samples", type=int, default=10_000_000)
    ap.add_argument("--val", type=int, default=1_000_000)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--out", default=S.WEIGHTS)
    ap.add_argument("--revalidate", action="store_true",
                    help="keep the parameters of --out and only re-measure the error envelope "
                         "with the current inference kernel")
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    t0 = time.time()
    tr = S.Trainer("cuda", seed=a.seed)
    Xv, Yv = tr.samples(a.val, a.seed + 1)
    prev = {}
    if a.revalidate:
        params, _ = S.load(a.out)
        with np.load(a.out) as f:
            prev = json.loads(str(f["meta"])) if "meta" in f.files else {}
        hist = [prev.get("final_loss")]
        t_gen, t_train = prev.get("gen_s", 0.0), prev.get("train_s", 0.0)
        a.samples, a.epochs, a.batch, a.lr = (prev.get(k, getattr(a, k)) for k in ("samples", "epochs", "batch", "lr"))
    else:
        X, Y = tr.samples(a.samples, a.seed)
        torch.cuda.synchronize()
        t_gen = time.time() - t0
        hist = tr.train(X, Y, a.epochs, a.batch, a.lr, seed=a.seed, log=print)
        torch.cuda.synchronize()
        t_train = time.time() - t0 - t_gen
        params = tr.params.cpu().numpy()
    sur = S.Surrogate(params, np.zeros((6, S.ENV_BINS), np.float32), tol=1.0)
    qv = sur.eval(Xv).cpu().numpy().astype(np.float64)
    qt = Yv.cpu().numpy().astype(np.float64)
    env = S.error_envelope(qv, qt)
    dq = np.abs(qv - qt)
    y = tr.thin_limit(Xv.cpu().numpy()) * np.exp(qt)
    rel = np.abs(y) * dq  # relative error of I_j
    meta = {"samples": a.samples, "epochs": a.epochs, "batch": a.batch, "lr": a.lr, "seed": a.seed,
            "final_loss": hist[-1], "gen_s": t_gen, "train_s": t_train,
            "val_max_err_q": dq.max(0).tolist(), "val_median_err_q": np.median(dq, 0).tolist(),
            "val_frac_rel_I_within_5e-4": np.mean(rel <= 5e-4, 0).tolist(),
            "val_frac_rel_I_within_5e-4_thin": float(np.mean(rel[np.abs(y[:, 0]) < 1, 0] <= 5e-4)),
            "envelope_revalidated": bool(a.revalidate)}
    S.save(params, env, a.out, {"meta": json.dumps(meta)})
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
