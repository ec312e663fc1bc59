"""Train the learned grid-level model on the GPU and write libgrpp_b200/level_model.bin.

    python -m libgrpp_b200.train_level_model [--samples 1000000] [--epochs 6] [--out PATH]

Training pairs (features, stop level) come from the engine's plain adaptive walk
(libgrpp_b200_level_samples) on random tasks with basis l <= 6: a seeded sample of
the task lists of the config-4 molecules (2..24 atoms, heavy atoms with the full
GRPP, projectors l <= 5) plus the config-1 system (64 atoms, s..g, projectors
l <= 4). The network is trained by the engine's CUDA kernels
(libgrpp_b200_mlp_train: forward, backward and Adam); 5% of the pairs are held out
and the held-out accuracy is stored with the model.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main():
    from . import engine, level_model, synthetic

    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--samples", type=int, default=1_000_000, help="target number of walked tasks")
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--batch", type=int, default=2048)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=level_model.MODEL_FILE)
    args = ap.parse_args()

    lib = engine.load()
    t0 = time.time()
    mols = synthetic.config4()
    per_mol = max(1, int(args.samples * 0.9 / len(mols) / 0.8))  # ~80% of tasks walk the grid
    X4, y4 = level_model.samples(lib, mols, per_system=per_mol, seed=args.seed)
    X1, y1 = level_model.samples(lib, [synthetic.config1()], per_system=int(args.samples * 0.1 / 0.8),
                                 seed=args.seed + 1)
    X = np.concatenate([X4, X1])
    y = np.concatenate([y4, y1])
    t_gen = time.time() - t0
    rng = np.random.default_rng(args.seed)
    perm = rng.permutation(len(y))
    n_hold = len(y) // 20
    hold, tr = perm[:n_hold], perm[n_hold:]
    t0 = time.time()
    params, losses = level_model.train(lib, X[tr], y[tr], epochs=args.epochs, batch=args.batch, lr=args.lr,
                                       seed=args.seed)
    t_train = time.time() - t0
    pred = lib.mlp_predict(params, X[hold])
    yh = y[hold].astype(int)
    majority = int(np.bincount(y[tr], minlength=9).argmax())
    meta = {
        "samples": int(len(y)), "train": int(len(tr)), "held_out": int(n_hold), "epochs": args.epochs,
        "batch": args.batch, "lr": args.lr, "seed": args.seed, "epoch_loss": [float(v) for v in losses],
        "held_out_accuracy": float(np.mean(pred == yh)),
        "held_out_within_one": float(np.mean(np.abs(pred.astype(int) - yh) <= 1)),
        "held_out_mean_abs_error": float(np.mean(np.abs(pred.astype(int) - yh))),
        "majority_level": majority,
        "majority_accuracy": float(np.mean(yh == majority)),
        "majority_mean_abs_error": float(np.mean(np.abs(yh - majority))),
        "level_histogram": np.bincount(y, minlength=9).tolist(),
        "seconds_sampling": round(t_gen, 1), "seconds_training": round(t_train, 1),
    }
    level_model.save(params, args.out, meta)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
