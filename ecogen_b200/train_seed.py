"""Trains the relaxation-seed MLPs shipped in ecogen_b200/models/ (on the GPU, with the library's kernels).

    python -m ecogen_b200.train_seed [--phases 2|3] [--pairs 2000000] [--epochs 20]

Three phases: pairs recorded by the plain solver on 3D cavity-collapse cases whose inclusion seeds
(1000..) are disjoint from the benchmark case's seed (12345).  Two phases: pairs recorded on 2D
shock-bubble cases with other shock positions and bubble radii than the benchmark case.  Writes
models/seed_np<N>.npz and prints the training loss per epoch and the recording statistics.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import cases, seed

HERE = os.path.dirname(os.path.abspath(__file__))
MODELS = os.path.join(HERE, "models")


def training_cases(nphases: int, n: int):
    if nphases == 3:
        return [cases.cavity_collapse_3d(n=n, iterations=10 ** 6, seed=1000 + s, ninclusions=max(8, (n // 16) ** 3),
                                         radius_cells=(3.0, 10.0)) for s in range(6)]
    out = []
    for s, (xs, r) in enumerate([(1.5e-3, 0.8e-3), (2.5e-3, 1.2e-3), (1.0e-3, 1.5e-3), (3.0e-3, 0.6e-3)]):
        out.append(cases.shock_bubble_2d(n=n, iterations=10 ** 6, shock_x=xs, bubble_radius=r, name=f"train{s}"))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--phases", type=int, default=3)
    ap.add_argument("--pairs", type=int, default=2_000_000)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--size", type=int, default=None)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warm", type=int, default=20)
    args = ap.parse_args()
    n = args.size or (64 if args.phases == 3 else 512)
    t0 = time.time()
    x, y = seed.record(training_cases(args.phases, n), steps=args.steps, max_pairs=args.pairs, warm=args.warm)
    t1 = time.time()
    model, losses = seed.train(x, y, epochs=args.epochs, batch=8192, lr=2e-3, log=print)
    t2 = time.time()
    os.makedirs(MODELS, exist_ok=True)
    path = os.path.join(MODELS, f"seed_np{args.phases}.npz")
    model.save(path)
    info = {"pairs": int(len(y)), "record_s": t1 - t0, "train_s": t2 - t1, "loss_first": losses[0],
            "loss_last": losses[-1], "epochs": args.epochs, "mesh": n, "steps_per_case": args.steps}
    with open(path.replace(".npz", ".json"), "w") as f:
        json.dump(info, f, indent=1)
    print(json.dumps(info))


if __name__ == "__main__":
    main()
