"""Trains the relaxation-seed MLPs shipped in ecogen_b200/models/ (on the GPU, with the library's kernels).

    python -m ecogen_b200.train_seed [--family cavity3d|bubble2d|tube1d|ptmu] [--pairs 2000000] [--epochs 20]

cavity3d (three phases, models/seed_np3.npz): pairs recorded by the plain solver on 3D
cavity-collapse cases whose inclusion seeds (1000..) are disjoint from the benchmark case's seed
(12345).  bubble2d (two phases, models/seed_np2.npz): 2D shock-bubble cases with other shock
positions and bubble radii than the benchmark case.  tube1d (two phases,
models/seed_np2_tube1d.npz): first-order 1D water/air shock tubes with other left pressures and
interface positions than the benchmark tube (1e9 Pa at 0.7).  Prints the training loss per epoch
and the recording statistics.  ptmu (models/seed_ptmu.npz, 8 -> 64 -> 64 -> 2): (p*, T_sat) of the
saturation solves of the p-T-mu relaxation, recorded on 2D expansion tubes with other strip velocities
and vapour fractions than the benchmark case.
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


FAMILIES = {"cavity3d": (3, "seed_np3.npz", 64), "bubble2d": (2, "seed_np2.npz", 512),
            "tube1d": (2, "seed_np2_tube1d.npz", 1000), "ptmu": (2, "seed_ptmu.npz", 256)}


def training_cases(family: str, n: int):
    if family == "tube1d":
        specs = [(3e8, 0.6), (6e8, 0.75), (2e9, 0.65), (1e8, 0.5), (8e8, 0.8), (5e9, 0.7)]
        return [cases.shock_tube_1d(ncells=n, iterations=10 ** 6, p_left=pl, x_interface=xi, name=f"tube{s}")
                for s, (pl, xi) in enumerate(specs)]
    if family == "ptmu":  # expansion tubes with other strip velocities and vapour fractions than the
        # benchmark's (500 m/s, alpha_vap 1e-2)
        specs = [(300.0, 5e-3), (700.0, 2e-2), (400.0, 1.5e-2), (600.0, 7e-3)]
        return [cases.expansion_tube_2d(n=n, iterations=10 ** 6, velocity=v, alpha_vap=a, name=f"expansion{s}")
                for s, (v, a) in enumerate(specs)]
    if family == "cavity3d":
        return [cases.cavity_collapse_3d(n=n, iterations=10 ** 6, seed=1000 + s, ninclusions=max(8, (n // 16) ** 3),
                                         radius_cells=(3.0, 10.0)) for s in range(6)]
    out = []
    for s, (xs, r) in enumerate([(1.5e-3, 0.8e-3), (2.5e-3, 1.2e-3), (1.0e-3, 1.5e-3), (3.0e-3, 0.6e-3)]):
        out.append(cases.shock_bubble_2d(n=n, iterations=10 ** 6, shock_x=xs, bubble_radius=r, name=f"train{s}"))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--family", default="cavity3d", choices=sorted(FAMILIES))
    ap.add_argument("--pairs", type=int, default=2_000_000)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--size", type=int, default=None)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warm", type=int, default=20)
    args = ap.parse_args()
    nphases, fname, default_n = FAMILIES[args.family]
    n = args.size or default_n
    t0 = time.time()
    steps, warm = args.steps, args.warm
    if args.family == "tube1d":  # small cases: record along the whole run
        steps, warm = max(steps, 400), 0
    # the p-T-mu seed learns from every saturation solve, the pressure seed from the hard relaxations
    min_evals = 1 if args.family == "ptmu" else 2
    x, y = seed.record(training_cases(args.family, n), steps=steps, max_pairs=args.pairs, warm=warm,
                       min_evals=min_evals)
    t1 = time.time()
    model, losses = seed.train(x, y, epochs=args.epochs, batch=8192, lr=2e-3, log=print)
    t2 = time.time()
    os.makedirs(MODELS, exist_ok=True)
    path = os.path.join(MODELS, fname)
    model.save(path)
    info = {"pairs": int(len(y)), "record_s": t1 - t0, "train_s": t2 - t1, "loss_first": losses[0],
            "loss_last": losses[-1], "epochs": args.epochs, "mesh": n, "steps_per_case": steps,
            "family": args.family}
    with open(path.replace(".npz", ".json"), "w") as f:
        json.dump(info, f, indent=1)
    print(json.dumps(info))


if __name__ == "__main__":
    main()
