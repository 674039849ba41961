"""Train the learned preconditioner on the GPU and write a checkpoint.

    python owt-krylov_b200/owtk_b200/train_learned.py --draws 500 \\
        --train-vertices 200000 --epochs 20 --out owt-krylov_b200/weights/learned_anisotropic_bs3.owtkgnn

Training data: `--draws` seeded coefficient draws of the anisotropic
unit-square Poisson-disk/Delaunay mesh of `--train-vertices` points (mesh
seed 41, RCM order, bs 3; the 8M-vertex solve mesh uses seed 4, so it is
never trained on).  Each draw gives `--pairs` residual/error pairs from the
iterates of the plain ILU(0)-preconditioned GMRES (owtk_b200.learned).  Adam
runs `--epochs` passes over all pairs, its rate decaying geometrically from
`--rate` to `--final-rate`.  Forward, backward and Adam are this library's
CUDA kernels; the host only orchestrates.  `--resume` continues from a
checkpoint's weights and Adam state.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np  # noqa: E402

from owtk_b200 import checkpoint, learned, native, problems  # noqa: E402

TRAIN_MESH_SEED = 41


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--draws", type=int, default=500)
    p.add_argument("--train-vertices", type=int, default=200_000)
    p.add_argument("--epochs", type=int, default=20)
    p.add_argument("--pairs", type=int, default=6)
    p.add_argument("--rate", type=float, default=3e-3)
    p.add_argument("--final-rate", type=float, default=3e-4)
    p.add_argument("--seed", type=int, default=1, help="initial weights")
    p.add_argument("--resume", default=None)
    p.add_argument("--out", required=True)
    p.add_argument("--device", type=int, default=0)
    a = p.parse_args(argv)

    ctx = native.Context(a.device)
    t0 = time.time()
    draws = problems.anisotropic_draws(a.train_vertices, TRAIN_MESH_SEED, range(a.draws))
    first = None
    net = None
    systems = []

    def stream():
        nonlocal first, net
        for d, s in draws:
            if first is None:
                first = s
                m0 = native.Matrix(ctx, "bsr", s.owned, 0, s.bs, s.rowptr, s.cols, s.vals)
                net = native.Learned(m0, seed=a.seed)
                systems.append(m0)
                if a.resume:
                    checkpoint.load_network(a.resume, net)
            if (d + 1) % 50 == 0:
                print(f"draw {d + 1}/{a.draws} ({time.time() - t0:.0f} s)", flush=True)
            yield s

    # learned.train needs the network before the first system is consumed.
    gen = stream()
    head = next(gen)

    def chained():
        yield head
        yield from gen

    hist = learned.train(ctx, net, chained(), epochs=a.epochs, learning_rate=a.rate, pairs_per_system=a.pairs,
                         final_learning_rate=a.final_rate, log=lambda msg: print(msg, flush=True))
    elapsed = time.time() - t0
    meta = {
        "command": "python owt-krylov_b200/owtk_b200/train_learned.py " + " ".join(argv if argv is not None else sys.argv[1:]),
        "draws": a.draws, "train_vertices": int(first.owned), "mesh_seed": TRAIN_MESH_SEED, "block_size": int(first.bs),
        "order": "rcm", "epochs": a.epochs, "pairs_per_draw": a.pairs, "rate": a.rate, "final_rate": a.final_rate,
        "initial_weights_seed": a.seed, "resumed_from": a.resume, "loss_history": hist, "seconds": round(elapsed, 1),
        "loss": "0.1 ||M(r)-e||^2/||e||^2 + ||r - A M(r)||^2/||r||^2",
    }
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    checkpoint.save_network(a.out, net, meta)
    print(json.dumps({"checkpoint": a.out, "loss_first": hist[0], "loss_last": hist[-1], "seconds": elapsed}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
