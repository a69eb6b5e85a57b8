"""Learned per-node Newton predictor: data generation, training, evaluation.

Training data are converged load increments the solver itself produces on
32^3 cubes whose top face follows seed-drawn affine motions (combined
tension/shear/bending, 6 components uniform in +-5% of the size, 20
increments); the network (12 -> 128 -> 128 -> 3, GELU) learns the correction
to linear extrapolation of the nodal increment, and is trained on the GPU by the
library's own forward/backward/Adam kernels (BF16 tensor cores, FP32
accumulation).  Evaluation runs held-out paths at 64^3 with the extrapolation
predictor and with the learned one (which falls back to extrapolation whenever
its guess has the larger FP64 residual).

    python -m plasticity_b200.predictor train --paths 64 --steps 3000 --out plasticity_b200/weights/predictor_mlp.npz
    python -m plasticity_b200.predictor evaluate --n 64 --paths 8
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "weights", "predictor_mlp.npz")


def weights_available(path: str = WEIGHTS) -> bool:
    return os.path.exists(path)


def load_params(path: str = WEIGHTS) -> np.ndarray:
    return np.load(path)["params"].astype(np.float32)


def load_into(model, path: str = WEIGHTS) -> None:
    model.mlp_params(load_params(path))


def _path_model(n, device=0):
    from . import model as Mo
    from . import workloads as W
    w = W.config4_path(n=n, seed=0)
    M = Mo.Model(w.mesh, Mo.J2Material(**w.material), device=device)
    return M


def run_path(M, w, predictor, precision="mixed", tol=1e-8):
    """Run one load path on an existing model with the path's BCs; returns stats."""
    w.apply(M)
    M.reset()
    its, kry, res0 = [], [], []
    t0 = time.perf_counter()
    for s in range(1, w.nsteps + 1):
        h, k = M.newton(s / w.nsteps, tol=tol, maxiter=40, precision=precision, predictor=predictor,
                        line_search=True)
        its.append(len(h)); kry.append(int(sum(k))); res0.append(float(h[0]))
    return dict(newton=its, krylov=kry, first_residual=res0, seconds=time.perf_counter() - t0,
                learned_used=None)


def generate(M, n, paths, seed0=1000, nsteps=20):
    """Record training pairs from `paths` solver-generated load paths."""
    from . import workloads as W
    cap = paths * (nsteps - 2) * M.nn
    M.mlp_init(0)
    M.mlp_record("start", cap)
    M.mlp_record("clear")
    for i in range(paths):
        w = W.config4_path(n=n, nsteps=nsteps, seed=seed0 + i)
        run_path(M, w, "extrapolate")
    size = M.mlp_record("size")
    M.mlp_record("stop")
    return size


def train(M, steps, batch=65536, lr=1e-3, seed=0):
    return M.mlp_train(steps, batch=batch, lr=lr, seed=seed)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "evaluate"])
    ap.add_argument("--n", type=int, default=32)
    ap.add_argument("--paths", type=int, default=64)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--seed0", type=int, default=5000)
    args = ap.parse_args()
    from . import workloads as W
    if args.cmd == "train":
        M = _path_model(args.n)
        t0 = time.perf_counter()
        size = generate(M, args.n, args.paths)
        t1 = time.perf_counter()
        losses = train(M, args.steps, args.batch, args.lr)
        t2 = time.perf_counter()
        os.makedirs(os.path.dirname(args.out), exist_ok=True)
        meta = dict(n=args.n, paths=args.paths, samples=int(size), steps=args.steps, batch=args.batch,
                    lr=args.lr, loss_first=float(losses[:10].mean()), loss_last=float(losses[-10:].mean()),
                    gen_seconds=t1 - t0, train_seconds=t2 - t1)
        np.savez(args.out, params=M.mlp_params(), meta=json.dumps(meta), losses=losses)
        print(json.dumps(meta))
    else:
        M = _path_model(args.n)
        have = weights_available(args.out)
        out = {}
        for pred in (["extrapolate", "learned"] if have else ["extrapolate"]):
            if pred == "learned":
                load_into(M, args.out)
            rows = []
            for i in range(args.paths):
                w = W.config4_path(n=args.n, seed=args.seed0 + i)
                rows.append(run_path(M, w, pred))
            out[pred] = dict(newton=int(sum(sum(r["newton"]) for r in rows)),
                             krylov=int(sum(sum(r["krylov"]) for r in rows)),
                             seconds=float(sum(r["seconds"] for r in rows)),
                             mean_first_residual=float(np.mean([np.mean(r["first_residual"][2:]) for r in rows])))
        print(json.dumps(out))


if __name__ == "__main__":
    main()
