"""Learned per-node Newton predictor: data generation, training, evaluation.

Training data are converged load increments the solver itself produces on
512 load paths of 32^3 cubes whose top face follows seed-drawn affine motions
(combined tension/shear/bending, 6 components uniform in +-5% of the size,
20 increments -- every fourth path 40, so the load-step-size input varies);
the network (12 -> 128 -> 128 -> 3, GELU) learns the correction
to linear extrapolation of the nodal increment, and is trained on the GPU by the
library's own forward/backward/Adam kernels (BF16 tensor cores, FP32
accumulation).  Evaluation runs held-out paths at 64^3 with the extrapolation
predictor and with the learned one (which falls back to extrapolation whenever
its guess has the larger FP64 residual).

    python -m plasticity_b200.predictor train --paths 512 --steps 12000 --out plasticity_b200/weights/predictor_mlp.npz
    python -m plasticity_b200.predictor evaluate --n 64 --paths 64
    python -m plasticity_b200.predictor guess --n 32 --paths 4 --smooth 16
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
    """Solve one load path on an existing model with the path's BCs; returns stats."""
    w.apply(M)
    t0 = time.perf_counter()
    r = M.solve(nsteps=w.nsteps, tol=tol, maxiter=60, precision=precision, predictor=predictor,
                line_search=True, max_cuts=4)
    sec = time.perf_counter() - t0
    return dict(converged=r.converged, newton=list(r.iters), krylov=[int(sum(k)) for k in r.cg_iters],
                first_residual=[float(h[0]) for h in r.residuals], seconds=sec,
                learned_used=int(r.stats["predictor_learned_used"]), cuts=int(r.stats["load_step_cuts"]),
                newton_total=int(r.stats["newton_iters_total"]), krylov_total=int(r.stats["krylov_iters_total"]),
                stats=r.stats)


def guess_errors(M, w, smooth=None, precision="mixed", tol=1e-10):
    """Quality of the two guesses along one load path.  At every load step from
    the third on (the learned guess needs two converged increments), both
    guesses are formed, Newton converges from the one the FP64 residual picks,
    and each guess's error is measured against the converged U as a fraction of
    the step's increment.  Returns per-step rows."""
    w.apply(M)
    M.reset()
    rows = []
    U_prev = np.zeros(M.ndof)
    kw = dict(precision=precision, line_search=True, tol=tol, maxiter=60)
    sm = {} if smooth is None else dict(predictor_smooth=smooth)
    from ._lib import PfemError
    for s in range(1, w.nsteps + 1):
        lam = s / w.nsteps
        try:
            if s <= 2:
                M.newton(lam, predictor="extrapolate", **kw)
                U_prev = M.U
                continue
            U_ex, _, _, _ = M.predict(lam, "extrapolate", precision=precision)
            U_ml, r_ex, r_ml, used = M.predict(lam, "learned", precision=precision, **sm)
            h, k = M.newton(lam, predictor="previous", **kw)
        except PfemError as e:  # a load step that does not converge ends the path
            rows.append(dict(step=s, failed=str(e)))
            break
        U = M.U
        inc = max(np.linalg.norm(U - U_prev), 1e-300)
        rows.append(dict(step=s, r_extrap=r_ex, r_learned=r_ml, used=used, newton=len(h), krylov=int(sum(k)),
                         err_extrap=float(np.linalg.norm(U_ex - U) / inc),
                         err_chosen=float(np.linalg.norm(U_ml - U) / inc)))
        U_prev = U
    return rows


def generate(M, n, paths, seed0=1000, nsteps=(20, 20, 20, 40)):
    """Record training pairs from `paths` solver-generated load paths; path i
    takes nsteps[i % len(nsteps)] increments, so the load-step-size input
    varies across the set."""
    from . import workloads as W
    cap = sum(nsteps[i % len(nsteps)] - 2 for i in range(paths)) * M.nn
    M.mlp_init(0)
    M.mlp_record("start", cap)
    M.mlp_record("clear")
    for i in range(paths):
        w = W.config4_path(n=n, nsteps=nsteps[i % len(nsteps)], seed=seed0 + i)
        run_path(M, w, "extrapolate")
    size = M.mlp_record("size")
    M.mlp_record("stop")
    return size


def train(M, steps, batch=65536, lr=1e-3, seed=0):
    return M.mlp_train(steps, batch=batch, lr=lr, seed=seed)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "evaluate", "guess"])
    ap.add_argument("--smooth", type=int, default=None)
    ap.add_argument("--n", type=int, default=32)
    ap.add_argument("--paths", type=int, default=512)
    ap.add_argument("--steps", type=int, default=12000)
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
    elif args.cmd == "guess":
        M = _path_model(args.n)
        load_into(M, args.out)
        allr, failed = [], 0
        for i in range(args.paths):
            rows = guess_errors(M, W.config4_path(n=args.n, seed=args.seed0 + i), args.smooth)
            failed += sum("failed" in r for r in rows)
            allr += [r for r in rows if "failed" not in r]
        med = lambda k: float(np.median([r[k] for r in allr]))
        print(json.dumps(dict(n=args.n, paths=args.paths, smooth=args.smooth, steps=len(allr), failed_paths=failed,
                              learned_kept=int(sum(r["used"] for r in allr)),
                              median_err_extrap=med("err_extrap"), median_err_chosen=med("err_chosen"),
                              median_r_extrap=med("r_extrap"), median_r_learned=med("r_learned"),
                              newton=int(sum(r["newton"] for r in allr)),
                              krylov=int(sum(r["krylov"] for r in allr)))))
    else:
        M = _path_model(args.n)
        have = weights_available(args.out)
        out = {}
        for pred in (["extrapolate", "learned"] if have else ["extrapolate"]):
            if pred == "learned":
                load_into(M, args.out)
            rows = [run_path(M, W.config4_path(n=args.n, seed=args.seed0 + i), pred) for i in range(args.paths)]
            out[pred] = dict(converged=all(r["converged"] for r in rows),
                             paths_converged=int(sum(r["converged"] for r in rows)),
                             load_step_cuts=int(sum(r["cuts"] for r in rows)),
                             newton=int(sum(r["newton_total"] for r in rows)),
                             krylov=int(sum(r["krylov_total"] for r in rows)),
                             seconds=float(sum(r["seconds"] for r in rows)),
                             learned_used=int(sum(r["learned_used"] for r in rows)),
                             steps=int(sum(len(r["newton"]) for r in rows)))
        print(json.dumps(out))

if __name__ == "__main__":
    main()
