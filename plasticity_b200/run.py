"""Run the first increments of a named workload on one GPU and print per-increment stats.

    python -m plasticity_b200.run config3 --n 150 --increments 3
    python -m plasticity_b200.run config2 --n 64 --increments 8 --precision fp64 --predictor previous

Workloads (plasticity_b200/workloads.py): config0 (cube, tension), config1 (necking bar),
config2 (jittered/lognormal cube, compression), config3 (jittered/lognormal cube, central
top-face indentation), config4 (cube, affine top-face path).  Each increment is one
`pfem_newton` call timed with CUDA events on the library stream; model construction (host
topology + uploads) is timed separately.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload", choices=["config0", "config1", "config2", "config3", "config4"])
    ap.add_argument("--n", type=int, default=None, help="elements per edge (cube workloads)")
    ap.add_argument("--increments", type=int, default=3)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--predictor", default="extrapolate", choices=["previous", "extrapolate", "learned"])
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--maxiter", type=int, default=60)
    args = ap.parse_args()

    from . import model as P
    from . import predictor as PR
    from . import workloads as W

    make = {"config0": W.config0, "config1": W.config1, "config2": W.config2, "config3": W.config3,
            "config4": W.config4_path}[args.workload]
    w = make(n=args.n) if args.n is not None and args.workload != "config1" else make()
    t0 = time.perf_counter()
    M = P.Model(w.mesh, P.J2Material(**w.material), sigy0_e=w.sigy0_e)
    w.apply(M)
    if args.predictor == "learned":
        PR.load_into(M)
    build_s = time.perf_counter() - t0
    print(json.dumps(dict(workload=w.name, elements=w.mesh.nelem, dofs=3 * w.mesh.nnodes,
                          increments_total=w.nsteps, model_build_s=round(build_s, 2))), flush=True)
    for s in range(1, min(args.increments, w.nsteps) + 1):
        M.timer_start()
        h, k = M.newton(s / w.nsteps, tol=args.tol, maxiter=args.maxiter, precision=args.precision,
                        predictor=args.predictor, line_search=True)
        ms = M.timer_stop()
        print(json.dumps(dict(increment=s, ms=round(ms, 1), newton=len(h), krylov=int(np.sum(k)),
                              residual_first=float(h[0]), residual_last=float(h[-1]))), flush=True)
    st = M.state()
    print(json.dumps(dict(max_abs_U=float(np.abs(st["U"]).max()), plastic_gp_fraction=float(st["flags"].mean()))),
          flush=True)


if __name__ == "__main__":
    main()
