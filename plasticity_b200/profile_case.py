"""Small, self-contained runs of the hot kernels, for profilers.

Builds the jittered compression cube at n^3 (the 64^3 bench workload by
default), sets a displacement that drives most Gauss points plastic (uniform
1% compression plus seeded noise), then launches:

  1. the mixed-precision assembly (element kernel per color, FP32 tangent) `reps` times,
  2. the FP64 assembly `reps` times,
  3. the level-0 FP32 block-CSR SpMV on that tangent `reps` times,
  4. the predictor network's forward pass over one row per node `reps` times
     (weights from plasticity_b200/weights when present, else random),
  5. two AMG set-ups and `reps` AMG-preconditioned CG solves (relative
     tolerance 1e-4, the device-side CG graph) on the imposed mixed-precision
     tangent at that displacement,
  6. `reps` single applications of the preconditioner (one V-cycle on level 0,
     W below where a level lies between level 0 and the dense coarse solve)
     outside the graph, so a launch list shows its kernels one by one,
  7. the imposed residual (assembly + Dirichlet imposition kernels) `reps` times,
  8. `reps` BiCGStab solves (host-driven loop: the Krylov vector and dot kernels
     run as separate launches, visible to a profiler),
  9. the predictor network's loss and gradient (the backward pass) `reps` times,
  10. four load increments (rows are recorded from the third on), then `reps`
     training steps (backward pass + Adam update) on the recorded rows.

Each family is timed with CUDA events on the library's stream and printed as one
JSON line, so the same command serves a launch list, a single-kernel capture
(`-k regex:element_color_kernel`, `bsr_spmv_kernel`, `mlp_tile_kernel`) and a
quick timing.

    python -m plasticity_b200.profile_case --n 64 --reps 3
    python -m plasticity_b200.profile_case --n 64 --reps 2 --what mlp,backward,train
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


FAMILIES = ("assembly", "spmv", "mlp", "amg", "residual", "bicgstab", "backward", "train")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--strain", type=float, default=0.01)
    ap.add_argument("--what", default="all",
                    help="comma-separated subset of " + ",".join(FAMILIES) + " (a profiler capture of one "
                         "kernel then runs few other launches before it)")
    args = ap.parse_args()
    what = set(FAMILIES) if args.what == "all" else set(args.what.split(","))
    bad = what - set(FAMILIES)
    if bad:
        raise SystemExit(f"unknown families {sorted(bad)}")

    from . import model as P
    from . import predictor as PR
    from . import workloads as W

    w = W.config2(n=args.n)
    M = P.Model(w.mesh, P.J2Material(**w.material), sigy0_e=w.sigy0_e)
    w.apply(M)
    X = w.mesh.nodes
    rng = np.random.default_rng(3)
    U = np.stack([0.3 * args.strain * X[0], 0.3 * args.strain * X[1], -args.strain * X[2]]).T.reshape(-1)
    U += 1e-2 * args.strain / args.n * rng.standard_normal(U.shape)
    M.set_displacement(U)

    out = {"n": args.n, "elements": w.mesh.nelem, "dofs": 3 * w.mesh.nnodes, "reps": args.reps}
    if "assembly" in what:
        out["assembly_mixed_ms"] = M.profile(1, reps=args.reps)
        out["assembly_fp64_ms"] = M.profile(0, reps=args.reps)
    if "spmv" in what:
        out["spmv_fp32_ms"] = M.profile(2, reps=args.reps)
    F = rng.standard_normal((M.nn, 12)).astype(np.float32)
    if what & {"mlp", "backward", "train"}:
        if PR.weights_available():
            PR.load_into(M)
        else:
            M.mlp_init(0)
    if "mlp" in what:
        M.mlp_forward(F)
        t0 = time.perf_counter()
        for _ in range(args.reps):
            M.mlp_forward(F)
        out["mlp_forward_host_ms"] = (time.perf_counter() - t0) * 1e3 / args.reps
    if what & {"amg", "bicgstab"}:
        _, R = M.residual(0.05, precision="mixed")
        M.linear_solve(-R, rtol=1e-4, rebuild=True, precision="mixed")  # symbolic hierarchy, once
    if "amg" in what:
        t0 = time.perf_counter()
        x, its = M.linear_solve(-R, rtol=1e-4, rebuild=True, precision="mixed")
        out["amg_setup_and_solve_ms"] = (time.perf_counter() - t0) * 1e3
        out["cg_iters"] = its
        t0 = time.perf_counter()
        for _ in range(args.reps):
            M.linear_solve(-R, rtol=1e-4, rebuild=False, precision="mixed")
        out["cg_solve_ms"] = (time.perf_counter() - t0) * 1e3 / args.reps
        M.amg_apply(-R)
        t0 = time.perf_counter()
        for _ in range(args.reps):
            M.amg_apply(-R)
        out["amg_cycle_host_ms"] = (time.perf_counter() - t0) * 1e3 / args.reps
        out["amg_cycle_graph_ms"] = M.profile(4, reps=20)
    if "residual" in what:
        t0 = time.perf_counter()
        for _ in range(args.reps):
            M.residual(0.05, precision="mixed")
        out["residual_host_ms"] = (time.perf_counter() - t0) * 1e3 / args.reps
    if "bicgstab" in what:
        _, R = M.residual(0.05, precision="mixed")
        t0 = time.perf_counter()
        for _ in range(args.reps):
            _, its_b = M.linear_solve(-R, rtol=1e-4, rebuild=False, precision="mixed", linsolve="bicgstab")
        out["bicgstab_solve_ms"] = (time.perf_counter() - t0) * 1e3 / args.reps
        out["bicgstab_iters"] = its_b
    if "backward" in what:
        T = 0.1 * rng.standard_normal((M.nn, 3)).astype(np.float32)
        t0 = time.perf_counter()
        for _ in range(args.reps):
            M.mlp_loss_grad(F, T)
        out["mlp_backward_host_ms"] = (time.perf_counter() - t0) * 1e3 / args.reps
    if "train" in what:
        # training rows: four converged increments from U = 0 (rows are recorded from the third on)
        M.reset()
        M.mlp_record("start", 4 * M.nn)
        for s in (1, 2, 3, 4):
            M.newton(s / w.nsteps, tol=1e-8, maxiter=40, precision="mixed", predictor="extrapolate",
                     line_search=True)
        out["recorded_rows"] = M.mlp_record("size")
        M.mlp_record("stop")
        t0 = time.perf_counter()
        M.mlp_train(args.reps, batch=65536, lr=1e-3)
        out["mlp_train_step_host_ms"] = (time.perf_counter() - t0) * 1e3 / args.reps
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
