#!/usr/bin/env python
"""Headline benchmark: Newton load-steps/s on the 64^3 jittered compression
workload (262,144 Hex8 F-bar elements, 823,875 DOF), mixed precision (FP32
tangent + FP32 CG/AMG inside the FP64 Newton residual loop) with the learned
predictor when trained weights are present, else the extrapolation predictor,
against the plain FP64 GPU solver on the same increments.  The plain FP64 arm
is the reference's algorithm on the GPU: FP64 throughout and the reference's
predictor (the previous converged U), with backtracking line search, without
which Newton diverges on this heterogeneous mesh; an FP64 arm with the
extrapolation predictor is reported beside it to separate the two gains.

One bench "step" is one load increment (Newton to convergence + commit).
W warm-up increments run first (untimed), then K increments are timed with CUDA
events on the library's stream.  The working set (the tangent alone is >250 MB)
exceeds the 126 MB L2, so no flush is needed between steps.

Multi-GPU: the path runs on one GPU; `--gpus N` runs N independent replicas
(one process per GPU, no collective in the data path) and reports the
aggregate over ranks with max-over-ranks timing.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class Clocks:
    """nvidia-smi sampler (SM clock + throttle reasons) during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def ncu_traffic(kernel):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of `kernel`
    from the committed ncu summary profiles/ncu_traffic.txt, or None."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        f = line.split()
        if len(f) >= 2 and not line.startswith("#") and f[0] == kernel:
            return float(f[1])
    return None


def spmv_bytes(nnzb, nbrow, bs, vbytes):
    """Algorithmic bytes of one block-CSR SpMV: values + block column ids +
    row pointers + x read once + y written once."""
    return nnzb * bs * bs * vbytes + nnzb * 4 + (nbrow + 1) * 4 + 2 * nbrow * bs * vbytes


METRIC = "Newton load-steps/s, mixed+learned vs plain FP64 GPU at 1e-8 rel. disp. error"


def run_increments(M, w, first, last, **kw):
    its = []
    for s in range(first, last + 1):
        h, k = M.newton(s / w.nsteps, tol=w.tol, maxiter=40, **kw)
        its.append((len(h), int(sum(k))))
    return its


def solver_kw(kind, have_mlp):
    if kind == "mixed":
        return dict(precision="mixed", predictor="learned" if have_mlp else "extrapolate",
                    line_search=True)
    if kind == "mixed_amg_per_step":
        return dict(precision="mixed", predictor="learned" if have_mlp else "extrapolate",
                    line_search=True, amg_rebuild=False)
    if kind == "fp64":
        return dict(precision="fp64", predictor="previous", line_search=True, eta_first=0.0,
                    amg_rebuild=False)
    if kind == "fp64_extrapolate":
        return dict(precision="fp64", predictor="extrapolate", line_search=True)
    if kind == "truth":
        return dict(precision="fp64", predictor="extrapolate", line_search=True, lin_rtol=1e-12)
    raise ValueError(kind)


def cpu_reference(args, w, newton_per_step, sample_reps):
    """Time the CPU oracle (a C++ restatement of the reference path) on the same
    workload: full-size assembly of K and R + Dirichlet imposition, all host threads."""
    from oracle import oracle as O
    O.build()
    mat = O.J2Material(**w.material)
    om = O.OracleModel(w.mesh.nodes, w.mesh.elements, mat, fbar=True, sigy0_e=w.sigy0_e, nthreads=0)
    w.apply(om)
    ramp, fix = om.freeze_bcs()
    rng = np.random.default_rng(1)
    X = w.mesh.nodes
    U = np.stack([0.01 * (X[0] - 0.5), 0.01 * (X[1] - 0.5), -0.02 * X[2]]).T.reshape(-1)
    U += 1e-5 * rng.standard_normal(U.shape)
    lam = 0.1
    t0 = time.perf_counter()
    for _ in range(sample_reps):
        K, R, _, _ = om.assemble(U)
        R -= om.fext(lam)
        om.impose(K, R, ramp[0], ramp[1], True, lam, U)
        om.impose(K, R, fix[0], fix[1], False, lam, U)
    t_iter = (time.perf_counter() - t0) / sample_reps
    cores = os.cpu_count()
    value = 1.0 / (newton_per_step * t_iter)
    sample = (f"{sample_reps} full-size Newton-iteration assemblies (K and R of {w.mesh.nelem} elements + "
              f"Dirichlet imposition) at {t_iter:.3f} s each, scaled by {newton_per_step:.2f} Newton "
              f"iterations per load step; the reference's UMFPACK LU solve at {3 * w.mesh.nnodes} DOF "
              f"does not fit the sample budget and is not timed, so this is an upper bound")
    return {"value": value, "unit": "load-steps/s", "cores": cores, "kind": "port", "sample": sample}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--cpu-reps", type=int, default=3)
    ap.add_argument("--no-compare", action="store_true")
    ap.add_argument("--tol", type=float, default=1e-10,
                    help="Newton relative residual tolerance of both timed arms")
    args = ap.parse_args()
    assert args.warmup >= 3, "at least 3 warm-up steps"

    from plasticity_b200.replicas import Replicas
    reps = Replicas("nccl")
    rank, world, local = reps.rank, reps.world, reps.local

    from plasticity_b200 import workloads as W
    w = W.config2(n=args.n)
    w.tol = args.tol
    nsteps_needed = args.warmup + args.steps
    assert nsteps_needed <= w.nsteps
    config = {"workload": f"{w.name}: unit cube {args.n}^3 Hex8 F-bar, interior nodes jittered +-10% h, "
                          f"lognormal sigma_y (CoV 0.1), top uz -20% in {w.nsteps} increments, bottom uz=0 + 3-2-1",
              "elements": w.mesh.nelem, "dofs": 3 * w.mesh.nnodes, "newton_tol": w.tol,
              "timed_increments": f"{args.warmup + 1}..{nsteps_needed} of {w.nsteps}",
              "l2": "working set > 126 MB L2 (tangent alone > 250 MB); no flush",
              "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"}

    if args.impl == "reference":
        if rank != 0:
            return
        ref = cpu_reference(args, w, newton_per_step=6.0, sample_reps=args.cpu_reps)
        line = {"metric": METRIC, "value": ref["value"], "unit": "load-steps/s",
                "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": config, "cpu_baseline": ref,
                "e2e": {"value": ref["value"], "unit": "load-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import plasticity_b200 as P
    from plasticity_b200 import predictor as PR
    have_mlp = PR.weights_available()
    mat = P.J2Material(**w.material)

    def fresh_model():
        M = P.Model(w.mesh, mat, sigy0_e=w.sigy0_e, device=local)
        w.apply(M)
        if have_mlp:
            PR.load_into(M)
        return M

    barrier = reps.barrier
    max_over_ranks = reps.max_over_ranks

    from plasticity_b200 import _lib as L

    # ---- headline: mixed precision (+ learned predictor) ----
    M = fresh_model()
    run_increments(M, w, 1, args.warmup, **solver_kw("mixed", have_mlp))
    clk = Clocks(local)
    barrier()
    clk.start()
    launches0 = L.lib().pfem_kernel_launches()
    M.timer_start()
    its = run_increments(M, w, args.warmup + 1, nsteps_needed, **solver_kw("mixed", have_mlp))
    ms = M.timer_stop()
    gpu_launches = int(L.lib().pfem_kernel_launches() - launches0)
    clocks = clk.stop()
    barrier()
    ms = max_over_ranks(ms)
    U_mixed = M.U
    value = world * args.steps / (ms / 1e3)

    # roofline of the dominant kernel family (level-0 block-CSR SpMV, FP32)
    pk, pk_kind = peaks()
    spmv_ms = M.profile(2, reps=20)
    asm_ms = M.profile(1, reps=3)
    nnzb = M.pattern()[1].size // 9
    by = spmv_bytes(nnzb, M.nn, 3, 4)
    achieved = by / (spmv_ms * 1e-3) / 1e9
    roof = {"kernel": "bsr_spmv_kernel<float,3> (level-0 tangent SpMV, FP32 values)", "bound": "hbm",
            "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
            "peak_source": f"{pk_kind} (MEASURED_PEAKS.json hbm_gbs)" if pk_kind == "measured" else pk_kind,
            "algorithmic_bytes_per_launch": by, "avg_launch_ms": spmv_ms,
            "traffic": ncu_traffic("bsr_spmv_kernel<float,3,0>"),
            "element_assembly_ms": asm_ms}
    del M

    out_extra = {}
    plain_value = None
    if not args.no_compare:
        def timed_arm(kind, mlp=False):
            Mx = fresh_model()
            run_increments(Mx, w, 1, args.warmup, **solver_kw(kind, mlp))
            barrier()
            Mx.timer_start()
            itx = run_increments(Mx, w, args.warmup + 1, nsteps_needed, **solver_kw(kind, mlp))
            msx = max_over_ranks(Mx.timer_stop())
            barrier()
            return Mx.U, itx, msx

        # ---- plain FP64 GPU solver (the reference's algorithm) on the same increments ----
        U_fp64, its2, ms2 = timed_arm("fp64")
        plain_value = world * args.steps / (ms2 / 1e3)
        # ---- FP64 with the extrapolation predictor (context: the predictor's share) ----
        U_fx, its3, ms3 = timed_arm("fp64_extrapolate")
        # ---- the headline arm with the reference's AMG policy (hierarchy rebuilt every load step) ----
        _, its4, ms4 = timed_arm("mixed_amg_per_step", have_mlp)
        # ---- FP64 truth (tight inner solves, Newton to 1e-11) for the displacement error ----
        M3 = fresh_model()
        for s in range(1, nsteps_needed + 1):
            M3.newton(s / w.nsteps, tol=1e-11, maxiter=30, **solver_kw("truth", False))
        U_true = M3.U
        del M3
        nrm = np.linalg.norm(U_true)
        out_extra = {
            "plain_fp64": {"what": "FP64 tangent and CG/AMG, previous-U predictor (the reference's), line search",
                           "value": plain_value, "ms_per_step": ms2 / args.steps,
                           "newton_iters": [a for a, _ in its2], "krylov_iters": [b for _, b in its2]},
            "fp64_extrapolate": {"value": world * args.steps / (ms3 / 1e3), "ms_per_step": ms3 / args.steps,
                                 "newton_iters": [a for a, _ in its3], "krylov_iters": [b for _, b in its3]},
            "mixed_learned_amg_per_load_step": {
                "what": "the headline arm with the AMG hierarchy rebuilt at the first Newton iteration of every "
                        "load step (the reference's policy) instead of the adaptive reuse",
                "value": world * args.steps / (ms4 / 1e3), "ms_per_step": ms4 / args.steps,
                "newton_iters": [a for a, _ in its4], "krylov_iters": [b for _, b in its4]},
            "speedup_vs_plain_fp64": value / plain_value,
            "speedup_vs_fp64_extrapolate": value / (world * args.steps / (ms3 / 1e3)),
            "rel_disp_err_vs_fp64_truth": {"mixed": float(np.linalg.norm(U_mixed - U_true) / nrm),
                                           "plain_fp64": float(np.linalg.norm(U_fp64 - U_true) / nrm),
                                           "fp64_extrapolate": float(np.linalg.norm(U_fx - U_true) / nrm)}}

    # ---- the whole load path through pfem_solve (solve!): nsteps / wall time, model built ----
    full = {}
    if not args.no_compare:
        for name, kind in (("mixed_learned", "mixed"), ("plain_fp64", "fp64")):
            Mf = fresh_model()
            barrier()
            r = Mf.solve(nsteps=w.nsteps, tol=w.tol, maxiter=60, max_cuts=4, **solver_kw(kind, have_mlp))
            st = r.stats
            full[name] = {"converged": bool(r.converged), "load_steps_per_s": w.nsteps / (st["time_total_ms"] / 1e3),
                          "wall_s": st["time_total_ms"] / 1e3, "newton_total": int(st["newton_iters_total"]),
                          "krylov_total": int(st["krylov_iters_total"]),
                          "amg_setup_s": st["time_amg_setup_ms"] / 1e3, "load_step_cuts": int(st["load_step_cuts"])}
            del Mf
        full["speedup"] = full["mixed_learned"]["load_steps_per_s"] / full["plain_fp64"]["load_steps_per_s"]
        full["what"] = (f"all {w.nsteps} increments through pfem_solve (solve!): load steps / its wall time, "
                        "model construction excluded, AMG set-up included and reported")
        out_extra["full_path"] = full

    # ---- e2e: the same increments through the public C-ABI calls from host buffers ----
    t_build = time.perf_counter()
    Me = P.Model(w.mesh, mat, sigy0_e=w.sigy0_e, device=local)
    w.apply(Me)
    if have_mlp:
        PR.load_into(Me)
    build_s = time.perf_counter() - t_build
    t_warm = time.perf_counter()
    for s in range(1, args.warmup + 1):
        Me.newton(s / w.nsteps, tol=w.tol, maxiter=40, **solver_kw("mixed", have_mlp))
    warm_s = time.perf_counter() - t_warm
    barrier()
    t0 = time.perf_counter()
    h2d = d2h = 0
    for s in range(args.warmup + 1, nsteps_needed + 1):
        w.apply(Me)                                   # this step's boundary-condition arrays, host -> device
        h, k = Me.newton(s / w.nsteps, tol=w.tol, maxiter=40, **solver_kw("mixed", have_mlp))
        Ue = P.nodal_displacements(Me)                # the step's result, device -> host
        h2d += (w.dir_dofs.nbytes + w.dir_vals.nbytes + w.dir_ramp.nbytes + w.neu_dofs.nbytes
                + w.neu_vals.nbytes)
        d2h += Ue.nbytes + 8 * 40 + 4 * 40
    sig = P.gauss_stress(Me)
    alp = P.equivalent_plastic_strain(Me)
    e2e_s = time.perf_counter() - t0
    d2h += sig.nbytes + alp.nbytes
    del Me
    e2e = {"value": world * args.steps / max_over_ranks(e2e_s), "unit": "load-steps/s",
           "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
           "what": "the timed increments through the C-ABI from host (pageable) arrays: per increment the "
                   "boundary-condition arrays are uploaded (pfem_set_bcs), pfem_newton runs, and U plus the "
                   "residual/Krylov histories come back; Cauchy stress and alpha come back at the end",
           "model_build_s": build_s, "warmup_increments_s": warm_s}

    cpu = None
    if rank == 0 and world == 1:
        nps = float(np.mean([a for a, _ in its]))
        cpu = cpu_reference(args, w, newton_per_step=nps, sample_reps=args.cpu_reps)

    if rank == 0:
        line = {"metric": METRIC,
                "value": value, "unit": "load-steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64 residual / f32 tangent",
                "data": "synthetic", "config": config,
                "predictor": "learned" if have_mlp else "extrapolate",
                "newton_iters": [a for a, _ in its], "krylov_iters": [b for _, b in its],
                "clocks": clocks, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": gpu_launches, **out_extra}
        print(json.dumps(line), flush=True)
    reps.close()


if __name__ == "__main__":
    main()
