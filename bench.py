#!/usr/bin/env python
"""Headline benchmark: Newton load-steps/s on the 64^3 jittered compression
workload (262,144 Hex8 F-bar elements, 823,875 DOF), mixed precision (FP32
tangent + FP32 CG/AMG inside the FP64 Newton residual loop) with the learned
predictor when trained weights are present, else the extrapolation predictor.

Beside it, on the same increments, the arms that split the speed-up into its
parts: mixed + extrapolation, FP64 + extrapolation, and the plain FP64 GPU
solver (the reference's algorithm on the GPU: FP64 throughout and the
reference's predictor, the previous converged U, with backtracking line
search), plus an FP64 "truth" run that every arm's displacements are measured
against.  A side arm that fails is reported as failed; it never suppresses the
headline line.

One bench "step" is one load increment (Newton to convergence + commit).
W warm-up increments run first (untimed), then K increments are timed with CUDA
events on the library's stream.  The working set (the tangent alone is >250 MB)
exceeds the 126 MB L2, so no flush is needed between steps.

`--impl reference` times the CPU restatement of the reference's algorithm
(oracle: C++ assembly on all host threads, SuperLU standing in for the
reference's UMFPACK, previous-U predictor) on whole load increments of the same
workload generator at the largest mesh whose increments fit the time budget.

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
import traceback

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
METRIC = "Newton load-steps/s, mixed+learned vs plain FP64 GPU at 1e-8 rel. disp. error"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)), "measured"
    return PEAKS_FALLBACK, "fallback"


class Clocks:
    """SM clock and throttle reasons sampled every 10 ms during a timed region
    (NVML through pynvml; nvidia-smi at its 200 ms floor if pynvml is absent)."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, index, period_s=0.01):
        self.index, self.period = index, period_s
        self.sm, self.mx, self.reasons = [], None, set()
        self._stop = threading.Event()
        self._t = None
        self._nv = None

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self._nv = nv
            h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))

            def run():
                while not self._stop.is_set():
                    try:
                        self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        for k, bit in self.REASONS.items():
                            if r & bit:
                                self.reasons.add(k)
                    except Exception:
                        pass
                    time.sleep(self.period)
            self._t = threading.Thread(target=run, daemon=True)
            self._t.start()
        except Exception:
            self._nv = None
            self._smi_start()

    def _smi_start(self):
        q = ("index,clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                           "--format=csv,noheader,nounits", "-lms", "200"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self._proc = None
            return

        def run():
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for ln in self._proc.stdout:
                f = [x.strip() for x in ln.split(",")]
                try:
                    self.sm.append(float(f[1])); self.mx = float(f[2])
                except (ValueError, IndexError):
                    continue
                for nm, v in zip(names, f[3:7]):
                    if v.lower().startswith("active"):
                        self.reasons.add(nm)
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._nv is None and getattr(self, "_proc", None) is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
        if self._t is not None:
            self._t.join(timeout=5)
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.mx,
                "reasons": sorted(self.reasons), "samples": len(self.sm),
                "sampler": "nvml 10 ms" if self._nv is not None else "nvidia-smi 200 ms"}


def ncu_traffic(kernel, algorithmic_bytes):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of `kernel`
    from the committed ncu summary profiles/ncu_traffic.txt, and how it was obtained.
    The capture is of the 64^3 launch; for another size the captured traffic is scaled
    by the ratio of algorithmic bytes (the SpMV's traffic grows in proportion)."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(p):
        return None, None
    for line in open(p):
        f = line.split()
        if len(f) >= 3 and not line.startswith("#") and f[0] == kernel:
            t, alg = float(f[1]), float(f[2])
            if abs(algorithmic_bytes - alg) <= 1e-6 * alg:
                return t, "ncu capture of this launch (profiles/ncu_traffic.txt)"
            return t * algorithmic_bytes / alg, "64^3 ncu capture scaled by algorithmic bytes"
    return None, None


def spmv_bytes(nnzb, nbrow, bs, vbytes, ibytes=4):
    """Algorithmic bytes of one block-CSR SpMV: values + block column ids (ibytes
    each) + row pointers + x read once + y written once."""
    return nnzb * bs * bs * vbytes + nnzb * ibytes + (nbrow + 1) * 4 + 2 * nbrow * bs * vbytes


def solver_kw(kind, have_mlp):
    """Solver options of each arm."""
    learned = "learned" if have_mlp else "extrapolate"
    if kind == "mixed":
        return dict(precision="mixed", predictor=learned, line_search=True)
    if kind == "mixed_extrapolate":
        return dict(precision="mixed", predictor="extrapolate", line_search=True)
    if kind == "mixed_amg_per_step":
        return dict(precision="mixed", predictor=learned, line_search=True, amg_rebuild=False)
    if kind == "fp64":
        return dict(precision="fp64", predictor="previous", line_search=True, eta_first=0.0,
                    amg_rebuild=False, ew_need=False)
    if kind == "fp64_extrapolate":
        return dict(precision="fp64", predictor="extrapolate", line_search=True)
    if kind == "truth":
        return dict(precision="fp64", predictor="previous", line_search=True, lin_rtol=1e-12)
    raise ValueError(kind)


# Newton's relative test is |R| <= tol * max(|R_1|, |F_ext|, 1) (Solver.jl:349-358).  The truth
# run starts every increment from the previous converged U, so |R_1| is set by the increment's
# boundary-value jump (~1e3 on this workload) and 1e-12 of it (~1e-9 absolute) stays above
# the FP64 rounding floor of the assembled residual (~1e-11 absolute at 64^3); with exact
# inner solves Newton converges quadratically, so the last iterate lands far below it.
TRUTH_TOL = 1e-12


def run_increments(M, w, first, last, maxiter=40, **kw):
    its = []
    for s in range(first, last + 1):
        h, k = M.newton(s / w.nsteps, tol=w.tol, maxiter=maxiter, **kw)
        its.append((len(h), int(sum(k))))
    return its


WORKLOADS = ("compress", "indent")


def make_workload(kind, n):
    """The bench workloads: 'compress' is the 64^3 jittered / lognormal cube under
    20 % top-face compression in 40 increments; 'indent' is the 150^3 cube of the
    same kind with a central 30 x 30-node top-face patch indented 10 % in 30
    increments (the patch scales with the mesh below 150^3)."""
    from plasticity_b200 import workloads as W
    if kind == "compress":
        return W.config2(n=n)
    return W.config3(n=n, patch=max(2, round(30 * n / 150)))


def cpu_reference(n_cpu, increments, tol, nthreads=0, kind="compress"):
    """Whole load increments of the reference's algorithm on the CPU oracle: the
    C++ restatement of assembly + Dirichlet imposition on all host threads, the
    linear solve by SuperLU in a nested-dissection order (sequential; stands in
    for UMFPACK, Solver.jl:237-240), the previous converged U as predictor
    (Solver.jl:321-323) and the commit re-assembly (Solver.jl:470-471), on the same
    workload generator at n_cpu^3.  Returns the workload, per-increment (Newton
    iterations, seconds) and the LU seconds."""
    from oracle import oracle as O
    O.build()
    w = make_workload(kind, n_cpu)
    om = O.OracleModel(w.mesh.nodes, w.mesh.elements, O.J2Material(**w.material), fbar=True,
                       sigy0_e=w.sigy0_e, nthreads=nthreads)
    w.apply(om)
    ramp, fix = om.freeze_bcs()
    stats = {}
    lu = O.nd_lu_solver(O.box_nd_dofs(n_cpu, n_cpu, n_cpu), stats)
    out = []
    for s in increments:
        t0 = time.perf_counter()
        # the indentation's patch edge inverts elements under plain Newton from the
        # previous U; there the baseline takes the same backtracking line search as
        # the GPU arms (the reference has none and stops)
        conv, hist = om.newton(s / w.nsteps, ramp, fix, tol, 40, linsolve=lu, line_search=kind == "indent")
        if not conv:
            raise RuntimeError(f"CPU reference: increment {s} at {n_cpu}^3 did not converge")
        _, _, tau, fl = om.assemble(om.U, commit=True)
        om.tau, om.flags = tau, fl
        out.append((len(hist), time.perf_counter() - t0))
    return w, out, stats.get("lu_s", 0.0)


def lscpu_summary():
    try:
        txt = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        keep = {}
        for ln in txt.splitlines():
            k, _, v = ln.partition(":")
            if k.strip() in ("Model name", "CPU(s)", "Thread(s) per core", "Socket(s)", "CPU max MHz"):
                keep[k.strip()] = v.strip()
        return keep
    except Exception:
        return {}


def cpu_baseline(n_cpu, first, last, tol, kind="compress", bench_mesh="64^3, 823,875 DOF"):
    w, out, t_lu = cpu_reference(n_cpu, range(first, last + 1), tol, kind=kind)
    secs = sum(t for _, t in out)
    newton = [k for k, _ in out]
    return {"value": len(out) / secs, "unit": "load-steps/s", "cores": os.cpu_count(), "kind": "port",
            "sample": (f"increments {first}..{last} of {w.nsteps} of the same workload generator at {n_cpu}^3 "
                       f"({3 * w.mesh.nnodes} DOF), whole increments end to end: the reference algorithm "
                       f"(previous-U predictor, exact LU every Newton iteration, "
                       f"{'backtracking line search' if kind == 'indent' else 'no line search'}) on the C++ "
                       f"oracle (assembly + imposition on {os.cpu_count()} threads) with SuperLU (sequential, "
                       f"nested-dissection order) standing in for UMFPACK; Newton iterations {newton}, LU "
                       f"{t_lu:.1f} s of {secs:.1f} s. The bench mesh ({bench_mesh}) is out of reach of a "
                       f"direct LU in the budget (factorisation time grows ~N^2: 1.0 / 3.4 s at 16^3 / 20^3)"),
            "mesh": f"{n_cpu}^3", "newton_iters": newton, "seconds": secs, "lu_seconds": t_lu,
            "lscpu": lscpu_summary()}


def reference_arm(args, config):
    """`--impl reference`: timed whole increments of the CPU restatement of the reference."""
    n_cpu = args.cpu_n
    nsteps = make_workload(args.workload, n_cpu).nsteps
    first = args.warmup + 1
    last = min(args.warmup + args.steps, nsteps)
    t_all = time.perf_counter()
    w, out, t_lu = cpu_reference(n_cpu, range(1, last + 1), 1e-10, kind=args.workload)
    timed = out[first - 1:]
    secs = sum(t for _, t in timed)
    value = len(timed) / secs
    cfg = dict(config)
    cfg["cpu_mesh"] = f"{n_cpu}^3 ({3 * w.mesh.nnodes} DOF): the largest mesh of this workload whose whole " \
                      f"increments fit the time budget with a direct LU"
    line = {"metric": METRIC, "value": value, "unit": "load-steps/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": len(timed), "warmup": first - 1, "ms_per_step": 1e3 * secs / len(timed),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": "load-steps/s", "cores": os.cpu_count(), "kind": "port",
                             "sample": f"increments {first}..{last} of {nsteps} at {n_cpu}^3, whole increments: "
                                       f"C++ oracle assembly on all threads + SuperLU (sequential, nested-dissection "
                                       f"order) in place of UMFPACK, previous-U predictor; Newton iterations "
                                       f"{[k for k, _ in timed]}; total run {time.perf_counter() - t_all:.1f} s",
                             "lscpu": lscpu_summary()},
            "e2e": {"value": value, "unit": "load-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="compress", choices=WORKLOADS,
                    help="compress: 64^3 jittered cube, 20%% compression (the headline); indent: 150^3 "
                         "jittered cube, central top-face indentation (10.3 M DOF)")
    ap.add_argument("--n", type=int, default=None, help="elements per edge (default 64 / 150)")
    ap.add_argument("--cpu-n", type=int, default=16, help="mesh of the CPU baseline (elements per edge)")
    ap.add_argument("--cpu-increments", type=int, default=2)
    ap.add_argument("--no-compare", action="store_true")
    ap.add_argument("--tol", type=float, default=1e-10,
                    help="Newton relative residual tolerance of the timed arms")
    args = ap.parse_args()
    assert args.warmup >= 3, "at least 3 warm-up steps"

    from plasticity_b200.replicas import Replicas
    reps = Replicas("nccl")
    rank, world, local = reps.rank, reps.world, reps.local

    if args.n is None:
        args.n = 64 if args.workload == "compress" else 150
    w = make_workload(args.workload, args.n)
    w.tol = args.tol
    nsteps_needed = args.warmup + args.steps
    assert nsteps_needed <= w.nsteps, f"warmup + steps must be <= {w.nsteps} increments"
    if args.workload == "compress":
        desc = (f"{w.name}: unit cube {args.n}^3 Hex8 F-bar, interior nodes jittered +-10% h, lognormal sigma_y "
                f"(CoV 0.1), top uz -20% in {w.nsteps} increments, bottom uz=0 + 3-2-1")
    else:
        # the FP64 comparison arms take minutes per increment-window at 10.3 M DOF
        args.no_compare = True
        desc = (f"{w.name}: unit cube {args.n}^3 Hex8 F-bar, interior nodes jittered +-10% h, lognormal sigma_y "
                f"(CoV 0.1), central {w.meta['patch']}x{w.meta['patch']}-node top-face patch uz -10% in "
                f"{w.nsteps} increments, bottom clamped; comparison arms not run at this size")
    config = {"workload": desc,
              "elements": w.mesh.nelem, "dofs": 3 * w.mesh.nnodes, "newton_tol": w.tol,
              "timed_increments": f"{args.warmup + 1}..{nsteps_needed} of {w.nsteps}",
              "l2": "working set > 126 MB L2 (tangent alone > 250 MB); no flush",
              "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"}

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args, config)
        reps.close()
        return

    import plasticity_b200 as P
    from plasticity_b200 import _lib as L
    from plasticity_b200 import predictor as PR
    have_mlp = PR.weights_available()
    mat = P.J2Material(**w.material)
    barrier, max_over_ranks = reps.barrier, reps.max_over_ranks
    errors = {}

    def fresh_model():
        M = P.Model(w.mesh, mat, sigy0_e=w.sigy0_e, device=local)
        w.apply(M)
        if have_mlp:
            PR.load_into(M)
        return M

    def guarded(name, fn):
        """Run a side measurement; a failure is recorded, never raised."""
        try:
            return fn()
        except Exception as e:  # noqa: BLE001 -- every failure of a side arm is reported, not fatal
            errors[name] = f"{type(e).__name__}: {e}"
            traceback.print_exc(file=sys.stderr)
            return None

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

    # ---- roofline of the dominant kernel family (level-0 block-CSR SpMV, FP32) ----
    def roofline():
        pk, pk_kind = peaks()
        spmv_ms = M.profile(2, reps=20)
        asm_ms = M.profile(1, reps=3)
        nnzb = M.pattern()[1].size // 9
        by = spmv_bytes(nnzb, M.nn, 3, 4, M.tangent_index_bytes())
        achieved = by / (spmv_ms * 1e-3) / 1e9
        traffic, traffic_src = ncu_traffic("bsr_spmv_kernel<float,3,0>", by)
        return {"kernel": "bsr_spmv_kernel<float,3> (level-0 tangent SpMV, FP32 values)", "bound": "hbm",
                "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                "peak_source": ("measured (MEASURED_PEAKS.json hbm_gbs)" if pk_kind == "measured"
                                else "fallback 6,650 GB/s (no MEASURED_PEAKS.json on this box)"),
                "algorithmic_bytes_per_launch": by, "avg_launch_ms": spmv_ms,
                "timing": "20 back-to-back launches on the library stream, CUDA events, after the timed region",
                "traffic": traffic, "traffic_source": traffic_src,
                "element_assembly_ms": asm_ms}
    roof = guarded("roofline", roofline)
    del M

    # ---- e2e: the same increments through the public C-ABI calls from host buffers ----
    def e2e_run():
        t_build = time.perf_counter()
        Me = fresh_model()
        build_s = time.perf_counter() - t_build
        t_warm = time.perf_counter()
        for s in range(1, args.warmup + 1):
            Me.newton(s / w.nsteps, tol=w.tol, maxiter=40, **solver_kw("mixed", have_mlp))
        warm_s = time.perf_counter() - t_warm
        # the step's result lands in a page-locked host buffer (allocated once, outside
        # the timed region), so the device -> host copy runs at the link's speed
        import torch
        u_pinned = torch.empty(Me.ndof, dtype=torch.float64, pin_memory=True).numpy()
        barrier()
        t0 = time.perf_counter()
        h2d = d2h = 0
        for s in range(args.warmup + 1, nsteps_needed + 1):
            w.apply(Me)                                   # this step's boundary-condition arrays, host -> device
            h, k = Me.newton(s / w.nsteps, tol=w.tol, maxiter=40, **solver_kw("mixed", have_mlp))
            L.check(L.lib().pfem_get_state(Me._ctx, L.ptr(u_pinned), None, None, None, None, None), Me._ctx)
            Ue = u_pinned.reshape(-1, 3).T                # the step's result, device -> host
            h2d += (w.dir_dofs.nbytes + w.dir_vals.nbytes + w.dir_ramp.nbytes + w.neu_dofs.nbytes
                    + w.neu_vals.nbytes)
            d2h += Ue.nbytes + 8 * 40 + 4 * 40
        sig = P.gauss_stress(Me)
        alp = P.equivalent_plastic_strain(Me)
        e2e_s = time.perf_counter() - t0
        d2h += sig.nbytes + alp.nbytes
        del Me
        return {"value": world * args.steps / max_over_ranks(e2e_s), "unit": "load-steps/s",
                "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
                "what": "the timed increments through the C-ABI from host arrays: per increment the "
                        "boundary-condition arrays are uploaded (pfem_set_bcs, pageable), pfem_newton runs, the "
                        "residual/Krylov histories come back and U comes back into a page-locked buffer "
                        "(pfem_get_state); Cauchy stress and alpha come back at the end",
                "model_build_s": build_s, "warmup_increments_s": warm_s}
    e2e = guarded("e2e", e2e_run)

    # ---- CPU baseline: whole increments of the reference algorithm on the oracle ----
    cpu = None
    if rank == 0 and world == 1:
        cpu = guarded("cpu_baseline", lambda: cpu_baseline(
            args.cpu_n, 1, args.cpu_increments, args.tol, kind=args.workload,
            bench_mesh=f"{args.n}^3, {3 * w.mesh.nnodes:,} DOF"))

    # ---- side arms on the same increments ----
    out_extra = {}
    if not args.no_compare:
        def timed_arm(kind, mlp=False):
            Mx = fresh_model()
            run_increments(Mx, w, 1, args.warmup, **solver_kw(kind, mlp))
            barrier()
            Mx.timer_start()
            itx = run_increments(Mx, w, args.warmup + 1, nsteps_needed, **solver_kw(kind, mlp))
            msx = max_over_ranks(Mx.timer_stop())
            barrier()
            U = Mx.U
            del Mx
            return {"U": U, "value": world * args.steps / (msx / 1e3), "ms_per_step": msx / args.steps,
                    "newton_iters": [a for a, _ in itx], "krylov_iters": [b for _, b in itx]}

        arms = {}
        arms["mixed_extrapolate"] = guarded("mixed_extrapolate", lambda: timed_arm("mixed_extrapolate"))
        arms["fp64_extrapolate"] = guarded("fp64_extrapolate", lambda: timed_arm("fp64_extrapolate"))
        arms["plain_fp64"] = guarded("plain_fp64", lambda: timed_arm("fp64"))
        arms["mixed_learned_amg_per_load_step"] = guarded(
            "mixed_learned_amg_per_load_step", lambda: timed_arm("mixed_amg_per_step", have_mlp))

        def truth():
            M3 = fresh_model()
            hist = []
            for s in range(1, nsteps_needed + 1):
                h, _ = M3.newton(s / w.nsteps, tol=TRUTH_TOL, maxiter=40, **solver_kw("truth", False))
                hist.append(h[-1])
            U = M3.U
            del M3
            return U, hist
        tr = guarded("truth", truth)
        what = {"mixed_extrapolate": "mixed precision with the extrapolation predictor",
                "fp64_extrapolate": "FP64 tangent and CG/AMG with the extrapolation predictor",
                "plain_fp64": "FP64 tangent and CG/AMG, previous-U predictor (the reference's), line search, "
                              "AMG rebuilt every load step (the reference's policy)",
                "mixed_learned_amg_per_load_step": "the headline arm with the AMG hierarchy rebuilt at the first "
                                                   "Newton iteration of every load step (the reference's policy)"}
        err = {}
        if tr is not None:
            U_true, last_res = tr
            nrm = np.linalg.norm(U_true)
            err["mixed_learned"] = float(np.linalg.norm(U_mixed - U_true) / nrm)
            out_extra["truth"] = {"what": f"FP64, inner solves to 1e-12, Newton to {TRUTH_TOL:g} relative "
                                          f"from the previous converged U, increments 1..{nsteps_needed}",
                                  "final_abs_residual_max": float(max(last_res))}
        for k, a in arms.items():
            if a is None:
                out_extra[k] = {"failed": errors.get(k, "unknown")}
                continue
            if tr is not None:
                err[k] = float(np.linalg.norm(a.pop("U") - U_true) / nrm)
            else:
                a.pop("U")
            out_extra[k] = {"what": what[k], **a}
        if err:
            out_extra["rel_disp_err_vs_fp64_truth"] = err
        # where the speed-up over the plain FP64 solver comes from (same timed increments)
        bd = {}
        pv = arms["plain_fp64"]["value"] if arms.get("plain_fp64") else None
        mx = arms["mixed_extrapolate"]["value"] if arms.get("mixed_extrapolate") else None
        fx = arms["fp64_extrapolate"]["value"] if arms.get("fp64_extrapolate") else None
        if pv:
            bd["total_vs_plain_fp64"] = value / pv
        if pv and fx:
            bd["extrapolation_predictor_alone"] = fx / pv
        if fx and mx:
            bd["mixed_precision_alone"] = mx / fx
        if mx:
            bd["learned_predictor_alone"] = value / mx
        if fx:
            bd["mixed_plus_learned_vs_fp64_extrapolate"] = value / fx
        out_extra["speedup_breakdown"] = bd

        # ---- the whole load path through pfem_solve (solve!): nsteps / wall time, model built ----
        def full_path():
            full = {}
            for name, kind in (("mixed_learned", "mixed"), ("plain_fp64", "fp64")):
                Mf = fresh_model()
                barrier()
                r = Mf.solve(nsteps=w.nsteps, tol=w.tol, maxiter=60, max_cuts=4, **solver_kw(kind, have_mlp))
                st = r.stats
                full[name] = {"converged": bool(r.converged),
                              "load_steps_per_s": w.nsteps / (st["time_total_ms"] / 1e3),
                              "wall_s": st["time_total_ms"] / 1e3, "newton_total": int(st["newton_iters_total"]),
                              "krylov_total": int(st["krylov_iters_total"]),
                              "amg_setup_s": st["time_amg_setup_ms"] / 1e3,
                              "load_step_cuts": int(st["load_step_cuts"])}
                del Mf
            full["speedup"] = full["mixed_learned"]["load_steps_per_s"] / full["plain_fp64"]["load_steps_per_s"]
            full["what"] = (f"all {w.nsteps} increments through pfem_solve (solve!): load steps / its wall time, "
                            "model construction excluded, AMG set-up included and reported")
            return full
        fp = guarded("full_path", full_path)
        out_extra["full_path"] = fp if fp is not None else {"failed": errors["full_path"]}

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
        if errors:
            line["failed_side_measurements"] = errors
        print(json.dumps(line), flush=True)
    reps.close()


if __name__ == "__main__":
    main()
