"""Generate the golden fixtures under tests/golden/ from the CPU oracle.

The reference (Julia) cannot run on these machines, so the oracle -- pinned by
tests/test_oracle_pins.py against the reference's own known-answer and
finite-difference tests -- produces these vectors.  Run:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from plasticity_b200 import workloads as W  # noqa: E402


def element_cases():
    mat = O.J2Material(200e3, 0.3, 250.0, 2000.0)
    nodes, el = O.box_mesh(1, 1, 1, 1, 1, 1)
    Xu = nodes.T[el[:, 0] - 1]
    S = np.array([[1.0, 0.15, 0.05], [0.0, 1.0, 0.1], [0.0, 0.0, 1.0]])
    Xd = Xu @ S.T + 0.03 * np.sin(np.arange(24)).reshape(8, 3)     # distorted element
    Fs = [np.eye(3),
          np.diag([1.001, 0.9995, 1.0003]),
          np.array([[1.05, 0.025, 0.005], [0.04, 0.98, 0.01], [0.01, 0.015, 1.02]]),
          np.array([[1.1, 0.05, 0.01], [0.08, 0.96, 0.02], [0.02, 0.03, 1.04]]),
          np.array([[0.85, 0.02, 0.0], [0.01, 1.07, 0.03], [0.0, 0.02, 1.06]])]
    out = {k: [] for k in ["fbar", "Xe", "ue", "cpi", "alpha", "Fe", "Ke", "tau", "flags", "cpi_new", "alpha_new"]}
    for fbar in (0, 1):
        for Xe in (Xu, Xd):
            cpi = np.tile([1, 1, 1, 0, 0, 0.0], (8, 1)); alpha = np.zeros(8)
            for F in Fs:
                ue = np.array([F @ x - x for x in Xe]).reshape(24)
                ue = ue + 1e-3 * np.cos(np.arange(24))           # non-homogeneous part
                r = O.element(fbar, mat, Xe, ue, cpi, alpha)
                for k, v in [("fbar", fbar), ("Xe", Xe), ("ue", ue), ("cpi", cpi), ("alpha", alpha),
                             ("Fe", r["Fe"]), ("Ke", r["Ke"]), ("tau", r["tau"]), ("flags", r["flags"]),
                             ("cpi_new", r["cpi_new"]), ("alpha_new", r["alpha"])]:
                    out[k].append(np.array(v))
                cpi, alpha = r["cpi_new"], r["alpha"]          # commit: path-dependent chain
    np.savez_compressed(os.path.join(HERE, "element_cases.npz"), **{k: np.array(v) for k, v in out.items()})


def solve_case(w, fname, line_search=False):
    """Newton counts from a run at the case's own tolerance (the reference's
    algorithm); U / stress / alpha / flags from a run tightened to 1e-12, which
    is the truth the 1e-8 displacement bar is measured against."""
    mat = O.J2Material(**{k: w.material[k] for k in ("E", "nu", "sigy0", "Hiso", "Hkin")})
    out = {}
    for tol in (w.tol, 1e-12):
        m = O.OracleModel(w.mesh.nodes, w.mesh.elements, mat, fbar=True, sigy0_e=w.sigy0_e)
        w.apply(m)
        res = m.solve(nsteps=w.nsteps, tol=tol, maxiter=25, line_search=line_search)
        assert res["converged"]
        if tol == w.tol:
            out["iters"] = np.array(res["iters"])
        else:
            out.update(U=m.U, tau=m.tau, alpha=m.alpha, flags=m.flags, sigma=m.gauss_stress(),
                       iters_tight=np.array(res["iters"]))
    np.savez_compressed(os.path.join(HERE, fname), nsteps=w.nsteps, tol=w.tol,
                        line_search=int(line_search), **out)
    print(fname, list(out["iters"]), float(np.abs(out["U"]).max()), float(out["alpha"].max()),
          float(out["flags"].mean()))


def solve_prefix_case(w, dims, last, fname, line_search=False):
    """The first `last` increments of a load path at a size where the LU needs a
    fill-reducing order: Newton counts at the case tolerance, U (FP64), Cauchy
    stress and alpha (FP32: the bars are 1e-6 relative to their maxima, FP32
    rounding is 6e-8 of each value) and flags (bit-packed) at 1e-12 after
    increment `last`."""
    mat = O.J2Material(**{k: w.material[k] for k in ("E", "nu", "sigy0", "Hiso", "Hkin")})
    perm = O.box_nd_dofs(*dims)
    out = {}
    for tol in (w.tol, 1e-12):
        m = O.OracleModel(w.mesh.nodes, w.mesh.elements, mat, fbar=True, sigy0_e=w.sigy0_e, nthreads=0)
        w.apply(m)
        ramp, fix = m.freeze_bcs()
        its = []
        for s in range(1, last + 1):
            conv, hist = m.newton(s / w.nsteps, ramp, fix, tol, 25, linsolve=O.nd_lu_solver(perm),
                                  line_search=line_search)
            assert conv, (fname, tol, s, hist)
            _, _, m.tau, m.flags = m.assemble(m.U, commit=True)
            its.append(len(hist))
            print(fname, tol, s, len(hist), flush=True)
        if tol == w.tol:
            out["iters"] = np.array(its)
        else:
            out.update(U=m.U, sigma=m.gauss_stress().astype(np.float32), alpha=m.alpha.astype(np.float32),
                       flags_bits=np.packbits(m.flags), ngp=len(m.flags), iters_tight=np.array(its))
    np.savez_compressed(os.path.join(HERE, fname), nsteps=w.nsteps, last=last, tol=w.tol,
                        line_search=int(line_search), **out)
    print(fname, list(out["iters"]), float(np.abs(out["U"]).max()), float(out["alpha"].max()))


CASES = {
    "element": element_cases,
    "config0": lambda: solve_case(W.config0(n=8), "config0_cube8.npz"),
    "cube4": lambda: solve_case(W.config2(n=4, nsteps=40), "cube4_jitter_compress.npz", line_search=True),
    "bar8": lambda: solve_case(W.config1(nx=8, ny=2, nz=2, nsteps=6, stretch=0.05), "bar8x2x2_neck.npz"),
    # configuration 1 at its stated size (80x16x16, 70,227 DOF), first 15 of its 60 increments
    "bar80": lambda: solve_prefix_case(W.config1(), (80, 16, 16), 15, "bar80x16x16_neck_15.npz"),
    # configuration 2's workload at 16^3 (14,739 DOF), the whole 40-increment path
    "cube16": lambda: solve_prefix_case(W.config2(n=16), (16, 16, 16), 40, "cube16_jitter_compress.npz"),
}

if __name__ == "__main__":
    for name in (sys.argv[1:] or list(CASES)):
        CASES[name]()
