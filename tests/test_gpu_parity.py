"""GPU parity of the CUDA path against the CPU oracle and its golden fixtures.

Bars: CSR pattern, colors and per-Gauss-point elastic/plastic flags
bit-exact; converged displacements within 1e-8 relative; Cauchy stress and
equivalent plastic strain within 1e-6 relative; Newton iterations within +-1.
Element-level quantities use tighter FP64 bars (1e-9 normwise) and 1e-6 for the
FP32 tangent.
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import plasticity_b200 as P
from plasticity_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    a = np.asarray(a, float); b = np.asarray(b, float)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def model_from(w, **kw):
    mat = P.J2Material(**w.material)
    M = P.Model(w.mesh, mat, element="finite_fbar", sigy0_e=w.sigy0_e, **kw)
    w.apply(M)
    return M


def one_element_model(Xe, fbar, mat):
    mesh = P.Mesh(np.ascontiguousarray(np.asarray(Xe).T), np.arange(1, 9, dtype=np.int64).reshape(8, 1))
    return P.Model(mesh, mat, element="finite_fbar" if fbar else "finite")


def test_element_cases_vs_golden():
    g = np.load(os.path.join(GOLD, "element_cases.npz"))
    mat = P.J2Material(200e3, 0.3, 250.0, 2000.0)
    for i in range(len(g["fbar"])):
        M = one_element_model(g["Xe"][i], int(g["fbar"][i]), mat)
        M.set_state(cpi=g["cpi"][i], alpha=g["alpha"][i])
        K, R, tau, fl = M.assemble(g["ue"][i])
        assert rel(R, g["Fe"][i]) < 1e-10, i
        assert rel(K.toarray(), g["Ke"][i]) < 1e-9, i
        assert rel(tau, g["tau"][i]) < 1e-10, i
        assert np.array_equal(fl, g["flags"][i]), i
        K32, R32, _, _ = M.assemble(g["ue"][i], precision="mixed")
        assert rel(K32.toarray(), g["Ke"][i]) < 1e-6, i
        assert rel(R32, g["Fe"][i]) < 1e-10, i
        M.assemble(g["ue"][i], commit=True)
        st = M.state()
        assert rel(st["cpi"], g["cpi_new"][i]) < 1e-12, i
        assert np.abs(st["alpha"] - g["alpha_new"][i]).max() < 1e-12, i


@pytest.mark.parametrize("fbar", [True, False])
def test_assembly_vs_oracle_jittered(oracle, fbar):
    w = W.config2(n=5)
    mat = P.J2Material(**w.material)
    M = P.Model(w.mesh, mat, element="finite_fbar" if fbar else "finite", sigy0_e=w.sigy0_e)
    om = oracle.OracleModel(w.mesh.nodes, w.mesh.elements, oracle.J2Material(**w.material), fbar=fbar,
                            sigy0_e=w.sigy0_e)
    rng = np.random.default_rng(7)
    X = w.mesh.nodes
    U = (np.stack([0.004 * X[0], 0.002 * X[1], -0.008 * X[2]]).T.reshape(-1)
         + 2e-4 * rng.standard_normal(M.ndof))
    # a plastic committed state from one commit at a smaller load
    M.assemble(0.5 * U, commit=True)
    om.assemble(0.5 * U, commit=True)
    K, R, tau, fl = M.assemble(U)
    Ko, Ro, tauo, flo = om.assemble(U)
    assert rel(R, Ro) < 1e-10
    assert abs(K - Ko.tocsr()).max() / abs(Ko).max() < 1e-10
    assert rel(tau, tauo) < 1e-10
    assert np.array_equal(fl, flo) and fl.mean() > 0.5
    K32, _, _, _ = M.assemble(U, precision="mixed")
    assert abs(K32 - Ko.tocsr()).max() / abs(Ko).max() < 1e-6
    cp, rv = M.pattern()
    assert np.array_equal(cp, om.colptr) and np.array_equal(rv, om.rowval)


def _check_solve(M, g, prec_label, iters_tol=1):
    st = M.state()
    U = st["U"]
    assert rel(U, g["U"]) < 1e-8, prec_label
    sig = P.gauss_stress(M).T
    assert np.abs(sig - g["sigma"]).max() / np.abs(g["sigma"]).max() < 1e-6, prec_label
    a = st["alpha"]
    assert np.abs(a - g["alpha"]).max() / max(np.abs(g["alpha"]).max(), 1e-300) < 1e-6, prec_label
    assert np.array_equal(st["flags"], g["flags"]), prec_label


def _solve_pair(w, g, precision):
    """Newton counts at the case tolerance (FP64, near-exact inner solves, the
    reference's algorithm) and the converged state at tol 1e-10.  The golden
    counts come from direct solves; the F-bar tangent is nonsymmetric, so the
    near-exact inner solve here is BiCGStab to 1e-12 inside iterative
    refinement (a looser solve lets rounding move the line search's accept
    decisions, and with them the counts)."""
    ls = bool(int(g["line_search"]))
    if precision == "fp64":
        M = model_from(w)
        res = M.solve(nsteps=w.nsteps, tol=float(g["tol"]), maxiter=25, linsolve="bicgstab", lin_rtol=1e-12,
                      cg_itmax=1000, line_search=ls)
        assert res.converged
        assert np.abs(np.array(res.iters) - g["iters"]).max() <= 1, (res.iters, list(g["iters"]))
    M = model_from(w)
    res = M.solve(nsteps=w.nsteps, tol=1e-10, maxiter=25, precision=precision, line_search=ls,
                  lin_rtol=1e-12 if precision == "fp64" else None)
    assert res.converged
    _check_solve(M, g, precision)
    return res


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config0_solve_vs_golden(precision):
    g = np.load(os.path.join(GOLD, "config0_cube8.npz"))
    _solve_pair(W.config0(n=8), g, precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_jittered_compression_vs_golden(precision):
    g = np.load(os.path.join(GOLD, "cube4_jitter_compress.npz"))
    _solve_pair(W.config2(n=4, nsteps=int(g["nsteps"])), g, precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_necking_bar_vs_golden(precision):
    g = np.load(os.path.join(GOLD, "bar8x2x2_neck.npz"))
    _solve_pair(W.config1(nx=8, ny=2, nz=2, nsteps=6, stretch=0.05), g, precision)


def test_predictors_reach_same_solution():
    w = W.config0(n=6, nsteps=6)
    sols = {}
    for pred in ("previous", "extrapolate"):
        M = model_from(w)
        res = M.solve(nsteps=w.nsteps, tol=1e-10, predictor=pred, lin_rtol=1e-12)
        assert res.converged
        sols[pred] = (M.U, sum(res.iters))
    assert rel(sols["extrapolate"][0], sols["previous"][0]) < 1e-8
    assert sols["extrapolate"][1] <= sols["previous"][1]


def test_bicgstab_matches_cg():
    w = W.config0(n=6, nsteps=3)
    out = []
    for kry in ("cg", "bicgstab"):
        M = model_from(w)
        res = M.solve(nsteps=3, tol=1e-10, maxiter=40, linsolve=kry, lin_rtol=1e-9)
        assert res.converged
        out.append(M.U)
    assert rel(out[1], out[0]) < 1e-8


def test_linear_solve_vs_direct(oracle):
    w = W.config0(n=6, nsteps=4)
    M = model_from(w)
    M.newton(0.25, maxiter=25, tol=1e-10, lin_rtol=1e-12)
    U = M.U
    # the oracle's imposed tangent at the same displacement / committed state
    om = oracle.OracleModel(w.mesh.nodes, w.mesh.elements, oracle.J2Material(**w.material), fbar=True)
    w.apply(om)
    ramp, fix = om.freeze_bcs()   # oracle state is the pre-step (virgin) committed state
    Ko, Ro, _, _ = om.assemble(U)
    om.impose(Ko, Ro, ramp[0], ramp[1], True, 0.25, U)
    om.impose(Ko, Ro, fix[0], fix[1], False, 0.25, U)
    b = np.sin(np.arange(M.ndof) * 0.37)
    x_ref = spla.splu(Ko.tocsc()).solve(b)
    x, it = M.linear_solve(b, rtol=1e-10)
    assert rel(x, x_ref) < 1e-7 and it < 100


def test_inverted_element_fails_loudly():
    mat = P.J2Material(200e3, 0.3, 250.0, 2000.0)
    Xe = P.box_mesh(1, 1, 1, 1, 1, 1).nodes.T
    for fbar in (0, 1):
        M = one_element_model(Xe, fbar, mat)
        F = np.diag([-1.1, 1.0, 1.0])
        ue = np.array([F @ x - x for x in Xe]).reshape(24)
        with pytest.raises(P.PfemError) as e:
            M.assemble(ue)
        assert e.value.code == -3 and "inverted" in str(e.value)


def test_profile_reports_kernel_times():
    w = W.config0(n=8)
    M = model_from(w)
    for what in (0, 1, 2, 3):
        assert M.profile(what, reps=3) > 0


def test_reused_model_takes_new_boundary_values():
    """Boundary conditions re-applied to a reused model (same constrained dofs, new
    values: the fast path of pfem_set_bcs) give the solution a fresh model gives."""
    wa = W.config4_path(n=4, nsteps=4, seed=11)
    wb = W.config4_path(n=4, nsteps=4, seed=12)
    M = P.Model(wa.mesh, P.J2Material(**wa.material))
    wa.apply(M)
    M.solve(nsteps=4, tol=1e-10, maxiter=40, line_search=True)
    wb.apply(M)
    M.solve(nsteps=4, tol=1e-10, maxiter=40, line_search=True)
    F = P.Model(wb.mesh, P.J2Material(**wb.material))
    wb.apply(F)
    F.solve(nsteps=4, tol=1e-10, maxiter=40, line_search=True)
    assert rel(M.U, F.U) < 1e-12


def test_load_step_cutting_recovers_a_failed_increment():
    """30 % compression in one increment moves the top nodes of the 4-element-high
    cube further than an element is tall, so the reference's plain Newton inverts
    an element on its first iterate and stops (the oracle does the same); with
    max_cuts the increment is retried at half size until it converges and then
    carried on to the full load (the oracle needs four cuts).  The inner solves
    are near-exact BiCGStab, like the oracle's LU: the strongly compressed
    iterates have nonsymmetric, nearly singular F-bar tangents on which capped CG
    directions invert elements at random, so the number of cuts CG needs is not a
    property of the cutting logic."""
    w = W.config2(n=4, nsteps=1, compress=0.3)
    kw = dict(nsteps=1, tol=1e-8, maxiter=25, linsolve="bicgstab", lin_rtol=1e-10, cg_itmax=1000)
    M = model_from(w)
    plain = M.solve(**kw)
    assert not plain.converged
    M = model_from(w)
    cut = M.solve(max_cuts=10, **kw)
    assert cut.converged and cut.stats["load_step_cuts"] > 0, cut.stats
    assert len(cut.iters) == 1


def test_write_vtu_from_gpu_model(tmp_path):
    """write_vtu(filename, model) (Visualization.jl:129-205) from a solved GPU model."""
    import xml.etree.ElementTree as ET
    from plasticity_b200 import visualization as V
    w = W.config0(n=3, nsteps=2)
    M = model_from(w)
    assert M.solve(nsteps=2, tol=1e-10).converged
    fn = V.write_vtu(str(tmp_path / "gpu_cube"), M)
    root = ET.parse(fn).getroot()
    arrs = {da.get("Name"): np.array(da.text.split(), float) for da in root.iter("DataArray") if da.get("Name")}
    sig = P.gauss_stress(M).T.reshape(M.ne, 8, 6).mean(axis=1)
    assert np.allclose(arrs["Stress"].reshape(M.ne, 6), sig, rtol=1e-15, atol=0)
    assert np.allclose(arrs["Displacement"], M.U, rtol=0, atol=0)


def _check_prefix_state(M, g, label):
    """State after increment g["last"] against a prefix fixture: U (FP64) within
    1e-8 relative, Cauchy stress and alpha (stored in FP32) within 1e-6 of their
    maxima, flags bit-exact."""
    st = M.state()
    assert rel(st["U"], g["U"]) < 1e-8, label
    sig = P.gauss_stress(M).T
    assert np.abs(sig - g["sigma"]).max() / np.abs(g["sigma"]).max() < 1e-6, label
    a = st["alpha"]
    assert np.abs(a - g["alpha"]).max() / max(np.abs(g["alpha"]).max(), 1e-300) < 1e-6, label
    flags = np.unpackbits(g["flags_bits"])[: int(g["ngp"])]
    assert np.array_equal(st["flags"], flags), (label, int((st["flags"] != flags).sum()))


def _prefix_pair(w, g, precision):
    """Increments 1..last of a load path: Newton counts of the reference's algorithm
    (FP64, previous-U predictor, near-exact BiCGStab inner solves) within +-1 of the
    oracle's LU-based counts, then the state at Newton tolerance 1e-10."""
    last = int(g["last"])
    if precision == "fp64":
        M = model_from(w)
        its = []
        for s in range(1, last + 1):
            h, _ = M.newton(s / w.nsteps, tol=float(g["tol"]), maxiter=25, linsolve="bicgstab", lin_rtol=1e-12,
                            cg_itmax=1000)
            its.append(len(h))
        assert np.abs(np.array(its) - g["iters"]).max() <= 1, (its, list(g["iters"]))
    M = model_from(w)
    for s in range(1, last + 1):
        M.newton(s / w.nsteps, tol=1e-10, maxiter=40, precision=precision, line_search=True,
                 predictor="previous" if precision == "fp64" else "extrapolate",
                 lin_rtol=1e-12 if precision == "fp64" else None)
    _check_prefix_state(M, g, precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_necking_bar_full_size_vs_golden(precision):
    """Configuration 1 at its stated size (80 x 16 x 16 Hex8, 70,227 DOF; sigma_y -2 %
    in the middle element layer, 30 % stretch in 60 increments), the first 15
    increments, against the oracle's LU-based solve."""
    g = np.load(os.path.join(GOLD, "bar80x16x16_neck_15.npz"))
    _prefix_pair(W.config1(), g, precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_jittered_compression_cube16_vs_golden(precision):
    """The bench workload's generator at 16^3 (14,739 DOF): all 40 increments of the
    20 % compression against the oracle's LU-based solve."""
    g = np.load(os.path.join(GOLD, "cube16_jitter_compress.npz"))
    _prefix_pair(W.config2(n=16), g, precision)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gathered_assembly_matches_colored(precision, monkeypatch):
    """The row-owned gather (one element launch + one gather) and the colored
    in-place scatter assemble the same K and R (up to summation order) on a
    jittered mesh, and the same stress and flags."""
    w = W.config2(n=6)
    X = w.mesh.nodes
    U = np.stack([0.004 * X[0], 0.002 * X[1], -0.012 * X[2]]).T.reshape(-1)
    U += 2e-4 * np.random.default_rng(2).standard_normal(U.shape)
    out = []
    for mode in ("gathered", "colored"):
        if mode == "colored":
            monkeypatch.setenv("PFEM_ASSEMBLY", "colored")
        M = model_from(w)
        M.assemble(0.5 * U, commit=True)
        out.append(M.assemble(U, precision=precision))
        monkeypatch.delenv("PFEM_ASSEMBLY", raising=False)
    (Kg, Rg, tg, fg), (Kc, Rc, tc, fc) = out
    tolk = 1e-12 if precision == "fp64" else 1e-6
    assert abs(Kg - Kc).max() <= tolk * abs(Kc).max()
    assert np.linalg.norm(Rg - Rc) <= 1e-13 * np.linalg.norm(Rc)
    assert np.array_equal(tg, tc) and np.array_equal(fg, fc)


def test_boundary_condition_update_semantics():
    """What the cheap same-dofs path of pfem_set_bcs must keep: a Dirichlet dof given
    twice takes its last value (_freeze_bcs, Solver.jl:192-218), and Neumann loads
    changed on a reused model act as on a fresh model (bit for bit)."""
    w = W.config0(n=3, nsteps=2)
    U = 1e-3 * np.random.default_rng(3).standard_normal(3 * w.mesh.nnodes)

    def residual(dd, dv, dr, nd, nv, M=None):
        if M is None:
            M = P.Model(w.mesh, P.J2Material(**w.material))
        M.dir_dofs, M.dir_vals, M.dir_ramp = dd, dv, dr
        M.neu_dofs, M.neu_vals = nd, nv
        M._bcs_dirty = True
        M.set_displacement(U)
        return M, M.residual(0.5)[1]

    d, v, r = w.dir_dofs, w.dir_vals, w.dir_ramp
    top = r == 1
    dd = np.concatenate([d[top], d])                       # the top dofs first at 0.02, then their own values
    dv = np.concatenate([np.full(int(top.sum()), 0.02), v])
    dr = np.concatenate([r[top], r])
    none_i, none_v = np.zeros(0, np.int64), np.zeros(0)
    _, Ra = residual(dd, dv, dr, none_i, none_v)
    _, Rb = residual(d, v, r, none_i, none_v)
    assert np.array_equal(Ra, Rb)
    nd = d[top][:5] - 2                                    # free x dofs of top-face nodes
    M, _ = residual(d, v, r, nd, np.full(5, 1.0))
    M, R2 = residual(d, v, r, nd, np.full(5, 3.0), M)       # same dofs, new loads: the cheap path
    _, R3 = residual(d, v, r, nd, np.full(5, 3.0))
    assert np.array_equal(R2, R3)
    assert not np.array_equal(R2, residual(d, v, r, none_i, none_v)[1])  # the loads do act
