"""Saturation (Voce) and kinematic hardening on the GPU against the oracle.

Element kernels: residual, tangent (FP64 and the FP32 tangent), stress, flags and
the committed state (Cp^-1 or eps_p, alpha, the back stress) for every element
kind and both laws (Materials.jl:159-250, FiniteStrain.jl:190-346, :503-547).
Solves: the reference's own T15 (test_solver.jl:74-93, Hkin = 500, quadratic
Newton), T18 (test_solver.jl:121-131, load-path consistency) and F11(b)
(test_finite_strain.jl:343-376, finite strain with Hkin = 2000), plus a
saturation solve, each checked against the oracle's exact-LU Newton.
"""
import numpy as np
import pytest

import plasticity_b200 as P
from plasticity_b200 import workloads as W

pytestmark = pytest.mark.gpu

MATS = {
    "voce": dict(E=206.9e3, nu=0.29, sigy0=450.0, Hiso=129.24, sigsat=715.0, delta=16.93),
    "kin": dict(E=210e3, nu=0.3, sigy0=250.0, Hiso=200.0, Hkin=2000.0),
}


def rel(a, b):
    a = np.asarray(a, float); b = np.asarray(b, float)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _pair(oracle, mesh, mat, kind, sigy0_e=None):
    M = P.Model(mesh, P.J2Material(**mat), element=kind, sigy0_e=sigy0_e)
    om = oracle.OracleModel(mesh.nodes, mesh.elements, oracle.J2Material(**mat), fbar=kind == "finite_fbar",
                            small=kind == "small", sigy0_e=sigy0_e)
    return M, om


@pytest.mark.parametrize("hard", ["voce", "kin"])
@pytest.mark.parametrize("kind", ["small", "finite", "finite_fbar"])
def test_assembly_and_commit_vs_oracle(oracle, kind, hard):
    w = W.config2(n=4)
    mat = MATS[hard]
    sy = w.sigy0_e * (mat["sigy0"] / 250.0)
    M, om = _pair(oracle, w.mesh, mat, kind, sy)
    X = w.mesh.nodes
    rng = np.random.default_rng(11)
    s = 2.0 * mat["sigy0"] / mat["E"]
    Ua = np.stack([2 * s * X[0], s * X[1], -4 * s * X[2]]).T.reshape(-1)
    Ub = np.stack([2 * s * X[2], 2 * s * X[0], -s * X[1]]).T.reshape(-1)
    U = Ua + Ub + 0.05 * s * rng.standard_normal(M.ndof)
    # committed history from two earlier, differently oriented loads
    for Uc in (0.6 * Ua, 1.1 * Ua + 0.5 * Ub):
        M.assemble(Uc, commit=True)
        om.assemble(Uc, commit=True)
    K, R, tau, fl = M.assemble(U)
    Ko, Ro, tauo, flo = om.assemble(U)
    assert rel(R, Ro) < 1e-10
    assert abs(K - Ko.tocsr()).max() / abs(Ko).max() < 1e-10
    assert rel(tau, tauo) < 1e-10
    assert np.array_equal(fl, flo) and fl.mean() > 0.3
    K32, R32, _, _ = M.assemble(U, precision="mixed")
    assert abs(K32 - Ko.tocsr()).max() / abs(Ko).max() < 1e-6
    assert rel(R32, Ro) < 1e-10
    M.assemble(U, commit=True)
    om.assemble(U, commit=True)
    st = M.state()
    slot = "epsp" if kind == "small" else "cpi"
    assert rel(st[slot], om.cpi) < 1e-10
    assert rel(st["alpha"], om.alpha) < 1e-10
    if kind != "small":
        assert rel(st["epsp"], om.epsp) < 1e-9
    if hard == "kin":
        assert np.abs(om.beta).max() > 0
        assert rel(M.back_stress(), om.beta) < 1e-10
    else:
        assert not M.back_stress().any()


def _uniaxial_bcs(M, mesh, eps):
    """uniaxial_cube (test_solver.jl:10-20): rollers on the min faces, xmax pulled."""
    M.fix(P.on_face(mesh, "xmin"), "x")
    M.fix(P.on_face(mesh, "ymin"), "y")
    M.fix(P.on_face(mesh, "zmin"), "z")
    M.prescribe(P.on_face(mesh, "xmax"), "x", eps)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_T15_kinematic_uniaxial_newton_vs_oracle(oracle, precision):
    # test_solver.jl:74-93: nx = 2, Hiso = 1000, Hkin = 500, 10 steps, tol 1e-9
    mat = dict(E=210e3, nu=0.3, sigy0=250.0, Hiso=1000.0, Hkin=500.0)
    mesh = P.box_mesh(1.0, 1.0, 1.0, 2, 2, 2)
    M, om = _pair(oracle, mesh, mat, "small")
    _uniaxial_bcs(M, mesh, 0.01)
    _uniaxial_bcs(om, mesh, 0.01)
    res = M.solve(nsteps=10, tol=1e-9, maxiter=15, precision=precision,
                  lin_rtol=1e-12 if precision == "fp64" else None)
    assert res.converged
    ores = om.solve(nsteps=10, tol=1e-12, maxiter=15)
    assert ores["converged"]
    h = next(h for h in res.residuals if len(h) >= 3)
    assert h[-1] < 1e-3 * h[-2] or h[-1] < 1e-9 * h[0]
    assert rel(M.U, om.U) < 1e-8
    sig = P.gauss_stress(M).T
    assert np.abs(sig - om.gauss_stress()).max() / np.abs(om.gauss_stress()).max() < 1e-6
    assert np.abs(M.state()["alpha"] - om.alpha).max() / om.alpha.max() < 1e-6
    assert rel(M.back_stress(), om.beta) < 1e-6


def test_T18_load_path_consistency_kinematic():
    # test_solver.jl:121-131: 10 vs 20 steps reach the same state
    mat = P.J2Material(210e3, 0.3, 250.0, Hiso=1000.0, Hkin=500.0)
    out = []
    for n in (10, 20):
        mesh = P.box_mesh(1.0, 1.0, 1.0, 1, 1, 1)
        M = P.Model(mesh, mat, element="small")
        _uniaxial_bcs(M, mesh, 0.01)
        assert M.solve(nsteps=n, tol=1e-10, lin_rtol=1e-12).converged
        out.append((P.gauss_stress(M)[0, 0], P.equivalent_plastic_strain(M)[0]))
    assert out[0][0] == pytest.approx(out[1][0], rel=1e-5)
    assert out[0][1] == pytest.approx(out[1][1], rel=1e-4)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_F11b_finite_kinematic_solve_vs_oracle(oracle, precision):
    # test_finite_strain.jl:343-376 case (b): 3x3x3 box, xmax pulled 0.08 in 4 steps
    mat = MATS["kin"]
    mesh = P.box_mesh(1.0, 1.0, 1.0, 3, 3, 3)
    M, om = _pair(oracle, mesh, mat, "finite")
    _uniaxial_bcs(M, mesh, 0.08)
    _uniaxial_bcs(om, mesh, 0.08)
    res = M.solve(nsteps=4, tol=1e-10, maxiter=25, precision=precision, linsolve="bicgstab",
                  lin_rtol=1e-12 if precision == "fp64" else None)
    assert res.converged
    if precision == "fp64":
        ref_iters = [len(h) for h in om.solve(nsteps=4, tol=1e-10, maxiter=25)["residuals"]]
        assert all(abs(a - b) <= 1 for a, b in zip(res.iters, ref_iters)), (res.iters, ref_iters)
    assert om.solve(nsteps=4, tol=1e-12, maxiter=25)["converged"]
    assert rel(M.U, om.U) < 1e-8
    sig = P.gauss_stress(M).T
    assert np.abs(sig - om.gauss_stress()).max() / np.abs(om.gauss_stress()).max() < 1e-6
    assert np.abs(M.state()["alpha"] - om.alpha).max() / om.alpha.max() < 1e-6
    assert rel(M.back_stress(), om.beta) < 1e-6
    assert np.array_equal(M.state()["flags"], om.flags)


@pytest.mark.parametrize("kind", ["small", "finite_fbar"])
def test_saturation_solve_vs_oracle(oracle, kind):
    # Simo's necking material (test_saturation.jl:22) on the uniaxial cube, 6% strain
    mat = MATS["voce"]
    mesh = P.box_mesh(1.0, 1.0, 1.0, 2, 2, 2)
    M, om = _pair(oracle, mesh, mat, kind)
    _uniaxial_bcs(M, mesh, 0.06)
    _uniaxial_bcs(om, mesh, 0.06)
    res = M.solve(nsteps=6, tol=1e-10, maxiter=25, linsolve="bicgstab", lin_rtol=1e-12)
    assert res.converged
    assert om.solve(nsteps=6, tol=1e-12, maxiter=25)["converged"]
    assert rel(M.U, om.U) < 1e-8
    sig = P.gauss_stress(M).T
    assert np.abs(sig - om.gauss_stress()).max() / np.abs(om.gauss_stress()).max() < 1e-6
    a = M.state()["alpha"]
    assert np.abs(a - om.alpha).max() / om.alpha.max() < 1e-6
    # on the saturated curve: sigma_xx of the homogeneous bar equals sigma_y(alpha)
    if kind == "small":
        m = P.J2Material(**mat)
        assert sig[:, 0].mean() == pytest.approx(m.yield_stress(a.mean()), rel=1e-6)


def test_back_stress_set_get_roundtrip():
    # pfem_set_back_stress / pfem_get_back_stress (GaussState.beta, Mesh.jl:124-130)
    mesh = P.box_mesh(1.0, 1.0, 1.0, 2, 2, 2)
    M = P.Model(mesh, P.J2Material(**MATS["kin"]), element="finite")
    b = np.random.default_rng(2).standard_normal((M.ngp, 6))
    M.set_back_stress(b)
    assert np.array_equal(M.back_stress(), b)
    M.reset()
    assert not M.back_stress().any()
    L_ = P.Model(mesh, P.J2Material(**MATS["voce"]), element="finite")
    assert not L_.back_stress().any()
    with pytest.raises(P.PfemError):
        L_.set_back_stress(b)
