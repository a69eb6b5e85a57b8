"""Finite-strain system tests of the reference (test_finite_strain.jl:97-113,
:270-300) on the product path, each also against the oracle's exact-LU answer:
the small-displacement limit (:finite -> :small), F-bar relieving volumetric
locking in near-incompressible plastic bending, and a large-rotation cantilever."""
import numpy as np
import pytest

import plasticity_b200 as P

pytestmark = pytest.mark.gpu
E, NU = 210e3, 0.3


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def _uniaxial(kind, disp):
    mesh = P.box_mesh(1.0, 1.0, 1.0, 2, 2, 2)
    M = P.Model(mesh, P.J2Material(E, NU, 250.0, 1000.0), element=kind)
    M.fix(P.on_face(mesh, "xmin"), "x"); M.fix(P.on_face(mesh, "ymin"), "y"); M.fix(P.on_face(mesh, "zmin"), "z")
    M.prescribe(P.on_face(mesh, "xmax"), "x", disp)
    assert M.solve(nsteps=5, tol=1e-10, lin_rtol=1e-12, linsolve="bicgstab").converged
    return M.U


def test_F1_small_displacement_limit():
    for disp in (1e-6, 1e-5, 1e-4):
        us, uf = _uniaxial("small", disp), _uniaxial("finite", disp)
        assert rel(uf, us) < 0.5 * disp + 1e-9


def _bend(kind, oracle_model=None):
    mesh = P.box_mesh(6.0, 1.0, 1.0, 6, 2, 2)
    mat = dict(E=E, nu=0.49, sigy0=250.0, Hiso=500.0)
    M = P.Model(mesh, P.J2Material(**mat), element=kind)
    for m in (M,) + ((oracle_model(mesh, mat),) if oracle_model else ()):
        m.fix(P.on_face(mesh, "xmin"), "all")
        m.load(P.on_face(mesh, "xmax"), "z", -10.0, distribute=True)
    # nu = 0.49: the FP64 residual floor (about 3e-9) rules out tighter than 1e-8
    res = M.solve(nsteps=6, tol=1e-8, maxiter=40, lin_rtol=1e-12, linsolve="bicgstab", line_search=True)
    return res.converged, M.U


def test_F6_F7_fbar_relieves_locking_and_matches_oracle(oracle):
    made = {}

    def om_factory(fbar):
        def f(mesh, mat):
            made["om"] = oracle.OracleModel(mesh.nodes, mesh.elements, oracle.J2Material(**mat), fbar=fbar)
            return made["om"]
        return f

    cf, Uf = _bend("finite_fbar", om_factory(True))
    om_f = made["om"]
    cs, Us = _bend("finite", om_factory(False))
    om_s = made["om"]
    assert cf and cs
    df, ds = np.abs(Uf.reshape(-1, 3)[:, 2]).max(), np.abs(Us.reshape(-1, 3)[:, 2]).max()
    assert df > 1.3 * ds
    for om, U in ((om_f, Uf), (om_s, Us)):
        assert om.solve(nsteps=6, tol=1e-8, maxiter=40)["converged"]
        assert rel(U, om.U) < 1e-6


def test_F8_large_rotation_cantilever(oracle):
    mesh = P.box_mesh(8.0, 1.0, 1.0, 8, 1, 1)
    M = P.Model(mesh, P.J2Material(E, NU, 1e9), element="finite")
    om = oracle.OracleModel(mesh.nodes, mesh.elements, oracle.J2Material(E, NU, 1e9), fbar=False)
    for m in (M, om):
        m.fix(P.on_face(mesh, "xmin"), "all")
        m.load(P.on_face(mesh, "xmax"), "z", -300.0, distribute=True)
    res = M.solve(nsteps=6, tol=1e-10, maxiter=40, lin_rtol=1e-12, linsolve="bicgstab", line_search=True)
    assert res.converged
    U = M.U
    assert np.all(np.isfinite(U)) and np.abs(U.reshape(-1, 3)[:, 2]).max() > 0.1
    assert om.solve(nsteps=6, tol=1e-10, maxiter=40)["converged"]
    assert rel(U, om.U) < 1e-6
