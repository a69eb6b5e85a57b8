"""The small-strain kind (Elements.jl:323-360, Materials.jl:159-250) on the GPU
against the oracle: element, assembly on a jittered mesh, and a full load path."""
import numpy as np
import pytest

import plasticity_b200 as P
from plasticity_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, float); b = np.asarray(b, float)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_small_strain_element_vs_oracle(oracle):
    rng = np.random.default_rng(21)
    mat = P.J2Material(200e3, 0.3, 250.0, 2000.0)
    omat = oracle.J2Material(200e3, 0.3, 250.0, 2000.0)
    nat = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                    [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)
    for case in range(3):
        Xe = 0.5 * (nat + 1) + 0.06 * rng.standard_normal((8, 3))
        ue = 0.003 * rng.standard_normal(24)
        epsp = 1e-4 * rng.standard_normal((8, 6))
        alpha = 1e-4 * rng.random(8)
        ref = oracle.element(2, omat, Xe, ue, cpi=epsp.reshape(-1), alpha=alpha)
        mesh = P.Mesh(np.ascontiguousarray(Xe.T), np.arange(1, 9, dtype=np.int64).reshape(8, 1))
        M = P.Model(mesh, mat, element="small")
        M.set_state(alpha=alpha, epsp=epsp)
        K, R, sig, fl = M.assemble(ue)
        assert rel(R, ref["Fe"]) < 1e-12, case
        assert rel(K.toarray(), ref["Ke"]) < 1e-12, case
        assert rel(sig, ref["tau"]) < 1e-12, case
        assert np.array_equal(fl, ref["flags"]), case
        K32, R32, _, _ = M.assemble(ue, precision="mixed")
        assert rel(K32.toarray(), ref["Ke"]) < 1e-6, case
        assert rel(R32, ref["Fe"]) < 1e-12, case
        M.assemble(ue, commit=True)
        st = M.state()
        assert rel(st["epsp"], ref["cpi_new"]) < 1e-12, case
        assert np.abs(st["alpha"] - ref["alpha"]).max() < 1e-14, case


def test_small_strain_assembly_jittered_vs_oracle(oracle):
    w = W.config2(n=5)
    mat = P.J2Material(**w.material)
    M = P.Model(w.mesh, mat, element="small", sigy0_e=w.sigy0_e)
    om = oracle.OracleModel(w.mesh.nodes, w.mesh.elements, oracle.J2Material(**w.material), small=True,
                            sigy0_e=w.sigy0_e)
    rng = np.random.default_rng(7)
    X = w.mesh.nodes
    U = np.stack([0.004 * X[0], 0.002 * X[1], -0.008 * X[2]]).T.reshape(-1) + 2e-4 * rng.standard_normal(M.ndof)
    M.assemble(0.5 * U, commit=True)
    om.assemble(0.5 * U, commit=True)
    K, R, sig, fl = M.assemble(U)
    Ko, Ro, sigo, flo = om.assemble(U)
    assert rel(R, Ro) < 1e-10
    assert abs(K - Ko.tocsr()).max() / abs(Ko).max() < 1e-10
    assert rel(sig, sigo) < 1e-10
    assert np.array_equal(fl, flo) and fl.mean() > 0.5


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_small_strain_solve_vs_oracle(oracle, precision):
    w = W.config0(n=6, nsteps=6)
    M = P.Model(w.mesh, P.J2Material(**w.material), element="small")
    w.apply(M)
    res = M.solve(nsteps=w.nsteps, tol=1e-10, maxiter=25, precision=precision,
                  lin_rtol=1e-12 if precision == "fp64" else None)
    assert res.converged
    om = oracle.OracleModel(w.mesh.nodes, w.mesh.elements, oracle.J2Material(**w.material), small=True)
    w.apply(om)
    ores = om.solve(nsteps=w.nsteps, tol=1e-12)
    assert ores["converged"]
    st = M.state()
    assert rel(st["U"], om.U) < 1e-8
    sig = P.gauss_stress(M).T
    assert np.abs(sig - om.gauss_stress()).max() / np.abs(om.gauss_stress()).max() < 1e-6
    assert np.abs(st["alpha"] - om.alpha).max() / max(np.abs(om.alpha).max(), 1e-300) < 1e-6
    assert np.array_equal(st["flags"], om.flags) and st["flags"].mean() > 0.2


def _roller_cube(n, sigy0=250.0, strain=0.01):
    """The reference's scaling cube (lagrangian/test/test_scaling.jl:16-26): rollers on
    xmin/ymin/zmin, xmax pulled to `strain`, E = 210 GPa, H = 1 GPa, small strain."""
    mesh = P.box_mesh(1.0, 1.0, 1.0, n, n, n)
    mat = P.J2Material(E=210e3, nu=0.3, sigy0=sigy0, Hiso=1000.0)
    M = P.Model(mesh, mat, element="small")
    M.fix(P.on_face(mesh, "xmin"), "x")
    M.fix(P.on_face(mesh, "ymin"), "y")
    M.fix(P.on_face(mesh, "zmin"), "z")
    M.prescribe(P.on_face(mesh, "xmax"), "x", strain)
    return M


def test_c1_cg_amg_matches_direct(oracle):
    """test_scaling.jl:29-55 (C1): the plastic roller cube, 16^3, 12 steps, Newton
    tol 1e-9: CG + AMG on the GPU against the direct (sparse LU) oracle, U and sigma
    within 10 x 1e-8."""
    M = _roller_cube(16)
    res = M.solve(nsteps=12, tol=1e-9, maxiter=25)
    assert res.converged
    om = oracle.OracleModel(M.mesh.nodes, M.mesh.elements,
                            oracle.J2Material(E=210e3, nu=0.3, sigy0=250.0, Hiso=1000.0), small=True)
    om.dir_dofs, om.dir_vals, om.dir_ramp = list(M.dir_dofs), list(M.dir_vals), [bool(r) for r in M.dir_ramp]
    ores = om.solve(nsteps=12, tol=1e-9)
    assert ores["converged"]
    assert rel(M.U, om.U) <= 1e-7
    assert rel(P.gauss_stress(M).T, om.gauss_stress()) <= 1e-7


def test_c2_mesh_independent_cg_count():
    """test_scaling.jl:84-104 (C2): elastic roller cubes n = 8, 12, 16, 20, one step to
    tol 1e-9; the largest CG count per Newton iteration grows with N at a log-log
    slope <= 0.15 and stays <= 25."""
    Ns, maxcg = [], []
    for n in (8, 12, 16, 20):
        M = _roller_cube(n, sigy0=1e9, strain=1e-3)
        res = M.solve(nsteps=1, tol=1e-9, maxiter=25)
        assert res.converged
        Ns.append(M.ndof)
        maxcg.append(max(res.cg_iters[0]))
    lx, ly = np.log(Ns), np.log(maxcg)
    slope = np.sum((lx - lx.mean()) * (ly - ly.mean())) / np.sum((lx - lx.mean()) ** 2)
    assert slope <= 0.15, (Ns, maxcg, slope)
    assert max(maxcg) <= 25, maxcg
