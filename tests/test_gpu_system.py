"""The reference's system tests on the product path (small-strain kind, the
reference's default element): test_element.jl T12, test_solver.jl T13, T14,
T17 and test_assembly.jl T16, with the oracle's exact-LU answers beside the
analytical ones.  A one-element model has no aggregation hierarchy, so the
patch test uses a 2 x 2 x 2 mesh and T13 runs nx = 2 and 4."""
import numpy as np
import pytest

import plasticity_b200 as P

pytestmark = pytest.mark.gpu
E, NU = 210e3, 0.3


def _uniaxial_bcs(M, mesh, eps):
    M.fix(P.on_face(mesh, "xmin"), "x")
    M.fix(P.on_face(mesh, "ymin"), "y")
    M.fix(P.on_face(mesh, "zmin"), "z")
    M.prescribe(P.on_face(mesh, "xmax"), "x", eps)


def test_T12_patch_test_constant_strain():
    # test_element.jl:87-109: all nodes prescribed with u = (c x, 0, 0)
    mesh = P.box_mesh(1.3, 0.9, 1.1, 2, 2, 2)
    mat = P.J2Material(E, NU, 1e9)
    M = P.Model(mesh, mat, element="small")
    c = 1e-3
    nodes = np.arange(1, mesh.nnodes + 1)
    for n in nodes:
        M.prescribe([n], "x", c * mesh.nodes[0, n - 1], ramp=False)
    M.prescribe(nodes, "y", 0.0, ramp=False)
    M.prescribe(nodes, "z", 0.0, ramp=False)
    assert M.solve(nsteps=1, tol=1e-10).converged
    lam, G = mat.lam, mat.G
    exact = np.array([(lam + 2 * G) * c, lam * c, lam * c, 0, 0, 0])
    sig = P.gauss_stress(M).T
    assert np.abs(sig - exact).max() <= 1e-7 * E * c


@pytest.mark.parametrize("nx", [2, 4])
def test_T13_uniaxial_plastic_mesh_independent(nx):
    # test_solver.jl:22-51
    sy, Hi = 250.0, 1000.0
    mesh = P.box_mesh(1.0, 1.0, 1.0, nx, nx, nx)
    M = P.Model(mesh, P.J2Material(E, NU, sy, Hi), element="small")
    _uniaxial_bcs(M, mesh, 0.01)
    assert M.solve(nsteps=20, tol=1e-9, maxiter=25).converged
    an = sy + E * Hi / (E + Hi) * (0.01 - sy / E)
    sig = P.gauss_stress(M)[0]
    assert np.abs(sig - an).max() <= 1e-6 * an


def test_T14_cantilever_vs_beam_theory_and_oracle(oracle):
    # test_solver.jl:53-72
    Lb, Pz = 10.0, 100.0
    delta_beam = Pz * Lb ** 3 / (3 * E * (1.0 / 12))

    def tip(nx):
        mesh = P.box_mesh(Lb, 1.0, 1.0, nx, 4, 4)
        M = P.Model(mesh, P.J2Material(E, NU, 1e9), element="small")
        M.fix(P.on_face(mesh, "xmin"), "all")
        M.load(P.on_face(mesh, "xmax"), "z", -Pz, distribute=True)
        # near-exact inner solves, so the displacement itself (not only the
        # residual) matches the oracle's direct solve; 1e-10 stays above the
        # FP64 residual floor of this slender beam (about 6e-12 relative)
        assert M.solve(nsteps=1, tol=1e-10, lin_rtol=1e-12).converged
        return M, mesh

    M20, _ = tip(20)
    M40, mesh40 = tip(40)
    d20 = np.abs(P.nodal_displacements(M20)[2]).max()
    d40 = np.abs(P.nodal_displacements(M40)[2]).max()
    assert abs(d40 - delta_beam) / delta_beam < 0.10
    assert abs(d40 - delta_beam) <= abs(d20 - delta_beam) + 1e-6
    om = oracle.OracleModel(mesh40.nodes, mesh40.elements, oracle.J2Material(E, NU, 1e9), small=True)
    om.fix(P.on_face(mesh40, "xmin"), "all")
    om.load(P.on_face(mesh40, "xmax"), "z", -Pz, distribute=True)
    assert om.solve(nsteps=1, tol=1e-10)["converged"]
    assert np.linalg.norm(M40.U - om.U) / np.linalg.norm(om.U) < 1e-7


def test_T16_elastic_stiffness_symmetric_spd():
    # test_assembly.jl:38-58
    mesh = P.box_mesh(1.0, 1.0, 1.0, 3, 2, 2)
    M = P.Model(mesh, P.J2Material(E, NU, 1e9), element="small")
    K, _, _, _ = M.assemble(np.zeros(M.ndof))
    Kd = K.toarray()
    assert np.linalg.norm(Kd - Kd.T) <= 1e-10 * np.linalg.norm(Kd)
    fixed = {3 * (n - 1) + c for n in P.on_face(mesh, "xmin") for c in range(3)}
    free = [d for d in range(M.ndof) if d not in fixed]
    np.linalg.cholesky(Kd[np.ix_(free, free)])


def test_T17_reaction_balance():
    # test_solver.jl:101-125
    mesh = P.box_mesh(4.0, 1.0, 1.0, 8, 2, 2)
    M = P.Model(mesh, P.J2Material(E, NU, 1e9), element="small")
    M.fix(P.on_face(mesh, "xmin"), "all")
    Ptot = -50.0
    M.load(P.on_face(mesh, "xmax"), "z", Ptot, distribute=True)
    assert M.solve(nsteps=3, tol=1e-10).converged
    _, Fint, _, _ = M.assemble(M.U, want_K=False)
    Rz = sum(Fint[3 * (n - 1) + 2] for n in P.on_face(mesh, "xmin"))
    assert abs(Rz + Ptot) <= 1e-7 * abs(Ptot) + 1e-7
