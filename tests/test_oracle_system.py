"""Pin the oracle's small-strain path (the reference's default element kind)
against the reference's element and system tests: test_element.jl T9-T12,
test_solver.jl T13, T14, T17, T19 and test_assembly.jl T16.  The product path
is checked against the same properties in tests/test_gpu_system.py."""
import numpy as np
import pytest

E, NU = 210e3, 0.3


def _uniaxial(O, nx, eps, **mat):
    """uniaxial_cube (test_solver.jl:10-20): rollers on the min faces, xmax pulled."""
    nodes, el = O.box_mesh(1.0, 1.0, 1.0, nx, nx, nx)
    om = O.OracleModel(nodes, el, O.J2Material(E, NU, **mat), small=True)
    X = nodes
    face = lambda d, v: [i + 1 for i in range(X.shape[1]) if abs(X[d, i] - v) < 1e-9]
    om.fix(face(0, 0.0), "x"); om.fix(face(1, 0.0), "y"); om.fix(face(2, 0.0), "z")
    om.prescribe(face(0, 1.0), "x", eps)
    return om


def test_T9_T11_partition_of_unity_and_rigid_translation(oracle):
    # test_element.jl:19-33, :53-85: a rigid translation gives zero strain and force
    nodes, el = oracle.box_mesh(2.0, 1.5, 1.0, 2, 2, 2)
    Xe = nodes.T[el[:, 0] - 1]
    mat = oracle.J2Material(E, NU, 1e9)
    ue = np.tile([0.3, -0.2, 0.5], 8)
    r = oracle.element(2, mat, Xe, ue)
    assert np.abs(r["Fe"]).max() <= 1e-9
    assert np.abs(r["tau"]).max() <= 1e-9
    # infinitesimal rotation: strain zero to linear order
    w = np.array([1e-6, -2e-6, 3e-6])
    ur = np.cross(w, Xe).reshape(24)
    assert np.abs(oracle.element(2, mat, Xe, ur)["tau"]).max() <= 1e-10 * E


def test_T10_volume(oracle):
    # test_element.jl:35-51: sum of detJ w over an element = its volume, seen
    # through the internal force of a uniform stress: sum over x-faces of F_x = sigma_xx * area
    nodes, el = oracle.box_mesh(2.0, 3.0, 4.0, 2, 3, 4)
    Xe = nodes.T[el[:, 0] - 1]                  # 1 x 1 x 1 element
    mat = oracle.J2Material(E, NU, 1e9)
    c = 1e-4
    ue = np.stack([c * Xe[:, 0], 0 * Xe[:, 0], 0 * Xe[:, 0]], axis=1).reshape(24)
    r = oracle.element(2, mat, Xe, ue)
    sxx = (mat.lam + 2 * mat.G) * c
    fx = r["Fe"].reshape(8, 3)[:, 0]
    xmax = Xe[:, 0] > Xe[:, 0].min() + 1e-9
    assert fx[xmax].sum() == pytest.approx(sxx * 1.0 * 1.0, rel=1e-12)


def test_T12_patch_test_constant_strain(oracle):
    # test_element.jl:87-109: every node prescribed with u = (c x, 0, 0)
    nodes, el = oracle.box_mesh(1.3, 0.9, 1.1, 1, 1, 1)
    mat = oracle.J2Material(E, NU, 1e9)
    om = oracle.OracleModel(nodes, el, mat, small=True)
    c = 1e-3
    for n in range(nodes.shape[1]):
        om.prescribe([n + 1], "x", c * nodes[0, n], ramp=False)
        om.prescribe([n + 1], "y", 0.0, ramp=False)
        om.prescribe([n + 1], "z", 0.0, ramp=False)
    assert om.solve(nsteps=1, tol=1e-10)["converged"]
    exact = mat.cmat() @ np.array([c, 0, 0, 0, 0, 0])
    assert np.abs(om.gauss_stress() - exact).max() <= 1e-7 * E * c


@pytest.mark.parametrize("nx", [1, 2, 4])
def test_T13_uniaxial_plastic_mesh_independent(oracle, nx):
    # test_solver.jl:22-51: sigma_xx = sigy0 + Ht (eps - eps_y) on every mesh
    sy, Hi = 250.0, 1000.0
    om = _uniaxial(oracle, nx, 0.01, sigy0=sy, Hiso=Hi)
    assert om.solve(nsteps=20, tol=1e-9)["converged"]
    Ht = E * Hi / (E + Hi)
    an = sy + Ht * (0.01 - sy / E)
    sig = om.gauss_stress()[:, 0]
    assert np.abs(sig - an).max() <= 1e-6 * an


def test_T14_cantilever_vs_beam_theory(oracle):
    # test_solver.jl:53-72: tip deflection within 10 % of Euler-Bernoulli, converging
    Lb, Pz = 10.0, 100.0
    delta_beam = Pz * Lb ** 3 / (3 * E * (1.0 / 12))

    def tip(nx):
        nodes, el = oracle.box_mesh(Lb, 1.0, 1.0, nx, 4, 4)
        om = oracle.OracleModel(nodes, el, oracle.J2Material(E, NU, 1e9), small=True)
        xmin = [i + 1 for i in range(nodes.shape[1]) if abs(nodes[0, i]) < 1e-9]
        xmax = [i + 1 for i in range(nodes.shape[1]) if abs(nodes[0, i] - Lb) < 1e-9]
        om.fix(xmin, "all")
        om.load(xmax, "z", -Pz, distribute=True)
        assert om.solve(nsteps=1, tol=1e-9)["converged"]
        return np.abs(om.U.reshape(-1, 3)[:, 2]).max()

    d20, d40 = tip(20), tip(40)
    assert abs(d40 - delta_beam) / delta_beam < 0.10
    assert abs(d40 - delta_beam) <= abs(d20 - delta_beam) + 1e-6


def test_T16_elastic_stiffness_symmetric_spd(oracle):
    # test_assembly.jl:38-58
    nodes, el = oracle.box_mesh(1.0, 1.0, 1.0, 3, 2, 2)
    om = oracle.OracleModel(nodes, el, oracle.J2Material(E, NU, 1e9), small=True)
    K, _, _, _ = om.assemble(np.zeros(om.ndof))
    Kd = K.toarray()
    assert np.linalg.norm(Kd - Kd.T) <= 1e-10 * np.linalg.norm(Kd)
    fixed = {3 * i + c for i in range(nodes.shape[1]) if abs(nodes[0, i]) < 1e-9 for c in range(3)}
    free = [d for d in range(om.ndof) if d not in fixed]
    np.linalg.cholesky(Kd[np.ix_(free, free)])


def test_T17_reaction_balance(oracle):
    # test_solver.jl:101-125: reactions at the clamped face balance the applied load
    nodes, el = oracle.box_mesh(4.0, 1.0, 1.0, 8, 2, 2)
    om = oracle.OracleModel(nodes, el, oracle.J2Material(E, NU, 1e9), small=True)
    xmin = [i + 1 for i in range(nodes.shape[1]) if abs(nodes[0, i]) < 1e-9]
    xmax = [i + 1 for i in range(nodes.shape[1]) if abs(nodes[0, i] - 4.0) < 1e-9]
    om.fix(xmin, "all")
    Ptot = -50.0
    om.load(xmax, "z", Ptot, distribute=True)
    assert om.solve(nsteps=3, tol=1e-10)["converged"]
    _, Fint, _, _ = om.assemble(om.U)
    Rz = sum(Fint[3 * (n - 1) + 2] for n in xmin)
    assert abs(Rz + Ptot) <= 1e-7 * abs(Ptot) + 1e-7


def test_T19_unload_is_elastic(oracle):
    # test_solver.jl:139-175
    mat = oracle.J2Material(E, NU, 250.0, 1000.0)

    def step(ep, b, a, exx):
        el = 0.0
        for _ in range(80):
            s, _, _, _, D, _ = oracle.return_map(mat, [exx, el, el, 0, 0, 0], ep, b, a)
            el -= s[1] / (D[1, 1] + D[1, 2])
            if abs(s[1]) < 1e-11:
                break
        s, ep2, b2, a2, _, _ = oracle.return_map(mat, [exx, el, el, 0, 0, 0], ep, b, a)
        return s[0], ep2, b2, a2

    ep = np.zeros(6); b = np.zeros(6); a = 0.0; sl = 0.0
    for n in range(1, 101):
        sl, ep, b, a = step(ep, b, a, 0.01 * n / 100)
    su, _, _, au = step(ep, b, a, 0.01 - 1e-5)
    assert (su - sl) / -1e-5 == pytest.approx(E, rel=1e-3)
    assert abs(au - a) <= 1e-12
