"""Pin the oracle's saturation (Voce) and kinematic-hardening branches.

Each test restates one from vinaysrao1/plasticity lagrangian/test/*.jl:
test_saturation.jl T9-T12 (Voce return map), test_material.jl T4/T5
(Bauschinger, tangent with Hkin > 0), test_finite_strain.jl F2 (the master FD
gate with the reference's Hkin = 500 material), F4b (objectivity of the
rotation-neutralised back stress) and F9b (consistent, non-symmetric tangent
with kinematic hardening).  Reference SMatrix literals are column-major; the
3x3 arrays below are written row by row.
"""
import numpy as np
import pytest

SIMO = dict(E=206.9e3, nu=0.29, sigy0=450.0, sigsat=715.0, delta=16.93, Hiso=129.24)


def _voce(O):
    return O.J2Material(SIMO["E"], SIMO["nu"], SIMO["sigy0"], Hiso=SIMO["Hiso"],
                        sigsat=SIMO["sigsat"], delta=SIMO["delta"])


def test_T9_saturation_reduces_to_linear_bitwise(oracle):
    # test_saturation.jl:25-38
    mL = oracle.J2Material(210e3, 0.3, 250.0, Hiso=1000.0)
    mS = oracle.J2Material(210e3, 0.3, 250.0, Hiso=1000.0, sigsat=250.0, delta=25.0)
    for eps in ([0.01, -0.002, 0.001, 0.003, 0, 0], [0.02, -0.005, -0.005, 0.0, 0.004, 0.0],
                [1e-4, -2e-5, 3e-5, 1e-5, -1e-5, 2e-5]):
        rL = oracle.return_map(mL, eps)
        rS = oracle.return_map(mS, eps)
        assert np.array_equal(rL[0], rS[0])
        assert rL[3] == rS[3]
        assert np.array_equal(rL[4], rS[4])


@pytest.mark.parametrize("eps", [[0.02, -0.003, -0.003, 0.004, 0, 0], [0.05, -0.01, -0.01, 0.0, 0.002, 0.0],
                                 [0.10, -0.02, -0.02, 0.01, 0.0, 0.0]])
def test_T10_saturation_lands_on_updated_surface(oracle, eps):
    # test_saturation.jl:40-56
    mat = _voce(oracle)
    s, _, _, a, _, _ = oracle.return_map(mat, eps)
    p = s[:3].mean()
    d = s - np.array([p, p, p, 0, 0, 0])
    q = np.sqrt(1.5 * (d[0] ** 2 + d[1] ** 2 + d[2] ** 2 + 2 * (d[3] ** 2 + d[4] ** 2 + d[5] ** 2)))
    assert q == pytest.approx(mat.yield_stress(a), rel=1e-12)
    assert a > 0


@pytest.mark.parametrize("exx", [0.01, 0.03, 0.08, 0.15])
def test_T11_uniaxial_saturation_curve(oracle, exx):
    # test_saturation.jl:58-101: incremental uniaxial stress vs the scalar
    # fixed point sigma = sigma_y(exx - sigma/E)
    mat = _voce(oracle)
    ep = np.zeros(6); b = np.zeros(6); a = 0.0; el = 0.0
    n = 80
    for k in range(1, n + 1):
        e = exx * k / n
        for _ in range(60):
            s, _, _, _, D, _ = oracle.return_map(mat, [e, el, el, 0, 0, 0], ep, b, a)
            el -= s[1] / (D[1, 1] + D[1, 2])
            if abs(s[1]) < 1e-10:
                break
        s, ep, b, a, _, _ = oracle.return_map(mat, [e, el, el, 0, 0, 0], ep, b, a)
    s, _, _, a, _, _ = oracle.return_map(mat, [exx, el, el, 0, 0, 0], ep, b, a)
    sig = SIMO["sigy0"]
    for _ in range(200):
        epa = max(exx - sig / SIMO["E"], 0.0)
        sig = 0.5 * sig + 0.5 * mat.yield_stress(epa)
    assert s[0] == pytest.approx(sig, rel=1e-4)
    assert abs(s[1]) < 1e-5 * s[0]
    assert s[0] < SIMO["sigsat"] + SIMO["Hiso"] * a + 1e-6


@pytest.mark.parametrize("eps", [[0.02, 0, 0, 0, 0, 0], [0.03, -0.006, 0, 0.004, 0.002, 0],
                                 [0.05, -0.012, 0.004, 0.006, 0.001, 0.003], [0.0, 0.0, 0.0, 0.02, 0, 0]])
def test_T12_saturation_tangent_fd(oracle, eps):
    # test_saturation.jl:103-126
    mat = _voce(oracle)
    eps = np.array(eps, float)
    D = oracle.return_map(mat, eps)[4]
    h = 1e-7
    Dfd = np.zeros((6, 6))
    for j in range(6):
        e = np.zeros(6); e[j] = h
        Dfd[:, j] = (oracle.return_map(mat, eps + e)[0] - oracle.return_map(mat, eps - e)[0]) / (2 * h)
    assert np.linalg.norm(D - Dfd) / np.linalg.norm(D) <= 1e-6
    assert np.linalg.norm(D - D.T) <= 1e-12 * np.linalg.norm(D)


def test_T4_bauschinger(oracle):
    # test_material.jl:78-126: pure kinematic hardening, elastic span 2 sigy0
    sy = 250.0
    mat = oracle.J2Material(210e3, 0.3, sy, Hiso=0.0, Hkin=2000.0)
    path = np.concatenate([np.linspace(0, 0.01, 500), np.linspace(0.01, -0.01, 1000)])
    ep = np.zeros(6); b = np.zeros(6); a = 0.0; el = 0.0
    sx, al = [], []
    for e in path:
        for _ in range(80):
            s, _, _, _, D, _ = oracle.return_map(mat, [e, el, el, 0, 0, 0], ep, b, a)
            el -= s[1] / (D[1, 1] + D[1, 2])
            if abs(s[1]) < 1e-10:
                break
        s, ep, b, a, _, _ = oracle.return_map(mat, [e, el, el, 0, 0, 0], ep, b, a)
        sx.append(s[0]); al.append(a)
    nf = 500
    rstart = next(k for k in range(nf + 1, len(sx)) if al[k] > al[k - 1] + 1e-12)
    assert max(sx) - sx[rstart - 1] == pytest.approx(2 * sy, rel=2e-2)
    assert max(sx) > sy


@pytest.mark.parametrize("eps", [[0.01, 0, 0, 0, 0, 0], [0.005, -0.001, 0, 0.004, 0.002, 0],
                                 [0.003, -0.002, 0.001, 0.002, 0.001, 0.0015]])
def test_T5_tangent_fd_with_kinematic(oracle, eps):
    # test_material.jl:128-147 (Hiso = 1000, Hkin = 800), from a nonzero back stress
    mat = oracle.J2Material(210e3, 0.3, 250.0, Hiso=1000.0, Hkin=800.0)
    b0 = np.array([20.0, -8.0, -12.0, 5.0, -3.0, 2.0])
    eps = np.array(eps, float)
    D = oracle.return_map(mat, eps, None, b0, 0.01)[4]
    h = 1e-7
    Dfd = np.zeros((6, 6))
    for j in range(6):
        e = np.zeros(6); e[j] = h
        Dfd[:, j] = (oracle.return_map(mat, eps + e, None, b0, 0.01)[0] -
                     oracle.return_map(mat, eps - e, None, b0, 0.01)[0]) / (2 * h)
    assert np.linalg.norm(D - Dfd) / np.linalg.norm(D) <= 1e-5
    assert np.linalg.norm(D - D.T) <= 1e-12 * np.linalg.norm(D)


# ---------------------------------------------------------------- finite strain
def _unit(O):
    nodes, el = O.box_mesh(1, 1, 1, 1, 1, 1)
    return nodes.T[el[:, 0] - 1]


def _ue(Xe, F):
    return np.array([F @ x - x for x in Xe]).reshape(24)


def _fd(O, fbar, mat, Xe, ue, st=None, h=1e-7):
    st = st or {}
    kw = dict(cpi=st.get("cpi"), alpha=st.get("alpha"), beta=st.get("beta"))
    K = O.element(fbar, mat, Xe, ue, **kw)["Ke"]
    Kfd = np.zeros((24, 24))
    for j in range(24):
        up = ue.copy(); up[j] += h
        um = ue.copy(); um[j] -= h
        Kfd[:, j] = (O.element(fbar, mat, Xe, up, **kw)["Fe"] - O.element(fbar, mat, Xe, um, **kw)["Fe"]) / (2 * h)
    return np.linalg.norm(Kfd - K) / np.linalg.norm(K), np.linalg.norm(K - K.T) / np.linalg.norm(K)


def _commit(O, fbar, mat, Xe, ue, st=None):
    st = st or {}
    r = O.element(fbar, mat, Xe, ue, cpi=st.get("cpi"), alpha=st.get("alpha"), beta=st.get("beta"))
    return dict(cpi=r["cpi_new"], alpha=r["alpha"], beta=r["beta"])


MAT_F2 = dict(E=210e3, nu=0.3, sigy0=250.0, Hiso=1000.0, Hkin=500.0)
F1c = np.array([[1.05, 0.025, 0.005], [0.04, 0.98, 0.01], [0.01, 0.015, 1.02]])
F2c = np.array([[1.1, 0.05, 0.01], [0.08, 0.96, 0.02], [0.02, 0.03, 1.04]])


@pytest.mark.parametrize("F", [np.diag([1.1, 0.95, 1.03]),
                               np.array([[1.08, 0.03, 0.01], [0.04, 0.97, 0.0], [0.0, 0.02, 1.05]])])
def test_F2a_master_gate_elastic_kinematic_material(oracle, F):
    # test_finite_strain.jl:115-127
    mat = oracle.J2Material(**MAT_F2)
    Xe = _unit(oracle)
    assert _fd(oracle, 0, mat, Xe, _ue(Xe, F))[0] < 1e-6


def test_F2b_master_gate_plastic_path_kinematic_material(oracle):
    # test_finite_strain.jl:129-140: committed history includes the back stress
    mat = oracle.J2Material(**MAT_F2)
    Xe = _unit(oracle)
    st = None
    for k in range(1, 9):
        Fk = np.diag([1 + 0.02 * k, 1 - 0.008 * k, 1 - 0.008 * k])
        assert _fd(oracle, 0, mat, Xe, _ue(Xe, Fk), st)[0] < 1e-6
        st = _commit(oracle, 0, mat, Xe, _ue(Xe, Fk), st)
    assert st["alpha"].max() > 0.05
    assert np.abs(st["beta"]).max() > 0


@pytest.mark.parametrize("fbar", [0, 1])
def test_F2cd_master_gate_noncoaxial_kinematic_material(oracle, fbar):
    # test_finite_strain.jl:142-161
    mat = oracle.J2Material(**MAT_F2)
    Xe = _unit(oracle)
    assert _fd(oracle, fbar, mat, Xe, _ue(Xe, F2c))[0] < 1e-6
    st = _commit(oracle, fbar, mat, Xe, _ue(Xe, F1c))
    assert np.abs(st["beta"]).max() > 0
    assert _fd(oracle, fbar, mat, Xe, _ue(Xe, F2c), st)[0] < 1e-6


def test_F4b_objectivity_with_kinematic_hardening(oracle):
    # test_finite_strain.jl:197-223
    mat = oracle.J2Material(210e3, 0.3, 250.0, Hiso=200.0, Hkin=2000.0)
    F1 = np.array([[1.2, 0.03, 0], [0.05, 0.92, 0], [0, 0, 0.95]])
    u1 = oracle.finite_update(mat, F1)
    assert u1["alpha"] > 0 and np.linalg.norm(u1["beta"]) > 0
    F2 = np.array([[1.3, 0.06, 0.0], [0.08, 0.9, 0.02], [0.02, 0.01, 0.97]])

    def sig(F):
        t = oracle.finite_update(mat, F, u1["cpi_new"], u1["alpha"], u1["beta"])["tau"]
        return np.array([[t[0], t[3], t[5]], [t[3], t[1], t[4]], [t[5], t[4], t[2]]]) / np.linalg.det(F)

    s1 = sig(F2)
    for th in (0.1, np.deg2rad(120.0), 3.0):
        Q = np.array([[np.cos(th), -np.sin(th), 0], [np.sin(th), np.cos(th), 0], [0, 0, 1]])
        assert np.linalg.norm(sig(Q @ F2) - Q @ s1 @ Q.T) / np.linalg.norm(s1) < 1e-10


def test_F9b_kinematic_tangent_consistent_nonsymmetric(oracle):
    # test_finite_strain.jl:323-341
    mat = oracle.J2Material(210e3, 0.3, 250.0, Hiso=200.0, Hkin=2000.0)
    Xe = _unit(oracle)
    F1 = np.array([[1.1, 0.03, 0.0], [0.04, 0.95, 0.01], [0.01, 0.02, 0.97]])
    F2 = np.array([[1.18, 0.06, 0.02], [0.09, 0.92, 0.03], [0.03, 0.04, 1.0]])
    st = _commit(oracle, 0, mat, Xe, _ue(Xe, F1))
    assert st["alpha"].max() > 0
    rel, sym = _fd(oracle, 0, mat, Xe, _ue(Xe, F2), st)
    assert rel < 1e-6
    assert sym > 1e-6


def test_small_strain_kinematic_element_fd(oracle):
    # Elements.jl:323-360 with the kinematic return map: consistent and symmetric
    mat = oracle.J2Material(210e3, 0.3, 250.0, Hiso=200.0, Hkin=2000.0)
    Xe = _unit(oracle)
    st = _commit(oracle, 2, mat, Xe, _ue(Xe, F1c))
    assert np.abs(st["beta"]).max() > 0
    rel, sym = _fd(oracle, 2, mat, Xe, _ue(Xe, F2c), st)
    assert rel < 1e-6 and sym < 1e-10
