"""The device smoothed-aggregation hierarchy: Galerkin coarse operators, a
contracting cycle, and AMG-preconditioned CG on a three-level mesh."""
import numpy as np
import pytest

import plasticity_b200 as P
from plasticity_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _model(n, precision):
    w = W.config2(n=n)
    M = P.Model(w.mesh, P.J2Material(**w.material), sigy0_e=w.sigy0_e)
    w.apply(M)
    X = w.mesh.nodes
    rng = np.random.default_rng(5)
    U = np.stack([0.002 * X[0], 0.001 * X[1], -0.006 * X[2]]).T.reshape(-1) + 1e-4 / n * rng.standard_normal(M.ndof)
    M.set_displacement(U)
    _, R = M.residual(0.03, precision=precision)
    return M, R


def test_galerkin_coarse_operator_fp64():
    M, R = _model(10, "fp64")
    M.linear_solve(-R, rtol=1e-8, rebuild=True, precision="fp64")
    A0, P0, A1 = M.amg_dense(0, 0), M.amg_dense(0, 1), M.amg_dense(1, 0)
    assert P0.shape == (A0.shape[0], A1.shape[0])
    G = P0.T @ A0 @ P0
    assert np.abs(G - A1).max() <= 1e-10 * np.abs(G).max()


def test_cycle_contracts():
    M, R = _model(10, "fp64")
    M.linear_solve(-R, rtol=1e-8, rebuild=True, precision="fp64")
    A0 = M.amg_dense(0, 0)
    e = np.random.default_rng(1).standard_normal(A0.shape[0])
    norms = []
    for _ in range(16):
        e = e - M.amg_apply(A0 @ e)
        norms.append(np.linalg.norm(A0 @ e))
    rho = (norms[-1] / norms[5]) ** (1.0 / 10)
    assert rho < 0.8, rho  # a broken cycle gives rho >= 1


@pytest.mark.parametrize("n,its_max", [(40, 30), (80, 45)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cg_iterations_bounded(precision, n, its_max):
    """The hierarchy stops at the first level with at most 1,500 unknowns and
    inverts it densely.  40^3: levels 0-1 and the dense solve on level 2 (570
    unknowns).  80^3 (1.6 M DOF): levels 0-2 and the dense solve on level 3, so
    the W branch on level 2 runs.  CG reaches 1e-6 (FP64) / 1e-5 (FP32, near its
    rounding floor on this operator) in a bounded number of iterations."""
    M, R = _model(n, precision)
    x, its = M.linear_solve(-R, rtol=1e-6 if precision == "fp64" else 1e-5, rebuild=True, precision=precision)
    assert its <= its_max, its
    assert np.all(np.isfinite(x))
    if n == 80:
        with pytest.raises(P.PfemError):
            M.amg_dense(4, 0)      # levels 0..2 plus the dense level 3: no level 4
        assert M.amg_dense(3, 0).shape[0] <= 1500 < M.amg_dense(2, 0).shape[0]


@pytest.mark.parametrize("n,device_path", [(8, False), (12, True), (48, True)])
def test_coarse_dense_inverse(n, device_path):
    """The coarsest level's dense inverse: on the host with partial pivoting up to
    300 unknowns (8^3: level 1), on the device by blocked Gauss-Jordan above (12^3:
    level 1, a few hundred unknowns, not a multiple of the 64-column panel; 48^3:
    level 2, about 1,300 unknowns); either way inverse times operator is the
    identity to rounding."""
    M, R = _model(n, "fp64")
    M.linear_solve(-R, rtol=1e-8, rebuild=True, precision="fp64")
    for L in range(1, 6):        # only the coarsest level answers what = 2
        try:
            Ai = M.amg_dense(L, 2)
            break
        except P.PfemError:
            continue
    Ac = M.amg_dense(L, 0)
    assert (Ac.shape[0] > 300) == device_path, Ac.shape
    # rows of rigid modes absent from an aggregate are empty; both inverses give
    # them a unit diagonal, so compare on the others
    nz = np.abs(Ac).sum(axis=1) > 0
    E = (Ai @ Ac)[np.ix_(nz, nz)] - np.eye(int(nz.sum()))
    assert np.abs(E).max() < 1e-8, np.abs(E).max()


def test_cycle_timed_in_a_graph():
    """pfem_profile what = 4 captures one cycle of the resident FP32 hierarchy into a
    CUDA graph and replays it: it takes a positive time and leaves the hierarchy as
    it was (a cycle applied afterwards gives the same result, bit for bit)."""
    M, R = _model(10, "mixed")
    M.linear_solve(-R, rtol=1e-4, rebuild=True, precision="mixed")
    r = np.ones(M.ndof)
    z = M.amg_apply(r)
    ms = M.profile(4, reps=3)
    assert ms > 0
    assert np.array_equal(M.amg_apply(r), z)


def test_sixteen_bit_column_offsets():
    """A node-ordered box mesh's block columns lie within 16-bit offsets of their row,
    so the level-0 SpMV reads 2-byte indices; its product equals the tangent's
    (the level-0 operator the cycle and CG use) applied on the host."""
    M, R = _model(10, "fp64")
    assert M.tangent_index_bytes() == 2
    M.linear_solve(-R, rtol=1e-8, rebuild=True, precision="fp64")
    A0 = M.amg_dense(0, 0)
    x, its = M.linear_solve(-R, rtol=1e-8, rebuild=False, precision="fp64")
    assert np.linalg.norm(A0 @ x + R) <= 1e-7 * np.linalg.norm(R)
