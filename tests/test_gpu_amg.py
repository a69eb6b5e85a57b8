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
    """The hierarchy stops at the first level with at most 3,600 unknowns and
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
        assert M.amg_dense(3, 0).shape[0] <= 3600 < M.amg_dense(2, 0).shape[0]
