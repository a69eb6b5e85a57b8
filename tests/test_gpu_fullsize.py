"""Size-independent properties at the bench's full size: the 64^3 jittered /
lognormal compression cube (262,144 elements, 823,875 DOF), where the oracle is
too slow to compare entry by entry.

- Global balance of the internal force vector (Elements.jl:405-494): each
  element's nodal forces sum to zero (sum_a N_a = 1), and sum_a x_a (x) f_a =
  int F P^T dV = int (F Fbar^-1) tau dV is symmetric, also with F-bar
  (F Fbar^-1 = s^-1 I).
- The FP64 residual, stress and flags do not depend on the tangent's type (the
  mixed path changes only the tangent records).
- The mixed-precision Newton path reaches an FP64 truth run (1e-12 inner solves,
  Newton to 1e-12 from the previous converged U) within 1e-8 relative in
  displacement over the bench's 25 increments.
"""
import numpy as np
import pytest

import plasticity_b200 as P
from plasticity_b200 import workloads as W

pytestmark = pytest.mark.gpu
N = 64


@pytest.fixture(scope="module")
def w():
    return W.config2(n=N)


def _model(w):
    M = P.Model(w.mesh, P.J2Material(**w.material), sigy0_e=w.sigy0_e)
    w.apply(M)
    return M


def test_fullsize_force_and_moment_balance(w):
    M = _model(w)
    X = w.mesh.nodes
    rng = np.random.default_rng(5)
    U = (np.stack([0.004 * X[0], 0.002 * X[1], -0.02 * X[2]]).T.reshape(-1)
         + 4e-4 / N * rng.standard_normal(M.ndof))
    M.assemble(0.5 * U, commit=True)
    _, R, tau, fl = M.assemble(U, want_K=False)
    _, R32, tau32, fl32 = M.assemble(U, precision="mixed", want_K=False)
    assert fl.mean() > 0.3
    f = R.reshape(-1, 3)
    assert np.abs(f.sum(axis=0)).max() / np.abs(f).sum() < 1e-12
    x = X.T + U.reshape(-1, 3)
    S = x.T @ f
    assert np.abs(S - S.T).max() / np.abs(S).max() < 1e-10
    assert np.linalg.norm(R32 - R) / np.linalg.norm(R) < 1e-13
    assert np.abs(tau32 - tau).max() / np.abs(tau).max() < 1e-13
    assert np.array_equal(fl32, fl)


def test_fullsize_mixed_path_matches_fp64_truth(w):
    """Over the bench's whole window (increments 1-25 of 40): the mixed-precision
    path, with the learned predictor when trained weights are present and with
    extrapolation, against an FP64 truth run (previous-U predictor, inner solves
    to 1e-12, Newton to 1e-12 relative of the increment's first residual)."""
    from plasticity_b200 import predictor as PR
    last = 25
    truth = _model(w)
    arms = {"extrapolate": _model(w)}
    if PR.weights_available():
        arms["learned"] = _model(w)
        PR.load_into(arms["learned"])
    for s in range(1, last + 1):
        lam = s / w.nsteps
        truth.newton(lam, tol=1e-12, maxiter=40, precision="fp64", predictor="previous", line_search=True,
                     lin_rtol=1e-12)
        for pred, M in arms.items():
            M.newton(lam, tol=1e-10, maxiter=40, precision="mixed", predictor=pred, line_search=True)
    Ut = truth.U
    at = P.equivalent_plastic_strain(truth)
    for pred, M in arms.items():
        assert np.linalg.norm(M.U - Ut) / np.linalg.norm(Ut) < 1e-8, pred
        am = P.equivalent_plastic_strain(M)
        assert np.abs(am - at).max() / np.abs(at).max() < 1e-6, pred
