"""Tensor-core predictor MLP vs its CPU oracle, and the learned predictor in Newton."""
import numpy as np
import pytest

import plasticity_b200 as P
from plasticity_b200 import workloads as W
from oracle import mlp_ref as R

pytestmark = pytest.mark.gpu


def _model(n=4):
    w = W.config0(n=n, nsteps=4)
    M = P.Model(w.mesh, P.J2Material(**w.material))
    w.apply(M)
    return M, w


def _rand_params(seed):
    rng = np.random.default_rng(seed)
    W1 = np.zeros((128, 16)); W1[:, :12] = rng.normal(0, 0.4, (128, 12))
    W2 = rng.normal(0, 0.12, (128, 128))
    W3 = np.zeros((16, 128)); W3[:3] = rng.normal(0, 0.12, (3, 128))
    b1 = rng.normal(0, 0.1, 128); b2 = rng.normal(0, 0.1, 128); b3 = np.zeros(16); b3[:3] = rng.normal(0, 0.1, 3)
    return R.join(W1, b1, W2, b2, W3, b3).astype(np.float32)


@pytest.mark.parametrize("n", [1, 127, 128, 1000])
def test_forward_matches_oracle(n):
    M, _ = _model()
    p = _rand_params(3)
    M.mlp_params(p)
    rng = np.random.default_rng(n)
    F = rng.normal(0, 1, (n, 12)).astype(np.float32)
    y = M.mlp_forward(F)
    yr, _ = R.forward(p, F.astype(np.float64), bf=True)
    assert np.linalg.norm(y - yr) / np.linalg.norm(yr) < 2e-3


def test_loss_and_gradient_match_oracle():
    M, _ = _model()
    p = _rand_params(4)
    M.mlp_params(p)
    rng = np.random.default_rng(9)
    n = 3000
    F = rng.normal(0, 1, (n, 12)).astype(np.float32)
    T = rng.normal(0, 1, (n, 3)).astype(np.float32)
    loss, g = M.mlp_loss_grad(F, T)
    lr, gr = R.loss_grad(p, F.astype(np.float64), T.astype(np.float64), bf=True)
    assert abs(loss - lr) <= 1e-3 * lr
    o = 0
    for name, size in [("W1", 128 * 16), ("b1", 128), ("W2", 128 * 128), ("b2", 128), ("W3", 16 * 128), ("b3", 16)]:
        a, b = g[o:o + size], gr[o:o + size]
        assert np.linalg.norm(a - b) <= 5e-3 * np.linalg.norm(b) + 1e-9, name
        o += size


def test_training_reduces_loss():
    M, _ = _model()
    M.mlp_init(1)
    rng = np.random.default_rng(2)
    F = rng.normal(0, 1, (20000, 12)).astype(np.float32)
    T = np.stack([np.tanh(F[:, 3]), 0.5 * F[:, 4] * F[:, 5], np.sin(F[:, 0])], 1).astype(np.float32)
    l0, _ = M.mlp_loss_grad(F, T)
    # plain gradient steps through the oracle-checked gradient
    p = M.mlp_params()
    for _ in range(60):
        _, g = M.mlp_loss_grad(F, T)
        p = p - 0.05 * g
        M.mlp_params(p)
    l1, _ = M.mlp_loss_grad(F, T)
    assert l1 < 0.6 * l0


def test_learned_predictor_in_newton_keeps_the_solution():
    w = W.config4_path(n=6, nsteps=8, seed=7)
    M = P.Model(w.mesh, P.J2Material(**w.material))
    # record a few solver-generated paths and train briefly on the GPU
    M.mlp_init(0)
    M.mlp_record("start", 20 * 8 * M.nn)
    for s in range(3):
        wi = W.config4_path(n=6, nsteps=8, seed=100 + s)
        wi.apply(M)
        M.reset()
        for k in range(1, 9):
            M.newton(k / 8, tol=1e-10, predictor="extrapolate", line_search=True, precision="fp64", lin_rtol=1e-10)
    assert M.mlp_record("size") == 3 * 6 * M.nn
    M.mlp_record("stop")
    losses = M.mlp_train(200, batch=4096, lr=1e-3)
    assert np.isfinite(losses).all() and losses[-20:].mean() < losses[:20].mean()
    sols = {}
    for pred in ("extrapolate", "learned"):
        w.apply(M)
        M.reset()
        for k in range(1, 9):
            M.newton(k / 8, tol=1e-11, predictor=pred, line_search=True, precision="fp64", lin_rtol=1e-11)
        sols[pred] = M.U
    rel = np.linalg.norm(sols["learned"] - sols["extrapolate"]) / np.linalg.norm(sols["extrapolate"])
    assert rel < 1e-8


def test_trained_predictor_gains_over_extrapolation():
    """The committed network (trained on solver-generated 32^3 paths) against the
    extrapolation predictor on a held-out path: the guess it hands to Newton is
    several times closer to the converged increment, its FP64 residual is lower,
    Newton and CG need no more iterations, and the converged solution is the same."""
    from plasticity_b200 import predictor as PR
    assert PR.weights_available(), "trained predictor weights are missing"
    w = W.config4_path(n=32, nsteps=20, seed=9001)
    M = P.Model(w.mesh, P.J2Material(**w.material))
    PR.load_into(M)
    rows = PR.guess_errors(M, w)
    err_ex = np.median([r["err_extrap"] for r in rows])
    err_ml = np.median([r["err_chosen"] for r in rows])
    r_ex = np.median([r["r_extrap"] for r in rows])
    r_ml = np.median([r["r_learned"] for r in rows])
    assert sum(r["used"] for r in rows) >= 0.8 * len(rows)
    assert err_ml < 0.25 * err_ex, (err_ml, err_ex)
    assert r_ml < 0.25 * r_ex, (r_ml, r_ex)
    sols, its = {}, {}
    for pred in ("extrapolate", "learned"):
        st = PR.run_path(M, w, pred, tol=1e-10)
        assert st["converged"]
        sols[pred], its[pred] = M.U, (sum(st["newton"]), sum(st["krylov"]))
    assert its["learned"][0] <= its["extrapolate"][0], its
    assert np.linalg.norm(sols["learned"] - sols["extrapolate"]) <= 1e-8 * np.linalg.norm(sols["extrapolate"])
