"""CPU checks of the predictor-MLP oracle (the checker of the tensor-core kernels)."""
import numpy as np

from oracle import mlp_ref as R


def _rand_params(seed):
    rng = np.random.default_rng(seed)
    W1 = np.zeros((128, 16)); W1[:, :12] = rng.normal(0, 0.5, (128, 12))
    W2 = rng.normal(0, 0.1, (128, 128))
    W3 = np.zeros((16, 128)); W3[:3] = rng.normal(0, 0.1, (3, 128))
    b1 = rng.normal(0, 0.1, 128); b2 = rng.normal(0, 0.1, 128); b3 = np.zeros(16); b3[:3] = rng.normal(0, 0.1, 3)
    return R.join(W1, b1, W2, b2, W3, b3)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = _rand_params(2)
    F = rng.normal(0, 1, (40, 12)); T = rng.normal(0, 1, (40, 3))
    _, g = R.loss_grad(p, F, T, bf=False)
    idx = np.concatenate([rng.choice(128 * 12, 8), 128 * 16 + rng.choice(128, 4),
                          128 * 16 + 128 + rng.choice(128 * 128, 8), R.NPARAMS - 16 - 128 * 16 + rng.choice(3 * 128, 6),
                          R.NPARAMS - 16 + np.arange(3)])
    for i in idx:
        e = np.zeros_like(p); e[i] = 1e-6
        fd = (R.loss_grad(p + e, F, T, bf=False)[0] - R.loss_grad(p - e, F, T, bf=False)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-9, (i, fd, g[i])


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1 + 2 ** -8, 1 + 2 ** -9, 1 + 3 * 2 ** -9, -2.5, 3.14159], np.float32)
    y = R.bf16(x)
    assert y[0] == 1.0 and y[1] == 1.0          # 1 + 2^-8 is a tie -> even (1.0)
    assert y[2] == 1.0                       # tie -> even
    assert y[3] == 1 + 2 ** -7               # above half -> up
    assert y[4] == -2.5
    assert abs(y[5] - 3.140625) < 1e-12
