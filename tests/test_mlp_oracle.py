"""CPU checks of the closure MLP reference (oracle/mlp_closure.py): the exact gradient against central
differences, BF16 rounding, and the BF16 gradient's closeness to the exact one."""
import numpy as np

from oracle import mlp_closure as M


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-20], dtype=np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 4 * 2 ** -8    # ties to even
    assert r[3] == -2.5 and abs(r[4] - 3.0e-20) < 3.0e-20 * 2 ** -8


def test_exact_gradient_matches_central_differences():
    rng = np.random.default_rng(0)
    X = rng.standard_normal((64, 12))
    Y = rng.standard_normal((64, 6))
    mu, sd, osd = X.mean(0), X.std(0), np.abs(Y).mean(0) + 0.5
    p = M.init_params(1)
    L, g = M.grad_exact(p, X, Y, mu, sd, osd)
    for k in rng.choice(M.NPARAMS, 40, replace=False):
        e = np.zeros_like(p)
        e[k] = 1e-6
        fd = (M.loss_exact(p + e, X, Y, mu, sd, osd) - M.loss_exact(p - e, X, Y, mu, sd, osd)) / 2e-6
        assert abs(fd - g[k]) < 1e-6 * max(1.0, abs(fd)) + 1e-8, (k, fd, g[k])


def test_bf16_gradient_close_to_exact():
    rng = np.random.default_rng(1)
    X = rng.standard_normal((256, 12))
    Y = rng.standard_normal((256, 6))
    p = M.init_params(2)
    args = (X, Y, X.mean(0), X.std(0), np.ones(6))
    _, ge = M.grad_exact(p, *args)
    _, gb = M.grad_bf16(p, *args)
    assert np.linalg.norm(gb - ge) < 3e-2 * np.linalg.norm(ge)
    assert M.NPARAMS == 5382
