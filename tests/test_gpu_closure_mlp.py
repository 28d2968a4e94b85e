"""GPU tests of the tensor-core closure MLP (cruna_mlp_*): forward, loss gradient and training against
the numpy reference (oracle/mlp_closure.py).

Tolerances: forward_bf16 / grad_bf16 restate the kernels' roundings (BF16 operands, FP32 accumulation),
so the kernels agree with them up to accumulation order and the odd BF16 rounding flip of an
activation: 5e-3 relative L2 for outputs, 2e-2 per parameter block for gradients.  Against the exact
FP64 network (the quantity BF16 approximates) the gradient agrees to 5e-2 and the loss to 1e-2."""
import numpy as np
import pytest

from oracle import mlp_closure as M

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-30))


def problem(n, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, 12)) * np.linspace(0.5, 3.0, 12) + np.linspace(-1, 1, 12)
    W = rng.standard_normal((12, 6)) * 0.3
    Y = np.tanh(X @ W) * np.array([2.0, 1.0, 0.5, 0.3, 0.2, 0.1]) + 0.05 * (X[:, :6] ** 2)
    in_mean, in_scale = X.mean(0), X.std(0)
    out_scale = Y.std(0)
    return X.astype(np.float32), Y.astype(np.float32), in_mean, in_scale, out_scale


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


@pytest.fixture
def mlp():
    from public_b200.closure import ClosureMLP
    with ClosureMLP(0, seed=1) as m:
        yield m


def test_forward_matches_reference(mlp):
    X, Y, mu, sd, osd = problem(1000)          # 1000: a partial last tile
    p = M.init_params(3)
    mlp.params = p
    mlp.set_scaling(mu, sd, osd)
    got = mlp.forward(dev(X)).cpu().numpy()
    ref = M.forward_bf16(np.float32(p), X, np.float32(mu), np.float32(sd), np.float32(osd))
    exact = M.forward_exact(p, X, mu, sd, osd)
    assert rel(got, ref) < 5e-3, rel(got, ref)
    assert rel(got, exact) < 3e-2, rel(got, exact)
    assert np.allclose(mlp.params, np.float32(p))


def test_gradient_matches_reference(mlp):
    X, Y, mu, sd, osd = problem(512, seed=1)
    p = M.init_params(4)
    mlp.params = p
    mlp.set_scaling(mu, sd, osd)
    loss, g = mlp.grad(dev(X), dev(Y))
    Lb, gb = M.grad_bf16(np.float32(p), X, Y, np.float32(mu), np.float32(sd), np.float32(osd))
    Le, ge = M.grad_exact(p, X, Y, mu, sd, osd)
    assert abs(loss - Lb) < 2e-3 * Lb, (loss, Lb)
    assert abs(loss - Le) < 1e-2 * Le, (loss, Le)
    o = 0
    for name, shp in M.SHAPES:
        k = int(np.prod(shp))
        assert rel(g[o:o + k], gb[o:o + k]) < 2e-2, (name, rel(g[o:o + k], gb[o:o + k]))
        assert rel(g[o:o + k], ge[o:o + k]) < 5e-2, (name, rel(g[o:o + k], ge[o:o + k]))
        o += k


def test_training_fits_a_smooth_map(mlp):
    X, Y, mu, sd, osd = problem(8192, seed=2)
    mlp.params = M.init_params(5)
    mlp.set_scaling(mu, sd, osd)
    Xd, Yd = dev(X), dev(Y)
    L0 = M.loss_exact(np.float64(mlp.params), X, Y, mu, sd, osd)
    hist = mlp.train(Xd, Yd, batch=1024, steps=400, lr=3e-3, seed=7)
    L1 = M.loss_exact(np.float64(mlp.params), X, Y, mu, sd, osd)
    assert np.all(np.isfinite(hist)) and len(hist) == 400
    assert L1 < 0.05 * L0, (L0, L1, hist[:3], hist[-3:])
    assert abs(hist[0] - L0) < 0.2 * L0
