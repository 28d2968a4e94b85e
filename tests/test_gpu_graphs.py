"""Step graphs: the run loops and the gradient replay repeating steps from CUDA graphs.  With graphs on
and off the same calls give bit-identical states, objectives and gradients, the same launch count, and
graphs are actually captured and replayed (two filter patterns: the filters run every second step)."""
import numpy as np
import pytest
import torch

from public_b200 import cases
from public_b200.cruna import Cruna, Settings

pytestmark = pytest.mark.gpu


def tgv_settings(n=24, precision="fp64"):
    s, q = cases.taylor_green(n=n, seed=1)
    s.update(mu0=0.01, filt=("o10_e_c_p",) * 3, di_freq=(2, 2, 2), ai_freq=(2, 2, 2), precision=precision)
    return s, q


def run_both(s, q, fn):
    out = []
    for on in (False, True):
        with Cruna(Settings.from_dict(s), qref=q) as c:
            c.set_graphs(on)
            l0 = c.launches
            r = fn(c)
            out.append((r, c.launches - l0, c.graph_stats()))
    return out


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_direct_run_replays_bit_identical(precision):
    s, q = tgv_settings(precision=precision)
    (a, la, sa), (b, lb, sb) = run_both(s, q, lambda c: c.calc_direct(q, 12))
    assert np.array_equal(a, b)
    assert la == lb
    assert sa == (0, 0)
    assert sb[0] == 2 and sb[1] == 8          # two filter patterns: 2 eager + 2 recorded + 8 replays


def test_adjoint_run_replays_bit_identical():
    s, q = tgv_settings()
    with Cruna(Settings.from_dict(s), qref=q) as c:
        _, Q = c.calc_direct(q, 10, store=True)
    rng = np.random.default_rng(4)
    qs0 = np.asfortranarray(rng.standard_normal(q.shape))
    (a, la, _), (b, lb, sb) = run_both(s, q, lambda c: c.calc_adjoint(qs0, Q))
    assert np.array_equal(a, b)
    assert la == lb
    assert sb[0] == 2 and sb[1] == 6          # host trajectories: one staging buffer, so keys repeat


def test_mixing_layer_with_boundaries_bit_identical():
    s, q = cases.mixing_layer(n=(32, 30, 16))
    (a, la, _), (b, lb, sb) = run_both(s, q, lambda c: c.calc_direct(q, 8))
    assert np.array_equal(a, b)
    assert la == lb and sb[1] > 0


@pytest.mark.parametrize("mode", [0, 1])
def test_gradient_bit_identical(mode):
    s, q = tgv_settings()
    s["mu0"] = 0.02

    def grad(c):
        c.set_adjoint_mode(mode)
        obj = c.objective("plane_p2", normal=1, index=5, p_inf=float(q[..., 4].mean()))
        return c.gradient(q, 9, 4, obj)

    (a, la, _), (b, lb, sb) = run_both(s, q, grad)
    assert a[0] == b[0] and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]) and a[3] == b[3]
    assert la == lb
    if mode == 0:
        assert sb[1] > 0


def test_profiling_runs_eagerly():
    s, q = tgv_settings()
    with Cruna(Settings.from_dict(s), qref=q) as c:
        c.profile(True)
        c.calc_direct(q, 6)
        assert c.graph_stats() == (0, 0)
        rep = c.profile_report()
        assert sum(v[0] for v in rep.values()) > 0


def test_device_loop_with_torch_buffers():
    s, q = tgv_settings()
    dev = torch.device("cuda", 0)
    qt = torch.from_numpy(np.ascontiguousarray(q.ravel(order="F"))).to(dev)
    with Cruna(Settings.from_dict(s), qref=q) as c:
        ref = c.calc_direct(q, 20)
        c.run_direct_dev(qt.data_ptr(), 0, 20)
        c.sync()
        got = qt.cpu().numpy().reshape(q.shape, order="F")
        cap, rep = c.graph_stats()
    assert np.array_equal(got, ref)
    assert cap == 4 and rep == 32             # two calls, each: 2 eager, 2 recorded, 16 replays


def test_restart_from_an_intermediate_step_is_bit_identical():
    """cruna_run_direct from nt0 continues a run exactly (the filter pattern follows the global step
    count), like a restart from (subset, step) in the reference's cruna_hpc.f90:109-148."""
    s, q = tgv_settings()
    with Cruna(Settings.from_dict(s), qref=q) as c:
        whole = c.calc_direct(q, 11)
        part = c.calc_direct(q, 4)
        rest = c.calc_direct(part, 7, nt0=4)
    assert np.array_equal(whole, rest)
