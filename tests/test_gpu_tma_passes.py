"""The TMA-fed FP64 fused adjoint pass (cruna_set_tma_passes) against the per-thread-load kernel and
against the oracle: RHS evaluations and RK steps on periodic and open grids, tiles wider than the grid, grids whose
sizes are not multiples of the 32 x 4 tile, and the benchmark's 256^3 grid.  Both kernels evaluate the
same sums; they agree to rounding (1e-13 relative to the field maximum)."""
import numpy as np
import pytest

from oracle import cruna_oracle as O
from public_b200 import cases
from public_b200.cruna import Cruna, Settings

pytestmark = pytest.mark.gpu
CFG_FIELDS = {f.name for f in O.dataclasses.fields(O.Config)}


def rel_max(a, b):
    return max(float(np.max(np.abs(a[..., v] - b[..., v])) / max(np.max(np.abs(b[..., v])), 1e-300))
               for v in range(b.shape[-1]))


GRIDS = [
    ("tgv16", dict(n=16)),
    ("tgv_40x36x20", dict(n=(40, 36, 20))),
    ("tgv_64x20x12", dict(n=(64, 20, 12))),
    ("open_y", dict(n=(48, 22, 24), diff=("o8_e_c_p", "o4_e_c_o", "o8_e_c_p"))),
    ("o4_periodic", dict(n=(34, 12, 14), diff=("o4_e_c_p", "o4_e_c_p", "o4_e_c_p"))),
]


def make(name, spec):
    n = spec["n"] if isinstance(spec["n"], tuple) else (spec["n"],) * 3
    q = cases.smooth_random_state(n, seed=hash(name) % 1000, p0=1.0, rho0=1.0, amp=0.05)
    s = dict(n=n, diff=spec.get("diff", ("o8_e_c_p",) * 3), x1=(1.0, 1.1, 0.9), R=1.0, W=1.0, T0=1.0,
             mu0=0.01, dt=1e-3)
    qs = cases.smooth_random_state(n, seed=7, p0=0.0, rho0=0.0, amp=1.0)
    return s, q, qs


@pytest.mark.parametrize("name,spec", GRIDS, ids=[g[0] for g in GRIDS])
def test_tma_adjoint_pass_matches_register_pass_and_oracle(name, spec):
    s, q, qs = make(name, spec)
    out = {}
    for tma in (True, False):
        with Cruna(Settings.from_dict(s)) as c:
            assert c.rhs_path == "fused"
            c.tma_passes(tma)
            out[tma] = (c.rhs_adjoint(qs, q), c.time_stepper_adjoint(qs, q))
    assert rel_max(out[True][0], out[False][0]) < 1e-13
    assert rel_max(out[True][1], out[False][1]) < 1e-13
    S = O.Solver(O.Config(**{k: v for k, v in s.items() if k in CFG_FIELDS}))
    ref = S.rhs_adjoint(qs, q, np.zeros_like(q))
    assert rel_max(out[True][0], ref) < 1e-12


@pytest.mark.parametrize("name,spec", GRIDS, ids=[g[0] for g in GRIDS])
def test_tma_direct_passes_match_register_passes_and_oracle(name, spec):
    s, q, _ = make(name, spec)
    out = {}
    for tma in (True, False):
        with Cruna(Settings.from_dict(s)) as c:
            c.tma_passes(tma)
            out[tma] = (c.rhs_direct(q), c.time_stepper_direct(q))
    assert rel_max(out[True][0], out[False][0]) < 1e-13
    assert rel_max(out[True][1], out[False][1]) < 1e-13
    S = O.Solver(O.Config(**{k: v for k, v in s.items() if k in CFG_FIELDS}))
    ref = S.rhs_direct(q)
    assert rel_max(out[True][0], ref) < 1e-12


def test_tma_passes_at_256_cubed():
    """The benchmark's grid: one adjoint and one direct RK step with and without TMA."""
    import torch

    s, q0 = cases.taylor_green(n=256, seed=0)
    qs0 = cases.smooth_random_state((256,) * 3, seed=5, p0=0.0, rho0=0.0, amp=1e-3)
    dev = torch.device("cuda", 0)
    res = {}
    for tma in (True, False):
        q = torch.from_numpy(np.ascontiguousarray(q0.ravel(order="F"))).to(dev)
        qs = torch.from_numpy(np.ascontiguousarray(qs0.ravel(order="F"))).to(dev)
        q1 = torch.empty_like(q)
        qs1 = torch.empty_like(q)
        torch.cuda.synchronize()
        with Cruna(Settings.from_dict(s)) as c:
            c.tma_passes(tma)
            c.step_direct_dev(q.data_ptr(), q1.data_ptr())
            c.step_adjoint_dev(qs.data_ptr(), q1.data_ptr(), None, qs1.data_ptr())
            c.sync()
        res[tma] = (q1.cpu().numpy().reshape(q0.shape, order="F"), qs1.cpu().numpy().reshape(q0.shape, order="F"))
    assert rel_max(res[True][0], res[False][0]) < 1e-13
    assert rel_max(res[True][1], res[False][1]) < 1e-13
