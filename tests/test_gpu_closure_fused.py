"""The closure network evaluated inside the flux pass (cruna_set_closure_fused, the default on the fused
RHS path) against the same closure run as separate launches (features, tensor-core network, stress
divergence through the forcing hook).  Both read the same velocity gradients, rho and T, round them
to the same BF16 operands and run the same tensor-core products, so the model stresses agree; the
fused pass differentiates tau - tau(model) in one sum, which differs from the separate divergence by
rounding only: 1e-9 of the closure term plus 1e-12 of the RHS.  Mass and energy equations carry no
closure term and agree to 1e-12."""
import numpy as np
import pytest

from oracle import mlp_closure as M
from public_b200 import cases
from public_b200.cruna import Cruna, Settings

pytestmark = pytest.mark.gpu


def run_both(s, q, normalised, precision="fp64", steps=False):
    from public_b200.closure import ClosureMLP
    st = Settings.from_dict(s)
    st.precision = precision
    out = {}
    with Cruna(st) as c, ClosureMLP(0, seed=4) as mlp:
        assert c.rhs_path == "fused"
        mlp.params = M.init_params(11)
        mlp.set_scaling(np.zeros(12), np.ones(12), np.full(6, 1e-2 if normalised else 2e-3))
        c.set_closure_normalisation(normalised)
        plain = c.time_stepper_direct(q) if steps else c.rhs_direct(q)
        c.set_closure(mlp, 0.3)
        for fused in (True, False):
            c.set_closure_fused(fused)
            n0 = c.launches
            r = c.time_stepper_direct(q) if steps else c.rhs_direct(q)
            out[fused] = (r, c.launches - n0)
        c.set_closure(None)
    return plain, out


@pytest.mark.parametrize("normalised", [False, True])
@pytest.mark.parametrize("grid", [16, (40, 36, 20)], ids=["iso16", "40x36x20"])
def test_fused_closure_rhs_matches_separate_launches(normalised, grid):
    n = grid if isinstance(grid, tuple) else (grid,) * 3
    if isinstance(grid, tuple):
        q = cases.smooth_random_state(n, seed=5, p0=1.0, rho0=1.0, amp=0.05)
        s = dict(n=n, diff=("o8_e_c_p",) * 3, x1=(1.0, 1.1, 0.9), R=1.0, W=1.0, T0=1.0, mu0=0.01, dt=1e-3)
    else:
        s, q = cases.isotropic_turbulence(n=grid, seed=3)
    plain, out = run_both(s, q, normalised)
    (rf, nf), (rs, ns) = out[True], out[False]
    term = rs - plain
    for v in (0, 4):
        assert np.max(np.abs(rf[..., v] - rs[..., v])) <= 1e-12 * np.max(np.abs(rs[..., v])) + 1e-14, v
    tol = 1e-9 * np.max(np.abs(term[..., 1:4])) + 1e-12 * np.max(np.abs(rs[..., 1:4]))
    assert np.max(np.abs(rf[..., 1:4] - rs[..., 1:4])) <= tol
    assert np.max(np.abs(term[..., 1:4])) > 0.0
    assert nf < ns          # the separate closure adds launches the fused pass does not need


def test_fused_closure_step_and_fp32_stencils():
    s, q = cases.isotropic_turbulence(n=16, seed=6)
    plain, out = run_both(s, q, False, steps=True)
    term = out[False][0] - plain
    assert np.max(np.abs(out[True][0] - out[False][0])) <= 1e-9 * np.max(np.abs(term)) + 1e-12 * np.max(np.abs(plain))
    plain32, out32 = run_both(s, q, False, precision="fp32")
    term32 = out32[False][0] - plain32
    # FP32 stencils: the fused pass forms the features from FP32 gradients, the separate path from the
    # FP64 generic ones; the model stresses then differ at the FP32 rounding of the inputs
    assert np.max(np.abs(out32[True][0] - out32[False][0])) <= 1e-3 * np.max(np.abs(term32)) + 1e-6 * np.max(np.abs(plain32))
