"""Enstrophy: the volume diagnostics (kinetic energy, enstrophy) and the final-time enstrophy
objective's gradients (continuous and exact discrete adjoint) through the C ABI against the oracle
(oracle/cruna_oracle.py: objective_enstrophy, gradient_store_all; oracle/discrete_adjoint.py:
gradient_discrete).  Tolerances: diagnostics 1e-12 relative; J 1e-12 relative; gradients 1e-10
relative L2 per variable (measured against max(its norm, 1e-3 of the state's norm))."""
import numpy as np
import pytest
import torch

from oracle import cruna_oracle as O
from oracle import discrete_adjoint as DA
from public_b200 import cases
from public_b200.cruna import Cruna, Settings

pytestmark = pytest.mark.gpu
CFG_FIELDS = {f.name for f in O.dataclasses.fields(O.Config)}


def ocfg(s):
    return O.Config(**{k: v for k, v in s.items() if k in CFG_FIELDS})


def cot_err(a, b):
    scale = np.linalg.norm(b.ravel())
    return max(float(np.linalg.norm((a[..., v] - b[..., v]).ravel()) /
                     max(np.linalg.norm(b[..., v].ravel()), 1e-3 * scale)) for v in range(b.shape[-1]))


@pytest.mark.parametrize("case", ["tgv", "tgv_compact", "mixing", "vortex"])
def test_diagnostics_match_oracle(case):
    if case == "mixing":
        s, q = cases.mixing_layer(n=(24, 22, 12))
    elif case == "vortex":
        s, q = cases.isentropic_vortex(n=32)
    else:
        s, q = cases.taylor_green(n=16, seed=2)
        if case == "tgv_compact":
            s["diff"] = ("o6_i_c_p",) * 3
    cfg = ocfg(s)
    ke_ref = O.objective_kinetic_energy(cfg, q)[0]
    z_ref = O.objective_enstrophy(cfg, q)[0]
    with Cruna(Settings.from_dict(s), qref=q) as c:
        ke, z = c.diagnostics(q)
        qt = torch.from_numpy(np.ascontiguousarray(q.ravel(order="F"))).cuda()
        assert c.diagnostics_dev(qt.data_ptr()) == (ke, z)
    assert abs(ke - ke_ref) < 1e-12 * abs(ke_ref)
    assert abs(z - z_ref) < 1e-12 * abs(z_ref), (z, z_ref)


@pytest.mark.parametrize("mode,scheme", [(0, "o8_e_c_p"), (1, "o8_e_c_p"), (0, "o6_i_c_p"), (1, "o6_i_c_p")])
def test_enstrophy_gradient_matches_oracle(mode, scheme):
    s, q = cases.taylor_green(n=12, seed=0)
    s["mu0"] = 0.02
    s["diff"] = (scheme,) * 3
    S = O.Solver(ocfg(s), force=np.zeros_like(q))
    obj = {"kind": "enstrophy"}
    if mode == 0:
        J_ref, gf_ref, gq_ref = O.gradient_store_all(S, q, 4, obj)
    else:
        J_ref, gf_ref, gq_ref = DA.gradient_discrete(S, q, 4, obj)
    with Cruna(Settings.from_dict(s), force=np.zeros_like(q)) as c:
        c.set_adjoint_mode(mode)
        J, gf, gq, steps = c.gradient(q, 4, 2, c.objective("enstrophy"))
        Jv = c.objective_value(q, 4, c.objective("enstrophy"))
    assert abs(J - J_ref) < 1e-12 * abs(J_ref) and abs(Jv - J_ref) < 1e-12 * abs(J_ref)
    assert cot_err(gq, gq_ref) < 1e-10, cot_err(gq, gq_ref)
    assert cot_err(gf, gf_ref) < 1e-10, cot_err(gf, gf_ref)


def test_enstrophy_gradient_fp32_stencils_close_to_fp64():
    s, q = cases.taylor_green(n=16, seed=0)
    s["mu0"] = 0.02
    out = {}
    for prec in ("fp64", "fp32"):
        with Cruna(Settings.from_dict(dict(s, precision=prec)), force=np.zeros_like(q)) as c:
            out[prec] = c.gradient(q, 6, 3, c.objective("enstrophy"))
    (J64, gf64, gq64, _), (J32, gf32, gq32, _) = out["fp64"], out["fp32"]
    assert abs(J32 - J64) < 1e-6 * abs(J64)
    assert np.linalg.norm(gq32 - gq64) < 1e-5 * np.linalg.norm(gq64)


@pytest.mark.parametrize("mode", [0, 1])
def test_host_snapshots_and_aliased_gradient_match_hbm(mode):
    """Snapshots in pinned host memory give the same bits as HBM snapshots, and cruna_gradient_dev
    may write dJ/dq0 over q0 itself."""
    s, q = cases.taylor_green(n=16, seed=1)
    s["mu0"] = 0.02
    out = {}
    for host in (False, True):
        with Cruna(Settings.from_dict(s), force=np.zeros_like(q)) as c:
            c.set_adjoint_mode(mode)
            c.set_snapshot_memory(host)
            out[host] = c.gradient(q, 7, 3, c.objective("enstrophy"))
            qt = torch.from_numpy(np.ascontiguousarray(q.ravel(order="F"))).cuda()
            torch.cuda.synchronize()
            J, steps = c.gradient_dev(qt.data_ptr(), 7, 3, c.objective("enstrophy"), None, qt.data_ptr())
            c.sync()
            assert J == out[host][0] and steps == out[host][3]
            assert np.array_equal(qt.cpu().numpy().reshape(q.shape, order="F"), out[host][2])
            if host:  # the pinned slots are reused by the second call above, then given back
                c.set_snapshot_memory(False)
                assert np.array_equal(c.gradient(q, 7, 3, c.objective("enstrophy"))[2], out[host][2])
    (J0, gf0, gq0, n0), (J1, gf1, gq1, n1) = out[False], out[True]
    assert J0 == J1 and n0 == n1
    assert np.array_equal(gq0, gq1) and np.array_equal(gf0, gf1)
