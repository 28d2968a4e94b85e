"""Zonal characteristic boundary conditions (types 202, 203, 205, 206 with the diagonal, orthogonal and
hedgehog normal-vector fields, nonreflecting.f90:141-233, :345-449, :558-661) against the oracle:
the boundary calls themselves, the RHS and a few steps of the direct and adjoint loops (type 203
applied inside and/or outside the RHS)."""
import numpy as np
import pytest

from oracle import cruna_oracle as O
from public_b200 import cases
from public_b200.cruna import Cruna, Settings

pytestmark = pytest.mark.gpu

CFG_FIELDS = {f.name for f in O.dataclasses.fields(O.Config)}


def ocfg(s):
    return O.Config(**{k: v for k, v in s.items() if k in CFG_FIELDS})


def rel_l2_vars(a, b):
    scale = np.linalg.norm(b.ravel())
    return [float(np.linalg.norm((a[..., v] - b[..., v]).ravel()) / max(np.linalg.norm(b[..., v].ravel()), 1e-3 * scale))
            for v in range(b.shape[-1])]


ROWS = {
    "202": [[202, 1, 10, 1, 1, 1, 12, 0, 0, 0], [202, 10, 10, 1, 11, 1, 12, 0, 0, 0]],
    "203": [[203, 1, 10, 1, 11, 1, 12, 0, 0, 0]],
    "203in": [[203, 1, 10, 1, 11, 1, 12, 1, 0, 0]],
    "203out": [[203, 1, 10, 1, 11, 1, 12, -1, 0, 0]],
    "205": [[205, 1, 10, 11, 11, 1, 12, 0, 0, 0]],
    "206": [[206, 1, 10, 1, 11, 1, 12, 0, 0, 0]],
}


def case(kind, kv, scheme="o4_e_c_o"):
    n = (10, 11, 12)
    q = cases.smooth_random_state(n, seed=7, p0=1.0, rho0=1.0, amp=0.05)
    qref = cases.smooth_random_state(n, seed=8, p0=1.0, rho0=1.0, amp=0.05)
    s = dict(n=n, diff=(scheme,) * 3, x1=(1.0, 1.2, 1.4), dt=1e-3, bc=np.array(ROWS[kind], dtype=float),
             sponge_length=(0.2, 0.3, 0.25), sponge_amplitude=0.8, R=1.0, W=1.0, T0=1.0, mu0=0.01, kvector=kv)
    return s, q, qref


@pytest.mark.parametrize("kv", ["diagonal", "orthogonal", "hedgehog"])
@pytest.mark.parametrize("kind", sorted(ROWS))
def test_zonal_boundary_calls_match_oracle(kind, kv):
    s, q, qref = case(kind, kv)
    S = O.Solver(ocfg(s), qref=qref)
    rhs = cases.smooth_random_state(s["n"], seed=9, p0=0.3, rho0=0.2, amp=0.5)
    qs = cases.smooth_random_state(s["n"], seed=10, p0=0.1, rho0=0.3, amp=0.5)
    with Cruna(Settings.from_dict(s), qref=qref) as c:
        pairs = [
            (c.set_boundary_condition_q(q, False), S.set_boundary_condition_q(q, False)),
            (c.set_boundary_condition_q(q, True), S.set_boundary_condition_q(q, True)),
            (c.set_boundary_condition_qs(qs, q, False), S.set_boundary_condition_qs(qs, q, False)),
            (c.set_boundary_condition_qs(qs, q, True), S.set_boundary_condition_qs(qs, q, True)),
            (c.set_boundary_condition_rhs(rhs, q), S.set_boundary_condition_rhs(rhs, q)),
        ]
    for i, (a, b) in enumerate(pairs):
        assert max(rel_l2_vars(a, b)) < 1e-12, (kind, kv, i, rel_l2_vars(a, b))


@pytest.mark.parametrize("kind", ["203", "203in", "203out", "206"])
def test_zonal_loops_match_oracle(kind):
    s, q, qref = case(kind, "diagonal")
    s["dt"] = 2e-3
    S = O.Solver(ocfg(s), qref=qref)
    ref, Q = S.calc_direct(q, 3, store=True)
    qs0 = cases.smooth_random_state(s["n"], seed=11, p0=0.0, rho0=0.0, amp=0.1)
    aref, _ = S.calc_adjoint(qs0, Q)
    with Cruna(Settings.from_dict(s), qref=qref) as c:
        got = c.calc_direct(q, 3)
        adj = c.calc_adjoint(qs0, Q)
    assert max(rel_l2_vars(got, ref)) < 1e-12, rel_l2_vars(got, ref)
    assert max(rel_l2_vars(adj, aref)) < 1e-12, rel_l2_vars(adj, aref)
