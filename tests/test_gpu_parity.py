"""GPU parity of the CUDA library (through the C ABI) against the CPU oracle and the golden fixtures.

Tolerances (FP64 path): single derivative / filter applications agree to 1e-13 relative to the field
maximum (1e-12 for compact cores: their solves use reciprocal multiplies instead of LAPACK's divides);
RHS evaluations and short runs to 1e-12 relative L2 per conservative variable.
"""
import math
import os

import numpy as np
import pytest

from oracle import cruna_oracle as O
from public_b200 import cases
from public_b200.cruna import Cruna, CrunaError, Settings

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
CFG_FIELDS = {f.name for f in O.dataclasses.fields(O.Config)}


def ocfg(s: dict) -> O.Config:
    return O.Config(**{k: v for k, v in s.items() if k in CFG_FIELDS})


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rel_l2_vars(a, b):
    """relative L2 per variable; a variable that is identically zero in b is compared to the state norm"""
    out = []
    scale = np.linalg.norm(b.ravel())
    for v in range(b.shape[-1]):
        nb = np.linalg.norm(b[..., v].ravel())
        out.append(float(np.linalg.norm((a[..., v] - b[..., v]).ravel()) / (nb if nb > 0 else scale)))
    return out


COMPACT = {"o4_i_c_p_pade", "o4_i_c_o_pade", "o6_i_c_p", "o6_i_c_o"}


@pytest.fixture(scope="module")
def ops_gold():
    return np.load(os.path.join(GOLD, "operators.npz"))


@pytest.mark.parametrize("scheme", O.DIFF_SCHEMES)
def test_diff_matches_golden(ops_gold, scheme):
    q = ops_gold["q"]
    n = q.shape[:3]
    with Cruna(Settings(n=n, diff=(scheme,) * 3)) as c:
        dx = c.dx
        odx = O.Config(n=n, diff=(scheme,) * 3).dx()
        for d in range(3):
            if math.isfinite(odx[d]):
                assert dx[d] == odx[d]
            got = getattr(c, f"Dx{d + 1}")(q[..., 4], h=dx[d])
            ref = ops_gold[f"diff_{scheme}_{d + 1}"]
            tol = 1e-12 if scheme in COMPACT else 1e-13
            if scheme == "empty":
                assert np.all(got == 0.0)
            else:
                assert rel_max(got, ref) < tol, (scheme, d, rel_max(got, ref))


@pytest.mark.parametrize("scheme", ["o4_e_c_o", "o6_i_c_p", "o8_e_c_p"])
def test_diff_h_absent_and_many_fields(scheme):
    n = (12, 11, 10)
    q = cases.smooth_random_state(n, seed=2)
    cfg = O.Config(n=n, diff=(scheme,) * 3)
    with Cruna(Settings(n=n, diff=(scheme,) * 3)) as c:
        for d in range(3):
            got = getattr(c, f"Dx{d + 1}")(q)              # 5 fields, h absent -> dx = 1
            for v in range(5):
                ref = O.Dx(cfg, d, q[..., v], None)
                assert rel_max(got[..., v], ref) < 1e-12


@pytest.mark.parametrize("scheme", O.FILTER_SCHEMES)
def test_filter_matches_golden(ops_gold, scheme):
    q = ops_gold["q"]
    n = q.shape[:3]
    with Cruna(Settings(n=n, filt=(scheme,) * 3, alpha=0.3)) as c:
        for d in range(3):
            got = getattr(c, f"filter_i{d + 1}")(q[..., 4])
            ref = ops_gold[f"filter_{scheme}_{d + 1}"]
            assert rel_max(got, ref) < 1e-13, (scheme, d, rel_max(got, ref))


def _tgv(generic=False):
    g = np.load(os.path.join(GOLD, "tgv12.npz"))
    s, q0 = cases.taylor_green(n=12, seed=0)
    s["mu0"] = float(g["mu0"])
    c = Cruna(Settings.from_dict(s))
    if generic:
        c.force_generic(True)
    return g, s, q0, c


@pytest.mark.parametrize("generic", [True, False])
def test_rhs_direct_tgv(generic):
    g, s, q0, c = _tgv(generic)
    with c:
        r = c.rhs_direct(q0)
    assert max(rel_l2_vars(r, g["rhs"])) < 1e-12, rel_l2_vars(r, g["rhs"])


@pytest.mark.parametrize("generic", [True, False])
def test_calc_direct_tgv_5_steps(generic):
    g, s, q0, c = _tgv(generic)
    with c:
        q5 = c.calc_direct(q0, 5)
    assert max(rel_l2_vars(q5, g["q5"])) < 1e-12, rel_l2_vars(q5, g["q5"])


def test_heat_flux_dx_option():
    n = (10, 9, 8)
    q = cases.smooth_random_state(n, seed=4)
    for flag in (False, True):
        cfg = O.Config(n=n, diff=("o4_e_c_p",) * 3, mu0=0.02, R=1.0, W=1.0, T0=1.0, heat_flux_dx=flag)
        ref = O.Solver(cfg).rhs_direct(q)
        with Cruna(Settings(n=n, diff=("o4_e_c_p",) * 3, mu0=0.02, R=1.0, W=1.0, T0=1.0,
                            heat_flux_dx=flag)) as c:
            assert max(rel_l2_vars(c.rhs_direct(q), ref)) < 1e-12


def test_vortex_10_steps():
    g = np.load(os.path.join(GOLD, "vortex32.npz"))
    s, q0 = cases.isentropic_vortex(n=32)
    with Cruna(Settings.from_dict(s)) as c:
        q10 = c.calc_direct(q0, 10)
    assert max(rel_l2_vars(q10, g["q10"])) < 1e-12


def _pulse():
    g = np.load(os.path.join(GOLD, "pulse14.npz"))
    s, q0 = cases.gaussian_pulse(n=(14, 15, 16))
    return g, s, q0


def test_rhs_direct_pulse_characteristic_bc():
    g, s, q0 = _pulse()
    with Cruna(Settings.from_dict(s), qref=q0) as c:
        r = c.rhs_direct(q0)
    assert max(rel_l2_vars(r, g["rhs"])) < 1e-11, rel_l2_vars(r, g["rhs"])


def test_calc_direct_pulse_5_steps():
    g, s, q0 = _pulse()
    with Cruna(Settings.from_dict(s), qref=q0) as c:
        q5 = c.calc_direct(q0, 5)
    assert max(rel_l2_vars(q5, g["q5"])) < 1e-12, rel_l2_vars(q5, g["q5"])


def test_rhs_adjoint_pulse():
    g, s, q0 = _pulse()
    with Cruna(Settings.from_dict(s), qref=q0) as c:
        r = c.rhs_adjoint(g["qs0"], g["q5"], np.zeros_like(q0))
    assert max(rel_l2_vars(r, g["rhs_adj"])) < 1e-12, rel_l2_vars(r, g["rhs_adj"])


def test_adjoint_steps_match_oracle():
    g, s, q0 = _pulse()
    S = O.Solver(ocfg(s), qref=q0.copy())
    q3, Q = S.calc_direct(q0, 3, store=True)
    qs0 = g["qs0"]
    gsrc = [np.asfortranarray(0.1 * (Qi - q0)) for Qi in Q]
    ref, _ = S.calc_adjoint(qs0, Q, g_fn=lambda qq, nt: gsrc[nt])
    with Cruna(Settings.from_dict(s), qref=q0) as c:
        got = c.calc_adjoint(qs0, Q, g=gsrc)
        one = c.time_stepper_adjoint(qs0, Q[3], gsrc[3])
    assert max(rel_l2_vars(got, ref)) < 1e-12
    ref1 = S.time_stepper_adjoint(qs0, Q[3], gsrc[3])
    assert max(rel_l2_vars(one, ref1)) < 1e-12


def _bc_case(rows, n=(10, 11, 12)):
    q = cases.smooth_random_state(n, seed=7, p0=1.0, rho0=1.0, amp=0.05)
    qref = cases.smooth_random_state(n, seed=8, p0=1.0, rho0=1.0, amp=0.05)
    s = dict(n=n, diff=("o4_e_c_o",) * 3, x1=(1.0, 1.2, 1.4), dt=1e-3, bc=np.array(rows, dtype=float),
             sponge_length=(0.2, 0.3, 0.0), sponge_amplitude=2.0, R=1.0, W=1.0, T0=1.0)
    return s, q, qref


BC_ROWS = {
    "200": [[200, 1, 1, 1, 11, 1, 12, -1, 0, 0], [200, 1, 10, 11, 11, 1, 12, 0, 1, 0]],
    "201": [[201, 1, 10, 1, 11, 1, 1, 0, 0, -1], [201, 10, 10, 1, 11, 1, 12, 1, 0, 0]],
    "204": [[204, 1, 10, 1, 1, 1, 12, 0, -1, 0]],
    "100": [[100, 1, 10, 1, 11, 12, 12, 4, 0, 0]],
    "400": [[400, 1, 10, 1, 11, 1, 12, 0, 0, 0]],
    "401": [[401, 1, 10, 1, 11, 1, 12, 0, 0, 0]],
}


@pytest.mark.parametrize("kind", sorted(BC_ROWS))
def test_boundary_conditions_match_oracle(kind):
    s, q, qref = _bc_case(BC_ROWS[kind])
    S = O.Solver(ocfg(s), qref=qref)
    rhs = cases.smooth_random_state(s["n"], seed=9, p0=0.3, rho0=0.2, amp=0.5)
    qs = cases.smooth_random_state(s["n"], seed=10, p0=0.1, rho0=0.3, amp=0.5)
    with Cruna(Settings.from_dict(s), qref=qref) as c:
        pairs = [
            (c.set_boundary_condition_q(q, True), S.set_boundary_condition_q(q, True)),
            (c.set_boundary_condition_qs(qs, q, True), S.set_boundary_condition_qs(qs, q, True)),
            (c.set_boundary_condition_rhs(rhs, q), S.set_boundary_condition_rhs(rhs, q)),
            (c.set_boundary_condition_rhss(rhs, qs, q), S.set_boundary_condition_rhss(rhs, qs, q)),
            (c.set_boundary_condition_rhss(rhs, qs), S.set_boundary_condition_rhss(rhs, qs)),
            (c.rhs_direct(q), S.rhs_direct(q)),
        ]
    for i, (a, b) in enumerate(pairs):
        assert max(rel_l2_vars(a, b)) < 1e-12, (kind, i, rel_l2_vars(a, b))


def test_forcing_is_added():
    n = (10, 9, 8)
    q = cases.smooth_random_state(n, seed=4)
    f = cases.smooth_random_state(n, seed=5, p0=0.0, rho0=0.0, amp=1.0)
    cfg = O.Config(n=n, diff=("o4_e_c_p",) * 3, mu0=0.01)
    ref = O.Solver(cfg, force=f).rhs_direct(q)
    with Cruna(Settings(n=n, diff=("o4_e_c_p",) * 3, mu0=0.01), force=f) as c:
        assert max(rel_l2_vars(c.rhs_direct(q), ref)) < 1e-12
        c.set_forcing(None)
        ref0 = O.Solver(cfg).rhs_direct(q)
        assert max(rel_l2_vars(c.rhs_direct(q), ref0)) < 1e-12


def test_100_steps_parity_fp64():
    """The north-star bar: FP64 path within 1e-12 relative L2 of the oracle after 100 steps."""
    s, q0 = cases.taylor_green(n=16, seed=0)
    s["mu0"] = 0.01
    S = O.Solver(ocfg(s))
    ref = S.calc_direct(q0, 100)
    with Cruna(Settings.from_dict(s)) as c:
        got = c.calc_direct(q0, 100)
    errs = rel_l2_vars(got, ref)
    assert max(errs) < 1e-12, errs


def test_errors_are_reported():
    with pytest.raises(CrunaError) as e:
        Cruna(Settings(n=(6, 6, 6), diff=("o8_e_c_p",) * 3))      # 8th order needs 8 points
    assert e.value.code == -1
    with pytest.raises(CrunaError) as e:
        Cruna(Settings(n=(8, 8, 8), bc=np.array([[301, 1, 1, 1, 8, 1, 8, -1, 0, 0]], dtype=float)))
    assert e.value.code == -5
    with Cruna(Settings(n=(8, 8, 8))) as c:
        with pytest.raises(CrunaError):
            c._check(c.lib.cruna_diff(c.h, 4, None, None, 1, 1.0))


def test_state_check_reports_bad_state():
    n = (8, 8, 8)
    s, q0 = cases.taylor_green(n=8)
    q0 = np.array(q0, order="F")
    q0[3, 3, 3, 0] = -1.0        # negative density made on the host
    st = Settings.from_dict(s)
    st.check_every = 1
    with Cruna(st) as c:
        with pytest.raises(CrunaError) as e:
            c.calc_direct(q0, 1)
    assert e.value.code == -4
