"""GPU tests of the exact discrete adjoint (cruna_rhs_direct_vjp, cruna_step_direct_vjp and
cruna_gradient in adjoint mode 1) through the C ABI, against the oracle's numpy restatement
(oracle/discrete_adjoint.py, itself checked against central differences on the CPU) and against
central differences of J computed by the library's own direct loop.

Tolerance: the library and the oracle evaluate the same sums in different orders (banded transposes
against dense matrix products, dual numbers against complex steps), so the cotangents agree to
rounding: 1e-10 relative L2 per variable (a variable is measured against max(its norm, 1e-3 of the
state's norm))."""
import numpy as np
import pytest

from oracle import cruna_oracle as O
from oracle import discrete_adjoint as DA
from public_b200 import cases
from public_b200.cruna import Cruna, CrunaError, Settings

pytestmark = pytest.mark.gpu

CFG_FIELDS = {f.name for f in O.dataclasses.fields(O.Config)}
TOL = 1e-10


def ocfg(s: dict) -> O.Config:
    return O.Config(**{k: v for k, v in s.items() if k in CFG_FIELDS})


def cot_err(a, b):
    scale = np.linalg.norm(b.ravel())
    out = []
    for v in range(b.shape[-1]):
        nb = max(np.linalg.norm(b[..., v].ravel()), 1e-3 * scale)
        out.append(float(np.linalg.norm((a[..., v] - b[..., v]).ravel()) / nb))
    return max(out)


def rnd(shape, seed):
    return np.asfortranarray(np.random.default_rng(seed).standard_normal(shape))


@pytest.mark.parametrize("generic", [False, True])
@pytest.mark.parametrize("heat_flux_dx", [False, True])
def test_rhs_vjp_periodic_matches_oracle(generic, heat_flux_dx):
    s, q = cases.taylor_green(n=12, seed=0)
    s.update(mu0=0.02, heat_flux_dx=heat_flux_dx)
    f = cases.smooth_random_state((12, 12, 12), seed=5, p0=0.0, rho0=0.0, amp=0.3)
    lam = rnd(q.shape, 3)
    mu_ref, gf_ref = DA.rhs_vjp(O.Solver(ocfg(s), force=f), q, lam)
    with Cruna(Settings.from_dict(s), force=f) as c:
        c.force_generic(generic)
        gf = np.zeros_like(q, order="F")
        mu = c.rhs_direct_vjp(q, lam, gf)
        mu2 = c.rhs_direct_vjp(q, lam, gf)   # second call: same result, grad_f accumulates
    assert cot_err(mu, mu_ref) < TOL, cot_err(mu, mu_ref)
    assert np.array_equal(mu, mu2)
    assert cot_err(gf, 2 * gf_ref) < TOL


BC_ROWS = {
    "200": [[200, 1, 1, 1, 11, 1, 12, -1, 0, 0], [200, 1, 10, 11, 11, 1, 12, 0, 1, 0]],
    "201": [[201, 1, 10, 1, 11, 1, 1, 0, 0, -1], [201, 10, 10, 1, 11, 1, 12, 1, 0, 0]],
    "204": [[204, 1, 10, 1, 1, 1, 12, 0, -1, 0]],
    "100": [[100, 1, 10, 1, 11, 12, 12, 4, 0, 0]],
    "400": [[400, 1, 10, 1, 11, 1, 12, 0, 0, 0]],
    "401": [[401, 1, 10, 1, 11, 1, 12, 0, 0, 0]],
}


@pytest.mark.parametrize("scheme", ["o4_e_c_o", "o6_i_c_o", "o4_i_c_o_pade"])
@pytest.mark.parametrize("kind", sorted(BC_ROWS))
def test_rhs_vjp_boundaries_match_oracle(kind, scheme):
    n = (10, 11, 12)
    q = cases.smooth_random_state(n, seed=7, p0=1.0, rho0=1.0, amp=0.05)
    qref = cases.smooth_random_state(n, seed=8, p0=1.0, rho0=1.0, amp=0.05)
    f = cases.smooth_random_state(n, seed=5, p0=0.0, rho0=0.0, amp=1.0)
    s = dict(n=n, diff=(scheme,) * 3, x1=(1.0, 1.2, 1.4), dt=1e-3, bc=np.array(BC_ROWS[kind], dtype=float),
             sponge_length=(0.2, 0.3, 0.0), sponge_amplitude=2.0, R=1.0, W=1.0, T0=1.0, mu0=0.01)
    lam = rnd(q.shape, 4)
    mu_ref, gf_ref = DA.rhs_vjp(O.Solver(ocfg(s), qref=qref, force=f), q, lam)
    with Cruna(Settings.from_dict(s), qref=qref, force=f) as c:
        gf = np.zeros_like(q, order="F")
        mu = c.rhs_direct_vjp(q, lam, gf)
    assert cot_err(mu, mu_ref) < TOL, (kind, scheme, cot_err(mu, mu_ref))
    assert cot_err(gf, gf_ref) < TOL, (kind, scheme, cot_err(gf, gf_ref))


def _tgv_filtered():
    s, q = cases.taylor_green(n=12, seed=1)
    s.update(mu0=0.02, filt=("o10_e_c_p",) * 3, di_freq=(1, 2, 1))
    return s, q


@pytest.mark.parametrize("nt", [1, 2])
def test_step_vjp_matches_oracle_filtered_periodic(nt):
    """Fused explicit path with the o10 explicit filter (i2 only every second step)."""
    s, q = _tgv_filtered()
    f = cases.smooth_random_state((12, 12, 12), seed=6, p0=0.0, rho0=0.0, amp=0.3)
    lam = rnd(q.shape, 9)
    l0_ref, gf_ref = DA.step_vjp(O.Solver(ocfg(s), force=f), q, lam, nt)
    with Cruna(Settings.from_dict(s), force=f) as c:
        assert c.rhs_path == "fused"
        gf = np.zeros_like(q, order="F")
        l0 = c.step_direct_vjp(q, lam, nt, gf)
    assert cot_err(l0, l0_ref) < TOL, cot_err(l0, l0_ref)
    assert cot_err(gf, gf_ref) < TOL, cot_err(gf, gf_ref)


def test_step_vjp_matches_oracle_mixing_layer():
    """Generic path: compact o6 in y, open o10 filter, type-201 boundaries and a sponge."""
    s, q = cases.mixing_layer(n=(16, 14, 12))
    lam = rnd(q.shape, 11)
    f = np.zeros_like(q)
    l0_ref, gf_ref = DA.step_vjp(O.Solver(ocfg(s), qref=q.copy(), force=f), q, lam, 1)
    with Cruna(Settings.from_dict(s), qref=q.copy(), force=f) as c:
        gf = np.zeros_like(q, order="F")
        l0 = c.step_direct_vjp(q, lam, 1, gf)
    assert cot_err(l0, l0_ref) < TOL, cot_err(l0, l0_ref)
    assert cot_err(gf, gf_ref) < TOL, cot_err(gf, gf_ref)


@pytest.mark.parametrize("kind", ["kinetic_energy", "plane_p2"])
def test_discrete_gradient_matches_oracle(kind):
    """cruna_gradient in mode 1 with 2, 3 and 6 snapshots for 5 steps against the oracle with the
    whole trajectory kept; J is the continuous mode's J and the number of direct steps is the schedule's
    minimum for the 4 step inputs to reverse plus the final step."""
    s, q0 = _tgv_filtered()
    f = cases.smooth_random_state((12, 12, 12), seed=8, p0=0.0, rho0=0.0, amp=0.3)
    S = O.Solver(ocfg(s), force=f)
    pinf = float(np.mean(q0[..., 4]))
    J, gf, gq = DA.gradient_discrete(S, q0, 5, {"kind": kind, "normal": 1, "index": 5, "p_inf": pinf})
    with Cruna(Settings.from_dict(s), force=f) as c:
        o = c.objective(kind, normal=2, index=6, p_inf=pinf)
        Jc, _, _, _ = c.gradient(q0, 5, 3, o)
        c.set_adjoint_mode(1)
        for nsnap in (2, 3, 6):
            Jg, gfg, gqg, nadv = c.gradient(q0, 5, nsnap, o)
            assert abs(Jg - J) <= 1e-12 * abs(J), (nsnap, Jg, J)
            assert abs(Jg - Jc) <= 1e-13 * abs(J)
            assert cot_err(gqg, gq) < TOL, (nsnap, cot_err(gqg, gq))
            assert cot_err(gfg, gf) < TOL, (nsnap, cot_err(gfg, gf))
            assert nadv == O.treeverse_schedule(4, nsnap)[1] + 1


def test_discrete_gradient_matches_finite_differences_mixing_layer():
    """dJ/dq0 and dJ/df of the plane objective on a mixing layer (o6 compact in y, o10 open filter,
    type-201 boundaries, sponge) against central differences of the library's own J: a step of 1e-7 keeps
    every characteristic boundary point on its branch."""
    s, q0 = cases.mixing_layer(n=(24, 20, 16))
    qref = q0.copy()
    pinf = float(np.mean(q0[..., 4]))
    rng = np.random.default_rng(2)
    eps = 1e-7
    with Cruna(Settings.from_dict(s), qref=qref, force=np.zeros_like(q0)) as c:
        o = c.objective("plane_p2", normal=2, index=8, p_inf=pinf)
        c.set_adjoint_mode(1)
        J, gf, gq, _ = c.gradient(q0, 4, 3, o)
        for _ in range(2):
            d = np.asfortranarray(rng.standard_normal(q0.shape))
            d[..., 4] *= 0.1
            Jp = c.gradient(q0 + eps * d, 4, 5, o)[0]
            Jm = c.gradient(q0 - eps * d, 4, 5, o)[0]
            fd = (Jp - Jm) / (2 * eps)
            assert abs(fd - np.sum(gq * d)) < 1e-6 * abs(fd), (fd, np.sum(gq * d))
        df = np.asfortranarray(rng.standard_normal(q0.shape))
        c.set_forcing(eps * df)
        Jp = c.gradient(q0, 4, 5, o)[0]
        c.set_forcing(-eps * df)
        Jm = c.gradient(q0, 4, 5, o)[0]
        fd = (Jp - Jm) / (2 * eps)
        assert abs(fd - np.sum(gf * df)) < 1e-6 * abs(fd), (fd, np.sum(gf * df))


def test_discrete_mode_needs_fp64():
    s, q = cases.taylor_green(n=12, seed=0)
    s["precision"] = "fp32"
    with Cruna(Settings.from_dict(s)) as c:
        with pytest.raises(CrunaError) as e:
            c.set_adjoint_mode(1)
        assert e.value.code == -5
        with pytest.raises(CrunaError):
            c.rhs_direct_vjp(q, q)


@pytest.mark.parametrize("mode", [0, 1])
def test_optimisation_loop_matches_oracle(mode):
    """cruna_optimize (cruna.f90:78-179 with ls_quadratic_fit) against the oracle's loop: the objective
    of every loop, the line-search step sizes and the final forcing."""
    s, q0 = cases.taylor_green(n=12, seed=3)
    s["mu0"] = 0.02
    S = O.Solver(ocfg(s))
    pinf = float(np.mean(q0[..., 4]))
    o = {"kind": "plane_p2", "normal": 1, "index": 5, "p_inf": pinf}
    f0 = cases.smooth_random_state((12, 12, 12), seed=8, p0=0.0, rho0=0.0, amp=0.01)
    Jr, ar, fr = DA.optimize(S, q0, 4, o, maxloop=3, ls_start=1, alpha0=10.0, f0=f0, discrete=mode == 1)
    with Cruna(Settings.from_dict(s), force=np.zeros_like(q0)) as c:
        c.set_adjoint_mode(mode)
        Jg, ag, fg = c.optimize(q0, c.objective("plane_p2", normal=2, index=6, p_inf=pinf), 4, 3, 3, 1, 10.0, f0)
    assert np.allclose(Jg, Jr, rtol=1e-10, atol=0), (Jg, Jr)
    assert np.allclose(ag, ar, rtol=1e-7, atol=0), (ag, ar)
    assert cot_err(fg, fr) < 1e-8, cot_err(fg, fr)
    assert Jg[-1] < 0.5 * Jg[0]


ZONAL_ROWS = {
    "202": [[202, 1, 10, 1, 1, 1, 12, 0, 0, 0], [202, 10, 10, 1, 11, 1, 12, 0, 0, 0]],
    "203": [[203, 1, 10, 1, 11, 1, 12, 0, 0, 0]],
    "203in": [[203, 1, 10, 1, 11, 1, 12, 1, 0, 0]],
    "203out": [[203, 1, 10, 1, 11, 1, 12, -1, 0, 0]],
    "205": [[205, 1, 10, 11, 11, 1, 12, 0, 0, 0]],
    "206": [[206, 1, 10, 1, 11, 1, 12, 0, 0, 0]],
}


@pytest.mark.parametrize("kv", ["diagonal", "hedgehog"])
@pytest.mark.parametrize("kind", sorted(ZONAL_ROWS))
def test_rhs_and_step_vjp_zonal_boundaries_match_oracle(kind, kv):
    """Zonal characteristic types (normal vectors from the k-vector field, 203/206 weighted by the
    sponge shape, 203 inside and/or outside the RHS): RHS transpose and one loop step transposed."""
    n = (10, 11, 12)
    q = cases.smooth_random_state(n, seed=7, p0=1.0, rho0=1.0, amp=0.05)
    qref = cases.smooth_random_state(n, seed=8, p0=1.0, rho0=1.0, amp=0.05)
    f = cases.smooth_random_state(n, seed=5, p0=0.0, rho0=0.0, amp=1.0)
    s = dict(n=n, diff=("o4_e_c_o",) * 3, x1=(1.0, 1.2, 1.4), dt=1e-3, bc=np.array(ZONAL_ROWS[kind], dtype=float),
             sponge_length=(0.2, 0.3, 0.25), sponge_amplitude=0.8, R=1.0, W=1.0, T0=1.0, mu0=0.01, kvector=kv)
    S = O.Solver(ocfg(s), qref=qref, force=f)
    lam = rnd(q.shape, 4)
    mu_ref, gf_ref = DA.rhs_vjp(S, q, lam)
    l0_ref, gs_ref = DA.step_vjp(S, q, lam, 1)
    with Cruna(Settings.from_dict(s), qref=qref, force=f) as c:
        gf = np.zeros_like(q, order="F")
        mu = c.rhs_direct_vjp(q, lam, gf)
        gs = np.zeros_like(q, order="F")
        l0 = c.step_direct_vjp(q, lam, 1, gs)
    assert cot_err(mu, mu_ref) < TOL, cot_err(mu, mu_ref)
    assert cot_err(gf, gf_ref) < TOL, cot_err(gf, gf_ref)
    assert cot_err(l0, l0_ref) < TOL, cot_err(l0, l0_ref)
    assert cot_err(gs, gs_ref) < TOL, cot_err(gs, gs_ref)
