"""CPU tests of the oracle's exact discrete adjoint (oracle/discrete_adjoint.py): the transposed RHS
against central differences of the oracle's own rhs_direct (dot-product identity
<lam, J v> = <J^T lam, v>), and whole-trajectory gradients against central differences of J.

The characteristic boundary treatments switch waves on and off with the sign of u.n (a kink of the
discrete map), so difference quotients on cases with such boundaries use a step small enough that no
boundary point changes branch."""
import numpy as np
import pytest

from oracle import cruna_oracle as O
from oracle import discrete_adjoint as DA
from public_b200 import cases


def ocfg(s):
    fields = {f.name for f in O.dataclasses.fields(O.Config)}
    return O.Config(**{k: v for k, v in s.items() if k in fields})


def rhs_dot_mismatch(S, q, seed=1, eps=1e-6):
    rng = np.random.default_rng(seed)
    lam = np.asfortranarray(rng.standard_normal(q.shape))
    v = np.asfortranarray(rng.standard_normal(q.shape))
    v[..., 4] *= 0.1
    jv = (S.rhs_direct(q + eps * v) - S.rhs_direct(q - eps * v)) / (2 * eps)
    mu, _ = DA.rhs_vjp(S, q, lam)
    a, b = float(np.sum(lam * jv)), float(np.sum(mu * v))
    return abs(a - b) / abs(a)


@pytest.mark.parametrize("heat_flux_dx", [False, True])
def test_rhs_transpose_periodic_viscous(heat_flux_dx):
    s, q = cases.taylor_green(n=12, seed=0)
    s["mu0"] = 0.02
    s["heat_flux_dx"] = heat_flux_dx
    assert rhs_dot_mismatch(O.Solver(ocfg(s)), q) < 1e-9


BC_ROWS = {
    "200": [[200, 1, 1, 1, 11, 1, 12, -1, 0, 0], [200, 1, 10, 11, 11, 1, 12, 0, 1, 0]],
    "201": [[201, 1, 10, 1, 11, 1, 1, 0, 0, -1], [201, 10, 10, 1, 11, 1, 12, 1, 0, 0]],
    "204": [[204, 1, 10, 1, 1, 1, 12, 0, -1, 0]],
    "100": [[100, 1, 10, 1, 11, 12, 12, 4, 0, 0]],
    "400": [[400, 1, 10, 1, 11, 1, 12, 0, 0, 0]],
    "401": [[401, 1, 10, 1, 11, 1, 12, 0, 0, 0]],
}


def bc_case(kind, scheme, n=(10, 11, 12)):
    q = cases.smooth_random_state(n, seed=7, p0=1.0, rho0=1.0, amp=0.05)
    qref = cases.smooth_random_state(n, seed=8, p0=1.0, rho0=1.0, amp=0.05)
    f = cases.smooth_random_state(n, seed=5, p0=0.0, rho0=0.0, amp=1.0)
    s = dict(n=n, diff=(scheme,) * 3, x1=(1.0, 1.2, 1.4), dt=1e-3, bc=np.array(BC_ROWS[kind], dtype=float),
             sponge_length=(0.2, 0.3, 0.0), sponge_amplitude=2.0, R=1.0, W=1.0, T0=1.0, mu0=0.01)
    return s, q, qref, f


@pytest.mark.parametrize("scheme", ["o4_e_c_o", "o6_i_c_o", "o4_i_c_o_pade", "o2_e_c_o"])
@pytest.mark.parametrize("kind", sorted(BC_ROWS))
def test_rhs_transpose_boundaries_open_and_compact(kind, scheme):
    s, q, qref, f = bc_case(kind, scheme)
    S = O.Solver(ocfg(s), qref=qref, force=f)
    assert rhs_dot_mismatch(S, q, eps=1e-7) < 1e-7, (kind, scheme)


def test_transposed_operators_are_transposes():
    """<D a, b> = <a, D^T b> and the same for the filters, on every scheme of the path."""
    rng = np.random.default_rng(0)
    for scheme in [s for s in O.DIFF_SCHEMES if s != "empty"]:
        cfg = O.Config(n=(14, 3, 2), diff=(scheme, "empty", "empty"), x1=(1.3, 1.0, 1.0))
        a, b = rng.standard_normal((2, 14, 3, 2))
        h = cfg.dx()[0]
        lhs = np.sum(O.Dx(cfg, 0, np.asfortranarray(a), h) * b)
        rhs = np.sum(a * DA.DT(cfg, 0, np.asfortranarray(b), h))
        assert abs(lhs - rhs) < 1e-11 * (abs(lhs) + 1), scheme
    for scheme in [s for s in O.FILTER_SCHEMES if s != "empty"]:
        cfg = O.Config(n=(16, 3, 2), filt=(scheme, "empty", "empty"), alpha=0.3)
        a, b = rng.standard_normal((2, 16, 3, 2, 5))
        lhs = np.sum(O.filter_dir(cfg, 0, np.asfortranarray(a)) * b)
        rhs = np.sum(a * DA.filter_T(cfg, 0, np.asfortranarray(b)))
        assert abs(lhs - rhs) < 1e-11 * (abs(lhs) + 1), scheme


def grad_mismatch(S, q0, steps, obj, eps, seed=2):
    J, gf, gq = DA.gradient_discrete(S, q0, steps, obj)
    assert abs(J - DA.objective_value(S, q0, steps, obj)) <= 1e-13 * abs(J)
    rng = np.random.default_rng(seed)
    d = np.asfortranarray(rng.standard_normal(q0.shape))
    d[..., 4] *= 0.1
    fd = (DA.objective_value(S, q0 + eps * d, steps, obj) - DA.objective_value(S, q0 - eps * d, steps, obj)) / (2 * eps)
    f0 = S.force
    df = np.asfortranarray(rng.standard_normal(q0.shape))
    S.force = f0 + eps * df
    Jp = DA.objective_value(S, q0, steps, obj)
    S.force = f0 - eps * df
    Jm = DA.objective_value(S, q0, steps, obj)
    S.force = f0
    fdf = (Jp - Jm) / (2 * eps)
    return abs(fd - np.sum(gq * d)) / abs(fd), abs(fdf - np.sum(gf * df)) / abs(fdf)


@pytest.mark.parametrize("obj", ["kinetic_energy", "plane_p2"])
def test_gradient_matches_finite_differences_periodic(obj):
    s, q = cases.taylor_green(n=12, seed=0)
    s["mu0"] = 0.02
    S = O.Solver(ocfg(s), force=np.zeros_like(q))
    o = {"kind": obj, "normal": 1, "index": 3, "p_inf": float(q[..., 4].mean())}
    eq, ef = grad_mismatch(S, q, 4, o, eps=1e-6)
    assert eq < 1e-7 and ef < 1e-6, (eq, ef)


def test_gradient_matches_finite_differences_compact_filter():
    s, q = cases.taylor_green(n=12, seed=0)
    s.update(mu0=0.02, filt=("o6_i_c_p",) * 3, alpha=0.3)
    S = O.Solver(ocfg(s), force=np.zeros_like(q))
    eq, ef = grad_mismatch(S, q, 3, {"kind": "kinetic_energy"}, eps=1e-6)
    assert eq < 1e-7 and ef < 1e-6, (eq, ef)


def test_gradient_matches_finite_differences_mixing_layer():
    """Mixing layer: compact o6 in y, o10 open filter, type-201 boundaries and a sponge."""
    s, q = cases.mixing_layer(n=(16, 14, 12))
    S = O.Solver(ocfg(s), qref=q.copy(), force=np.zeros_like(q))
    o = {"kind": "plane_p2", "normal": 2, "index": 5, "p_inf": float(q[..., 4].mean())}
    eq, ef = grad_mismatch(S, q, 3, o, eps=1e-7)
    assert eq < 1e-6 and ef < 1e-6, (eq, ef)


@pytest.mark.parametrize("kind", ["kinetic_energy", "plane_p2"])
def test_continuous_gradient_points_along_the_exact_one(kind):
    """CRUNA's continuous adjoint (with the source sign -dj/dq its backward stepper needs) gives a
    dJ/dq0 and dJ/df along the exact discrete gradient: identical for the terminal kinetic energy, within
    a few degrees for the plane objective (whose source is a plane of delta functions)."""
    s, q = cases.taylor_green(n=12, seed=3)
    s["mu0"] = 0.02
    S = O.Solver(ocfg(s), force=np.zeros_like(q))
    o = {"kind": kind, "normal": 1, "index": 5, "p_inf": float(q[..., 4].mean())}
    _, gfd, gqd = DA.gradient_discrete(S, q, 4, o)
    _, gfc, gqc = O.gradient_store_all(S, q, 4, o)
    cos = lambda a, b: float(np.sum(a * b) / np.linalg.norm(a) / np.linalg.norm(b))
    lim = 0.9999 if kind == "kinetic_energy" else 0.97
    assert cos(gqc, gqd) > lim and cos(gfc, gfd) > lim, (cos(gqc, gqd), cos(gfc, gfd))


def test_optimisation_loop_reduces_the_objective():
    s, q = cases.taylor_green(n=12, seed=3)
    s["mu0"] = 0.02
    S = O.Solver(ocfg(s))
    o = {"kind": "plane_p2", "normal": 1, "index": 5, "p_inf": float(q[..., 4].mean())}
    for discrete in (False, True):
        Js, alphas, f = DA.optimize(S, q, 4, o, maxloop=3, ls_start=1, alpha0=10.0, f0=np.zeros_like(q),
                                    discrete=discrete)
        assert Js[1] < 0.5 * Js[0] and Js[2] <= Js[1] * 1.001, (discrete, Js)
        assert np.all(alphas > 0)


@pytest.mark.parametrize("scheme", ["o8_e_c_p", "o6_i_c_p"])
def test_enstrophy_gradient_matches_finite_differences(scheme):
    """dZ/dq of the enstrophy objective (curl with the solver's operators, transposed for the gradient)."""
    s, q = cases.taylor_green(n=10, seed=1)
    s["diff"] = (scheme,) * 3
    cfg = ocfg(s)
    Z, g = O.objective_enstrophy(cfg, q)
    rng = np.random.default_rng(0)
    d = rng.standard_normal(q.shape)
    eps = 1e-6
    fd = (O.objective_enstrophy(cfg, q + eps * d)[0] - O.objective_enstrophy(cfg, q - eps * d)[0]) / (2 * eps)
    assert Z > 0 and abs(fd - np.sum(g * d)) < 1e-8 * abs(fd)


def test_enstrophy_gradient_through_steps():
    s, q = cases.taylor_green(n=12, seed=0)
    s["mu0"] = 0.02
    S = O.Solver(ocfg(s), force=np.zeros_like(q))
    eq, ef = grad_mismatch(S, q, 3, {"kind": "enstrophy"}, eps=1e-6)
    assert eq < 1e-7 and ef < 1e-6, (eq, ef)
    _, gfd, gqd = DA.gradient_discrete(S, q, 3, {"kind": "enstrophy"})
    _, gfc, gqc = O.gradient_store_all(S, q, 3, {"kind": "enstrophy"})
    cos = float(np.sum(gqc * gqd) / np.linalg.norm(gqc) / np.linalg.norm(gqd))
    assert cos > 0.9999, cos


ZONAL_ROWS = {
    "202": [[202, 1, 10, 1, 1, 1, 12, 0, 0, 0], [202, 10, 10, 1, 11, 1, 12, 0, 0, 0]],
    "203": [[203, 1, 10, 1, 11, 1, 12, 0, 0, 0]],
    "203in": [[203, 1, 10, 1, 11, 1, 12, 1, 0, 0]],
    "203out": [[203, 1, 10, 1, 11, 1, 12, -1, 0, 0]],
    "205": [[205, 1, 10, 11, 11, 1, 12, 0, 0, 0]],
    "206": [[206, 1, 10, 1, 11, 1, 12, 0, 0, 0]],
}


def zonal_case(kind, kv="hedgehog", scheme="o4_e_c_o"):
    n = (10, 11, 12)
    q = cases.smooth_random_state(n, seed=7, p0=1.0, rho0=1.0, amp=0.05)
    qref = cases.smooth_random_state(n, seed=8, p0=1.0, rho0=1.0, amp=0.05)
    s = dict(n=n, diff=(scheme,) * 3, x1=(1.0, 1.2, 1.4), dt=1e-3, bc=np.array(ZONAL_ROWS[kind], dtype=float),
             sponge_length=(0.2, 0.3, 0.25), sponge_amplitude=0.8, R=1.0, W=1.0, T0=1.0, mu0=0.01, kvector=kv)
    return s, q, qref


@pytest.mark.parametrize("kind", sorted(ZONAL_ROWS))
def test_rhs_transpose_zonal_boundaries(kind):
    """Zonal characteristic types 202/203 (on q) and 205/206 (on the RHS): <lam, J v> = <J^T lam, v>."""
    s, q, qref = zonal_case(kind)
    S = O.Solver(ocfg(s), qref=qref)
    assert rhs_dot_mismatch(S, q, eps=1e-7) < 1e-7, kind


@pytest.mark.parametrize("kind", ["203out", "206"])
def test_step_transpose_zonal_boundaries(kind):
    """One loop step (RK4, the outside-RHS boundary update, filters) against central differences of J."""
    s, q, qref = zonal_case(kind, kv="diagonal")
    S = O.Solver(ocfg(s), qref=qref, force=np.zeros_like(q))
    eq, ef = grad_mismatch(S, q, 2, {"kind": "kinetic_energy"}, eps=1e-7)
    assert eq < 1e-6 and ef < 1e-6, (eq, ef)
