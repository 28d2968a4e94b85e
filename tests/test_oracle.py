"""CPU tests of the oracle: the known-answer properties of the reference's own unit tests
(usr/unit_test/diff, usr/unit_test/filter), LAPACK agreement, conservation and the golden fixtures."""
import math
import os

import numpy as np
import pytest
from scipy.linalg import lapack

from oracle import cruna_oracle as O
from public_b200 import cases

GOLD = os.path.join(os.path.dirname(__file__), "golden")

DESIGN_ORDER = {"o2_e_c_o": 2, "o4_e_c_p": 4, "o4_e_c_o": 4, "o4_i_c_p_pade": 4, "o4_i_c_o_pade": 4,
                "o6_i_c_p": 6, "o6_i_c_o": 4, "o8_e_c_p": 8}


@pytest.mark.parametrize("scheme", [s for s in O.DIFF_SCHEMES if s != "empty"])
def test_diff_known_answers(scheme):
    """usr/unit_test/diff/computation_direct.f90: d/dx of 0 and 1 is 0, d/dx sin(x) = cos(x)."""
    errs = []
    for n in (32, 64):
        per = O.diff_type(scheme) == "periodic"
        L = 2 * math.pi
        dx = L / n if per else L / (n - 1)
        x = np.arange(n) * dx
        f = np.sin(x)[:, None] * np.ones((1, 3))
        d = O.diff_core(scheme, f, dx)
        errs.append(np.max(np.abs(d[:, 0] - np.cos(x))))
        assert np.max(np.abs(O.diff_core(scheme, np.zeros((n, 2)), dx))) == 0.0
        assert np.max(np.abs(O.diff_core(scheme, np.ones((n, 2)), dx))) < 1e-12
    order = math.log2(errs[0] / errs[1])
    assert order > DESIGN_ORDER[scheme] - 0.3, (scheme, order, errs)


def test_diff_empty_is_zero():
    assert np.all(O.diff_core("empty", np.random.rand(7, 3), math.inf) == 0.0)


@pytest.mark.parametrize("scheme", O.FILTER_SCHEMES)
def test_filter_constant_preservation(scheme):
    """usr/unit_test/filter/computation_direct.f90: filter(1) = 1.  The open o2 core applies the
    periodic Sherman-Morrison correction to a line whose end points are left untouched, so it does
    not preserve constants next to the ends; the oracle keeps that reference behaviour."""
    one = O.filter_core(scheme, np.ones((120, 2)), 0.35)
    err = np.max(np.abs(one - 1.0))
    if scheme == "o2_i_c_o":
        assert err > 1e-3
        assert np.max(np.abs(one[50:70] - 1.0)) < 1e-9    # the defect decays away from the ends
    else:
        assert err < 1e-14


def test_cyclic_factors_solve_the_cyclic_matrix():
    n, alpha = 17, 1.0 / 3.0
    f = O.cyclic_factors(n, alpha, 1.0)
    B = np.eye(n) + alpha * (np.eye(n, k=1) + np.eye(n, k=-1))
    B[0, n - 1] = B[n - 1, 0] = alpha
    b = np.random.default_rng(0).standard_normal((n, 3))
    x = f.solve(b)
    assert np.max(np.abs(B @ x - b)) < 1e-13


def test_oracle_factors_are_lapack():
    f = O.diff_factors("o6_i_c_o", 20)
    dl = np.full(19, 1.0 / 3.0)
    d = np.ones(20)
    du = np.full(19, 1.0 / 3.0)
    du[0], du[1], du[18] = 3.0, 0.25, 0.25
    dl[0], dl[18], dl[17] = 0.25, 3.0, 0.25
    ref = lapack.dgttrf(dl, d, du)
    assert np.array_equal(f.ipiv, ref[4]) and np.array_equal(f.d, ref[1])


def test_mass_conservation_periodic():
    s, q = cases.taylor_green(n=12)
    s["mu0"] = 0.01
    cfg = O.Config(**{k: v for k, v in s.items() if k in {f.name for f in O.dataclasses.fields(O.Config)}})
    S = O.Solver(cfg)
    q3 = S.calc_direct(q, 3)
    assert abs(q3[..., 0].sum() - q[..., 0].sum()) < 1e-11 * q[..., 0].sum()


def test_inviscid_limit_drops_viscous_terms():
    """mu0 = 0 makes tau and the heat flux vanish: the NS RHS equals its Euler part."""
    n = (12, 10, 8)
    q = cases.smooth_random_state(n, seed=3)
    cfg = O.Config(n=n, diff=("o4_e_c_p",) * 3, mu0=0.0)
    S = O.Solver(cfg)
    r = S.rhs_direct(q)
    dx = cfg.dx()
    D = lambda d, f: O.Dx(cfg, d, f, dx[d])
    u = [q[..., 1] / q[..., 0], q[..., 2] / q[..., 0], q[..., 3] / q[..., 0]]
    mass = -(D(0, q[..., 1]) + D(1, q[..., 2]) + D(2, q[..., 3]))
    assert np.max(np.abs(r[..., 0] - mass)) < 1e-12 * np.max(np.abs(mass))
    g = cfg.gamma
    e = (g / (g - 1) * -(D(0, q[..., 4] * u[0]) + D(1, q[..., 4] * u[1]) + D(2, q[..., 4] * u[2]))
         + u[0] * D(0, q[..., 4]) + u[1] * D(1, q[..., 4]) + u[2] * D(2, q[..., 4])) * (g - 1)
    assert np.max(np.abs(r[..., 4] - e)) < 1e-11 * np.max(np.abs(e))


def test_goldens_reproduce():
    """The committed fixtures are what the oracle computes (a change of the oracle is noticed)."""
    g = np.load(os.path.join(GOLD, "operators.npz"))
    q = g["q"]
    n = q.shape[:3]
    for s in O.DIFF_SCHEMES:
        cfg = O.Config(n=n, diff=(s, s, s))
        dx = cfg.dx()
        for d in range(3):
            np.testing.assert_array_equal(O.Dx(cfg, d, q[..., 4], dx[d]), g[f"diff_{s}_{d + 1}"])
    for s in O.FILTER_SCHEMES:
        cfg = O.Config(n=n, filt=(s, s, s), alpha=0.3)
        for d in range(3):
            np.testing.assert_array_equal(O.filter_dir(cfg, d, q[..., 4:5])[..., 0], g[f"filter_{s}_{d + 1}"])
    t = np.load(os.path.join(GOLD, "tgv12.npz"))
    s, q0 = cases.taylor_green(n=12, seed=0)
    np.testing.assert_array_equal(q0, t["q0"])
    s["mu0"] = float(t["mu0"])
    cfg = O.Config(**{k: v for k, v in s.items() if k in {f.name for f in O.dataclasses.fields(O.Config)}})
    np.testing.assert_array_equal(O.Solver(cfg).rhs_direct(q0), t["rhs"])


def test_sponge_shape_matches_reference_formula():
    cfg = O.Config(n=(20, 30, 1), x0=(0, 0, 0), x1=(1.0, 2.0, 1.0), diff=("o4_e_c_o", "o4_e_c_o", "empty"),
                   sponge_length=(0.2, 0.5, 0.0), sponge_amplitude=3.0)
    sh = O.sponge_shape(cfg)
    assert sh.shape == (20, 30, 1)
    assert abs(sh[0, 15, 0] - 3.0) < 1e-14           # at the x-boundary phi = 0 -> shape = amp
    assert abs(sh[10, 15, 0]) < 1e-14                  # interior: no sponge
    assert np.all(sh >= 0) and np.all(sh <= 3.0 + 1e-14)


def test_cpu_twin_matches_oracle():
    """The C + OpenMP restatement used as the timed CPU baseline reproduces the numpy oracle."""
    from oracle import cpu_twin
    s, q0 = cases.taylor_green(n=12, seed=2)
    s["mu0"] = 0.02
    s["ai_freq"] = (1, 1, 1)
    fields = {f.name for f in O.dataclasses.fields(O.Config)}
    S = O.Solver(O.Config(**{k: v for k, v in s.items() if k in fields}))
    qs0 = cases.smooth_random_state((12, 12, 12), seed=3, p0=0.0, rho0=0.0, amp=1.0)
    q, qs = q0.copy(order="F"), qs0.copy(order="F")
    for it in range(2):
        q = S.calc_direct(q, 1, nt0=it)
        qs, _ = S.calc_adjoint(qs, [q, q])
    qc, qsc = q0.copy(order="F"), qs0.copy(order="F")
    cpu_twin.run(s, qc, qsc, 2, 2)
    assert max(O.rel_l2(qc[..., v], q[..., v]) for v in range(5)) < 1e-12
    assert max(O.rel_l2(qsc[..., v], qs[..., v]) for v in range(5)) < 1e-12


def test_checkpoint_schedule_order_memory_and_optimality():
    """Binomial checkpointing: adjoint steps T..1 each once, never more than `slots` snapshots alive,
    store-all when slots > steps, and the advanced-step count equals the exhaustive minimum."""
    import functools

    @functools.lru_cache(None)
    def exhaustive(n, s):
        if n <= 0:
            return 0
        if s == 0:
            return n * (n + 1) // 2
        return min(k + exhaustive(n - k, s - 1) + exhaustive(k - 1, s) for k in range(1, n + 1))

    for steps in range(1, 41):
        for slots in range(1, 7):
            acts, adv = O.treeverse_schedule(steps, slots)
            assert [a[1] for a in acts if a[0] == "adjoint"] == list(range(steps, 0, -1))
            live = mx = 1
            for a in acts:
                if a[0] == "store":
                    live += 1
                    mx = max(mx, live)
                elif a[0] == "free":
                    live -= 1
            assert mx <= slots
            assert adv == exhaustive(steps, min(slots - 1, steps))
    assert O.treeverse_schedule(25, 26)[1] == 25


def test_continuous_adjoint_gradient_plumbing_single_step():
    """Sign and assembly of dJ/dq0 (final-time kinetic energy) with CRUNA's continuous adjoint
    (ns_rho_rhou_p.f90:257-536) on one small step, where the continuous adjoint's O(dt^2) deviation
    from the discrete map is negligible."""
    n = (12, 12, 12)
    q0 = cases.smooth_random_state(n, seed=21, p0=1.0, rho0=1.0, amp=0.05, x1=(1.0, 1.0, 1.0))
    cfg = O.Config(n=n, diff=("o8_e_c_p",) * 3, dt=2e-5, mu0=0.0, R=1.0, W=1.0, T0=1.0)
    S = O.Solver(cfg)
    J, gf, gq = O.gradient_store_all(S, q0, 1, {"kind": "kinetic_energy"})
    for k in range(3):
        d = cases.smooth_random_state(n, seed=40 + k, p0=0.0, rho0=0.0, amp=0.01)
        eps = 1e-4
        fd = (O.objective_kinetic_energy(cfg, S.calc_direct(q0 + eps * d, 1))[0]
              - O.objective_kinetic_energy(cfg, S.calc_direct(q0 - eps * d, 1))[0]) / (2 * eps)
        assert abs(fd - float(np.sum(gq * d))) < 1e-3 * float(np.linalg.norm(gq) * np.linalg.norm(d))


def test_continuous_adjoint_is_not_the_discrete_transpose():
    """Dot-product test <qs, L dq> vs <rhs_adjoint(qs), dq> with L the linearised direct RHS: CRUNA's
    continuous adjoint does not satisfy it (it is not the transpose of the discrete operator), which is
    why an exact finite-difference gradient check needs a discrete adjoint."""
    n = (12, 12, 12)
    q = cases.smooth_random_state(n, seed=21, p0=1.0, rho0=1.0, amp=0.05)
    S = O.Solver(O.Config(n=n, diff=("o8_e_c_p",) * 3, mu0=0.0, R=1.0, W=1.0, T0=1.0))
    ratios = []
    for seed in range(2):
        dq = cases.smooth_random_state(n, seed=50 + seed, p0=0.0, rho0=0.0, amp=1.0)
        qs = cases.smooth_random_state(n, seed=60 + seed, p0=0.0, rho0=0.0, amp=1.0)
        eps = 1e-6
        Ldq = (S.rhs_direct(q + eps * dq) - S.rhs_direct(q - eps * dq)) / (2 * eps)
        ratios.append(float(np.sum(S.rhs_adjoint(qs, q, np.zeros_like(q)) * dq)) / float(np.sum(qs * Ldq)))
    assert any(abs(abs(r) - 1.0) > 0.2 for r in ratios), ratios


def test_cpu_twin_matches_oracle_mixing_layer():
    """The C restatement on the mixing-layer scheme set (o6 compact open y-derivatives with dgttrs on the
    LAPACK factors, the o10 compact open y filter, type-201 characteristic rows at both y ends, the
    20-point type-400 sponge) reproduces the numpy oracle over 3 direct + adjoint step pairs."""
    from oracle import cpu_twin
    n = (24, 20, 16)
    s, q0 = cases.mixing_layer(n=n)
    assert cpu_twin.supports(s)
    fields = {f.name for f in O.dataclasses.fields(O.Config)}
    S = O.Solver(O.Config(**{k: v for k, v in s.items() if k in fields}), qref=q0.copy())
    qs0 = cases.smooth_random_state(n, seed=3, p0=0.0, rho0=0.0, amp=1e-2)
    q, qs = q0.copy(order="F"), qs0.copy(order="F")
    for it in range(3):
        q = S.calc_direct(q, 1, nt0=it)
        qs, _ = S.calc_adjoint(qs, [q, q])
    qc, qsc = q0.copy(order="F"), qs0.copy(order="F")
    cpu_twin.run(s, qc, qsc, 3, 2, qref=q0)
    assert max(O.rel_l2(qc[..., v], q[..., v]) for v in range(5)) < 1e-12
    assert max(O.rel_l2(qsc[..., v], qs[..., v]) for v in range(5)) < 1e-12
