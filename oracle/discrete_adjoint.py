"""Exact discrete adjoint of the direct time step (TEST INFRASTRUCTURE: the reference the tests hold
the library's discrete-adjoint entry points against; only ``tests/`` may import it).

The reference has no discrete adjoint: its adjoint (src/equations/ns_rho_rhou_p.f90:257-536) is the
continuous inviscid adjoint, which is not the transpose of the discrete direct operator.  This module
restates, in numpy and in reverse mode, the exact transpose of the direct step the oracle computes
(``cruna_oracle.Solver``):

* ``rhs_vjp``: (d rhs_direct / d q)^T lam for right_hand_side_direct_3d (ns_rho_rhou_p.f90:31-253),
  through the BC on q (:92), the primitives, the 42 derivatives, Sutherland viscosity, stresses, heat
  flux and friction work (:95-209), the forcing (:212) and the BC on the RHS (:218);
* ``step_vjp``: the transpose of one loop step of calc_direct (computation_direct.f90:64-107):
  classical RK4 (rk_o4_e.f90:17-58), BC on q outside the RHS, filters i1, i2, i3;
* ``gradient_discrete``: J, dJ/df and dJ/dq0 of the objectives of ``cruna_oracle.gradient_store_all``
  with the whole trajectory stored, exact to rounding for the discrete solution.

Transposed line operators come from dense line matrices (the oracle's own derivative / filter cores
applied to the identity), transposed with numpy -- an independent route from the library's banded
transposes.  Boundary-condition Jacobians of the characteristic treatments (nonreflecting.f90:46-137
and :237-341) are taken by complex-step differentiation of the oracle's own functions, which is exact
to rounding (no difference quotient).
"""
from __future__ import annotations

import functools
from typing import Dict, Optional, Tuple

import numpy as np

from oracle import cruna_oracle as O

S1 = 110.4


# ------------------------------------------------------------------------------------------------
# transposed line operators
# ------------------------------------------------------------------------------------------------
@functools.lru_cache(maxsize=64)
def _diff_matrix(name: str, n: int, h: float) -> np.ndarray:
    return O.diff_core(name, np.eye(n), h)


@functools.lru_cache(maxsize=64)
def _filter_matrix(name: str, n: int, alpha: float, strength: float) -> np.ndarray:
    return O.filter_core(name, np.eye(n), alpha, strength)


def DT(cfg: O.Config, d: int, f: np.ndarray, h: Optional[float] = None) -> np.ndarray:
    """Transpose of Dx_d (``cruna_oracle.Dx``) applied to a field."""
    M = _diff_matrix(cfg.diff[d], cfg.n[d], 1.0 if h is None else float(h))
    return O._along(f, d, lambda L: M.T @ L)


def filter_T(cfg: O.Config, d: int, q: np.ndarray) -> np.ndarray:
    """Transpose of filter_i_d (``cruna_oracle.filter_dir``) applied to a state."""
    M = _filter_matrix(cfg.filt[d], cfg.n[d], float(cfg.alpha), float(cfg.strength))
    out = np.empty_like(q)
    for v in range(q.shape[3]):
        out[..., v] = O._along(q[..., v], d, lambda L: M.T @ L)
    return out


# ------------------------------------------------------------------------------------------------
# complex-step Jacobians of point-wise boundary treatments
# ------------------------------------------------------------------------------------------------
_CS = 1e-40


def _cs_vjp(fn, args, wrt, lam):
    """sum_i lam_i d fn_i / d args[wrt]_j for a point-wise fn of (..., 5) arrays, by complex step."""
    x = args[wrt]
    out = np.zeros(x.shape, dtype=np.float64)
    for j in range(x.shape[-1]):
        a = [np.asarray(v, dtype=np.complex128) for v in args]
        a[wrt] = a[wrt].copy()
        a[wrt][..., j] += 1j * _CS
        col = np.imag(fn(*a)) / _CS        # d fn / d x_j, shape (..., 5)
        out[..., j] = np.sum(lam * col, axis=-1)
    return out


def _apply_q_row(S: O.Solver, row, q: np.ndarray, outside_rhs: bool = False) -> np.ndarray:
    """One row of set_boundary_condition_q (boundary_conditions.f90:52-136), as the oracle applies it."""
    cfg = S.cfg
    t = int(round(row[0]))
    b = O._box(row)
    q = q.copy(order="F")
    if t == 200:
        sh = O._zero_grad_shift(row)
        b2 = tuple(slice(s.start + o, s.stop + o) for s, o in zip(b, sh))
        q[b] = O.characteristic_q_k1d(cfg, q[b], q[b2], row[7:10])
    elif t == 201:
        q[b] = O.characteristic_q_k1d(cfg, q[b], S.qref[b], row[7:10])
    elif t == 202:
        q[b] = O.characteristic_q_k1d(cfg, q[b], S.qref[b], S.kvec[b])
    elif t == 203 and O._zonal_active(row, outside_rhs):
        q = O.characteristic_q_k1d(cfg, q, S.qref, S.kvec, S.shape)
    elif t == 401:
        for v in range(5):
            q[..., v] = q[..., v] - S.shape * (q[..., v] - S.qref[..., v])
    return q


def bc_q_vjp(S: O.Solver, q_in: np.ndarray, lam: np.ndarray,
             outside_rhs: bool = False) -> Tuple[np.ndarray, np.ndarray]:
    """Transpose of set_boundary_condition_q(q, outside_rhs) at q_in; returns (lam_in, q after the BC)."""
    states = []
    q = q_in
    for row in S.bc:
        states.append(q)
        q = _apply_q_row(S, row, q, outside_rhs)
    lam = lam.copy(order="F")
    cfg = S.cfg
    for row, qpre in zip(S.bc[::-1], states[::-1]):
        t = int(round(row[0]))
        b = O._box(row)
        k = row[7:10]
        if t == 401:
            lam = lam * (1.0 - S.shape)[..., None]
        elif t == 202:
            fn = lambda qq: O.characteristic_q_k1d(cfg, qq, S.qref[b], S.kvec[b])
            lam[b] = _cs_vjp(fn, [qpre[b]], 0, lam[b])
        elif t == 203 and O._zonal_active(row, outside_rhs):
            fn = lambda qq: O.characteristic_q_k1d(cfg, qq, S.qref, S.kvec, S.shape)
            lam = _cs_vjp(fn, [qpre], 0, lam)
        elif t == 201:
            fn = lambda qq: O.characteristic_q_k1d(cfg, qq, S.qref[b], k)
            lam[b] = _cs_vjp(fn, [qpre[b]], 0, lam[b])
        elif t == 200:
            sh = O._zero_grad_shift(row)
            b2 = tuple(slice(s.start + o, s.stop + o) for s, o in zip(b, sh))
            fn = lambda qq, aa: O.characteristic_q_k1d(cfg, qq, aa, k)
            lb = lam[b].copy()
            lq = _cs_vjp(fn, [qpre[b], qpre[b2]], 0, lb)
            la = _cs_vjp(fn, [qpre[b], qpre[b2]], 1, lb)
            lam[b] = lq
            lam[b2] = lam[b2] + la
    return np.asfortranarray(lam), q


def _rhs_pre_bc(S: O.Solver, qb: np.ndarray) -> np.ndarray:
    """rhs_direct of the post-BC state before set_boundary_condition_rhs (:31-212)."""
    S0 = O.Solver(S.cfg.__class__(**{**S.cfg.__dict__, "bc": None}), qref=S.qref, force=S.force)
    return S0.rhs_direct(qb)


def bc_rhs_vjp(S: O.Solver, qb: np.ndarray, lam: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Transpose of set_boundary_condition_rhs(rhs, qb) (boundary_conditions.f90:228-298):
    returns (cotangent of the RHS before the BC, cotangent of qb)."""
    cfg = S.cfg
    rows = [r for r in S.bc if int(round(r[0])) in (100, 204, 205, 206, 400)]
    lam_q = np.zeros_like(qb)
    if not rows:
        return lam.copy(order="F"), lam_q
    pre = []
    if any(int(round(r[0])) in (204, 205, 206) for r in rows):
        rhs = _rhs_pre_bc(S, qb)
        for row in rows:
            pre.append(rhs.copy())
            t = int(round(row[0]))
            b = O._box(row)
            if t == 100:
                rhs[b + (int(round(row[7])) - 1,)] = 0.0
            elif t == 204:
                rhs[b] = O.characteristic_rhs_k1d(cfg, rhs[b], qb[b], S.qref[b], row[7:10])
            elif t == 205:
                rhs[b] = O.characteristic_rhs_k1d(cfg, rhs[b], qb[b], S.qref[b], S.kvec[b])
            elif t == 206:
                rhs = O.characteristic_rhs_k1d(cfg, rhs, qb, S.qref, S.kvec, S.shape)
            else:
                for v in range(5):
                    rhs[..., v] = rhs[..., v] - S.shape * (qb[..., v] - S.qref[..., v])
    else:
        pre = [None] * len(rows)
    lam = lam.copy(order="F")
    for row, rpre in zip(rows[::-1], pre[::-1]):
        t = int(round(row[0]))
        b = O._box(row)
        if t == 100:
            lam[b + (int(round(row[7])) - 1,)] = 0.0
        elif t == 400:
            lam_q = lam_q - S.shape[..., None] * lam
        elif t == 205:
            fn = lambda rr, qq: O.characteristic_rhs_k1d(cfg, rr, qq, S.qref[b], S.kvec[b])
            lb = lam[b].copy()
            lam_q[b] = lam_q[b] + _cs_vjp(fn, [rpre[b], qb[b]], 1, lb)
            lam[b] = _cs_vjp(fn, [rpre[b], qb[b]], 0, lb)
        elif t == 206:
            fn = lambda rr, qq: O.characteristic_rhs_k1d(cfg, rr, qq, S.qref, S.kvec, S.shape)
            lb = lam.copy()
            lam_q = lam_q + _cs_vjp(fn, [rpre, qb], 1, lb)
            lam = _cs_vjp(fn, [rpre, qb], 0, lb)
        else:
            k = row[7:10]
            fn = lambda rr, qq: O.characteristic_rhs_k1d(cfg, rr, qq, S.qref[b], k)
            lb = lam[b].copy()
            lam_q[b] = lam_q[b] + _cs_vjp(fn, [rpre[b], qb[b]], 1, lb)
            lam[b] = _cs_vjp(fn, [rpre[b], qb[b]], 0, lb)
    return lam, lam_q


# ------------------------------------------------------------------------------------------------
# transpose of the interior RHS (ns_rho_rhou_p.f90:95-209)
# ------------------------------------------------------------------------------------------------
def _unique(v: int, d: int) -> Tuple[int, int]:
    return (v, d) if v <= d else (d, v)


def rhs_interior_vjp(S: O.Solver, q: np.ndarray, lam: np.ndarray) -> np.ndarray:
    cfg = S.cfg
    g = cfg.gamma
    gm1 = g - 1.0
    gt = g / gm1
    dx = S.dx
    hT = S.dx if cfg.heat_flux_dx else (None, None, None)
    rho = q[..., 0]
    m = [q[..., 1 + v] for v in range(3)]
    p = q[..., 4]
    u = [m[v] / rho for v in range(3)]
    T = O.give_T(cfg, q)
    mu = O.give_mu(cfg, T)
    lam_th = O.give_lambda(cfg, mu)
    cp_pr = cfg.cp() / cfg.Pr
    G = [[O.Dx(cfg, d, u[v], dx[d]) for d in range(3)] for v in range(3)]      # G[v][d] = d_d u_v
    Tg = [O.Dx(cfg, d, T, hT[d]) for d in range(3)]
    P = [O.Dx(cfg, v, p, dx[v]) for v in range(3)]
    div = G[0][0] + G[1][1] + G[2][2]

    def tau(v, d):
        if v == d:
            return -(2.0 / 3.0 * mu * div) + 2 * mu * G[v][v]
        return mu * (G[v][d] + G[d][v])

    z = np.zeros_like(rho)
    mb = [z.copy() for _ in range(3)]
    ub = [z.copy() for _ in range(3)]
    pb = z.copy()
    mub = z.copy()
    taub: Dict[Tuple[int, int], np.ndarray] = {(a, b): z.copy() for a in range(3) for b in range(a, 3)}
    Tgb = [None] * 3
    L5 = gm1 * lam[..., 4]
    for d in range(3):
        Lam = [DT(cfg, d, lam[..., k], dx[d]) for k in range(5)]
        mb[d] = mb[d] - Lam[0]                                   # mass (:131-135)
        for v in range(3):                                       # momentum fluxes and stresses (:138-177)
            mb[d] = mb[d] - u[v] * Lam[1 + v]
            ub[v] = ub[v] - m[d] * Lam[1 + v]
            taub[_unique(v, d)] = taub[_unique(v, d)] + Lam[1 + v]
        e = -gt * gm1 * Lam[4]                                   # pressure flux (:180-186)
        ub[d] = ub[d] + p * e
        pb = pb + u[d] * e
        hb = gm1 * DT(cfg, d, lam[..., 4], hT[d])                # heat-flux divergence (:189-200)
        Tgb[d] = lam_th * hb
        mub = mub + cp_pr * Tg[d] * hb
    Gb = [[None] * 3 for _ in range(3)]
    for v in range(3):                                           # friction work (:204-206)
        for d in range(3):
            taub[_unique(v, d)] = taub[_unique(v, d)] + L5 * G[v][d]
            Gb[v][d] = L5 * tau(v, d)
        ub[v] = ub[v] + L5 * P[v]                                # u . grad p (:187)
    for (a, b), tb in taub.items():                              # stresses (:118-128)
        if a == b:
            mub = mub + tb * (-(2.0 / 3.0) * div + 2 * G[a][a])
        else:
            mub = mub + tb * (G[a][b] + G[b][a])
    st = taub[(0, 0)] + taub[(1, 1)] + taub[(2, 2)]
    for v in range(3):
        Gb[v][v] = Gb[v][v] + 2 * mu * taub[(v, v)] - (2.0 / 3.0) * mu * st
        for d in range(3):
            if d != v:
                Gb[v][d] = Gb[v][d] + mu * taub[_unique(v, d)]
    Tb = mub * mu * (1.5 / T - 1.0 / (T + S1))                  # Sutherland (trafos.f90:140)
    for v in range(3):
        pb = pb + DT(cfg, v, -lam[..., 1 + v] + L5 * u[v], dx[v])
        for d in range(3):
            ub[v] = ub[v] + DT(cfg, d, Gb[v][d], dx[d])
    for d in range(3):
        Tb = Tb + DT(cfg, d, Tgb[d], hT[d])
    out = np.zeros_like(q)
    WoR = cfg.W / cfg.R
    out[..., 0] = -(ub[0] * u[0] + ub[1] * u[1] + ub[2] * u[2]) / rho - Tb * T / rho
    for v in range(3):
        out[..., 1 + v] = mb[v] + ub[v] / rho
    out[..., 4] = pb + WoR * Tb / rho
    return out


def rhs_vjp(S: O.Solver, q_in: np.ndarray, lam: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """(d rhs_direct/d q)^T lam at q_in, and the cotangent of the forcing (d rhs/d f)^T lam."""
    _, qb = bc_q_vjp(S, q_in, np.zeros_like(q_in))
    lam_pre, lam_qb = bc_rhs_vjp(S, qb, lam)
    lam_qb = lam_qb + rhs_interior_vjp(S, qb, lam_pre)
    lam_q, _ = bc_q_vjp(S, q_in, lam_qb)
    return lam_q, lam_pre


# ------------------------------------------------------------------------------------------------
# one loop step of calc_direct and its transpose
# ------------------------------------------------------------------------------------------------
def loop_step(S: O.Solver, q: np.ndarray, nt: int) -> np.ndarray:
    """computation_direct.f90:64-107 for one step (the oracle's calc_direct body)."""
    qn = S.time_stepper_direct(q, nt * S.cfg.dt)
    qn = S.set_boundary_condition_q(qn, outside_rhs=True)
    for d in range(3):
        if nt % S.cfg.di_freq[d] == 0:
            qn = S.filter_i(d, qn)
    return qn


def step_vjp(S: O.Solver, q0: np.ndarray, lam1: np.ndarray, nt: int) -> Tuple[np.ndarray, np.ndarray]:
    """Transpose of ``loop_step`` at q0 applied to lam1; returns (lam0, dJ/df contribution)."""
    cfg = S.cfg
    dt = cfg.dt
    dth = 0.5 * dt
    Q1 = q0
    k1 = S.rhs_direct(Q1)
    Q2 = q0 + dth * k1
    k2 = S.rhs_direct(Q2)
    Q3 = q0 + dth * k2
    k3 = S.rhs_direct(Q3)
    Q4 = q0 + dt * k3
    k4 = S.rhs_direct(Q4)
    q1 = np.asfortranarray(q0 + dt / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4))
    lam = lam1
    for d in (2, 1, 0):
        if nt % cfg.di_freq[d] == 0:
            lam = filter_T(cfg, d, lam)
    lam_q1, _ = bc_q_vjp(S, q1, lam, outside_rhs=True)
    lk = dt / 6.0 * lam_q1
    mu4, f4 = rhs_vjp(S, Q4, lk)
    lk = dt / 3.0 * lam_q1 + dt * mu4
    mu3, f3 = rhs_vjp(S, Q3, lk)
    lk = dt / 3.0 * lam_q1 + dth * mu3
    mu2, f2 = rhs_vjp(S, Q2, lk)
    lk = dt / 6.0 * lam_q1 + dth * mu2
    mu1, f1 = rhs_vjp(S, Q1, lk)
    lam0 = lam_q1 + mu1 + mu2 + mu3 + mu4
    return np.asfortranarray(lam0), np.asfortranarray(f1 + f2 + f3 + f4)


def objective_value(S: O.Solver, q0: np.ndarray, steps: int, objective: dict) -> float:
    """J of ``cruna_oracle.gradient_store_all`` for the discrete trajectory started from q0."""
    cfg = S.cfg
    q = q0
    J = 0.0
    for nt in range(1, steps + 1):
        q = loop_step(S, q, nt)
        if objective["kind"] == "plane_p2":
            J += cfg.dt * O.objective_plane_p2(cfg, q, objective["normal"], objective["index"],
                                               objective["p_inf"])[0]
    if objective["kind"] != "plane_p2":
        J = O.terminal_objective(cfg, q, objective["kind"])[0]
    return J


def gradient_discrete(S: O.Solver, q0: np.ndarray, steps: int, objective: dict):
    """J, dJ/df and dJ/dq0 of the discrete trajectory, exact to rounding (whole trajectory kept)."""
    cfg = S.cfg
    Q = [np.asfortranarray(q0.copy())]
    for nt in range(1, steps + 1):
        Q.append(loop_step(S, Q[-1], nt))
    plane = objective["kind"] == "plane_p2"

    def source(q):
        return O.objective_plane_p2(cfg, q, objective["normal"], objective["index"], objective["p_inf"])

    if plane:
        J = 0.0
        lam = np.zeros_like(q0)
        j, g = source(Q[steps])
        J += cfg.dt * j
        lam = lam + cfg.dt * g
    else:
        J, lam = O.terminal_objective(cfg, Q[steps], objective["kind"])
    gf = np.zeros_like(q0)
    for nt in range(steps, 0, -1):
        lam, f = step_vjp(S, Q[nt - 1], lam, nt)
        gf = gf + f
        if plane and nt - 1 >= 1:
            j, g = source(Q[nt - 1])
            J += cfg.dt * j
            lam = lam + cfg.dt * g
    return J, np.asfortranarray(gf), np.asfortranarray(lam)


# ------------------------------------------------------------------------------------------------
# optimisation loop of cruna.f90:78-179 with ls_quadratic_fit (line_search.f90:23-127)
# ------------------------------------------------------------------------------------------------
def optimize(S: O.Solver, q0: np.ndarray, steps: int, objective: dict, maxloop: int, ls_start: int,
             alpha0: float, f0: np.ndarray, discrete: bool = False):
    """Steepest descent on the time-constant forcing f: per loop the direct run and J, then (except in
    the last loop) the adjoint gradient, the quadratic line search over alpha in {0, alpha0/2, alpha0}
    (two more direct runs, dgesv of [alpha^2, alpha, 1] c = J; alpha = -c1 / (2 c0), capped at
    10 alpha0, alpha0 when the system is singular), and f <- f - alpha dJ/df.
    Returns (J per loop, alpha per loop except the last, final f)."""
    f = np.asfortranarray(f0.copy())
    Js, alphas = [], []
    for loop in range(1, maxloop + 1):
        S.force = f
        if loop == maxloop:
            Js.append(objective_value(S, q0, steps, objective))
            break
        if discrete:
            J, gf, _ = gradient_discrete(S, q0, steps, objective)
        else:
            J, gf, _ = O.gradient_store_all(S, q0, steps, objective)
        Js.append(J)
        alpha = alpha0
        if loop >= ls_start:
            a = np.array([0.0, 0.5, 1.0]) * alpha0
            Jl = [J]
            for ls in (1, 2):
                S.force = np.asfortranarray(f - a[ls] * gf)
                Jl.append(objective_value(S, q0, steps, objective))
            M = np.stack([a ** 2, a, np.ones(3)], axis=1)
            try:
                coef = np.linalg.solve(M, np.array(Jl))
                alpha = -coef[1] / (2.0 * coef[0])
                if alpha > 10.0 * alpha0:
                    alpha = 10.0 * alpha0
            except np.linalg.LinAlgError:
                alpha = alpha0
        alphas.append(alpha)
        f = np.asfortranarray(f - alpha * gf)
    S.force = f
    return np.array(Js), np.array(alphas), f
