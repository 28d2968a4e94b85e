"""CPU oracle for the CRUNA direct + adjoint Navier-Stokes time step (TEST INFRASTRUCTURE).

This module is test infrastructure, never the product: only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it.  The shipped path is the
CUDA library in ``public_b200/csrc`` and fails loudly when that library is missing.

It restates, in numpy, the algorithms of CRUNA (cruna-toolkit/public, Fortran 2003) that sit on the
direct and adjoint time step.  Every function cites the reference file:line it follows.  The
arithmetic order of the reference is kept where it matters for rounding (central differences are
formed as ``a*(f[i+1]-f[i-1]) + b*(f[i+2]-f[i-2])``, sums are left to right).

Third-party arithmetic: the compact cores call LAPACK ``dgttrf``/``dgttrs`` (reference links
MKL/OpenBLAS/AOCL, version not pinned).  The oracle calls the same LAPACK routines through
``scipy.linalg.lapack`` (scipy 1.18, bundled OpenBLAS), so pivots and multipliers are the ones
LAPACK produces.

Parity pinning: the reference cannot be compiled here (no Fortran compiler, MPI or HDF5) and its
only thresholded regression data (12 HDF5 snapshots of ``usr/unit_test/grid_transform_ns_and_euler``)
is absent from the source tree.  The oracle is therefore pinned by the known-answer properties the
reference's own unit tests check (``usr/unit_test/diff``: d/dx of 0 and 1 is 0, d/dx sin = cos at
design order; ``usr/unit_test/filter``: filter(1) = 1) and by identities of the equations
(NS with mu0 = 0 equals Euler, mass conservation on periodic grids), not by reference outputs.

Layout: a field is a Fortran-ordered array ``(n1, n2, n3)``; a state is ``(n1, n2, n3, 5)`` holding
``(rho, rho*u, rho*v, rho*w, p)`` as in ``src/data/data_rhs.f90:3-4`` and
``src/boundaries/nonreflecting.f90:48``.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np
from scipy.linalg import lapack

# ------------------------------------------------------------------------------------------------
# scheme names (the reference selects them at compile time through discretisation_x_core /
# filter_x_core selector modules, e.g. usr/unit_test/grid_transform_ns_and_euler/05_ns_pulse/
# discretisation_x_core.f90)
# ------------------------------------------------------------------------------------------------
DIFF_SCHEMES = (
    "empty",          # src/diff/diff_pen_core_empty.f90
    "o2_e_c_o",       # src/diff/diff_pen_core_o2_e_c_o.f90
    "o4_e_c_p",       # src/diff/diff_pen_core_o4_e_c_p.f90
    "o4_e_c_o",       # src/diff/diff_pen_core_o4_e_c_o.f90
    "o4_i_c_p_pade",  # src/diff/diff_pen_core_o4_i_c_p_pade.f90
    "o4_i_c_o_pade",  # src/diff/diff_pen_core_o4_i_c_o_pade.f90
    "o6_i_c_p",       # src/diff/diff_pen_core_o6_i_c_p.f90
    "o6_i_c_o",       # src/diff/diff_pen_core_o6_i_c_o.f90
    "o8_e_c_p",       # no reference counterpart: 8th-order explicit central, periodic
)
FILTER_SCHEMES = (
    "empty",          # src/filter/filter_pen_core_empty.f90
    "o2_i_c_p",       # src/filter/filter_pen_core_o2_i_c_p.f90
    "o6_i_c_p",       # src/filter/filter_pen_core_o6_i_c_p.f90
    "o2_i_c_o",       # src/filter/filter_pen_core_o2_i_c_o.f90
    "o4_i_c_o",       # src/filter/filter_pen_core_o4_i_c_o.f90
    "o6_i_c_o",       # src/filter/filter_pen_core_o6_i_c_o.f90
    "o8_i_c_o",       # src/filter/filter_pen_core_o8_i_c_o.f90
    "o10_i_c_o",      # src/filter/filter_pen_core_o10_i_c_o.f90
    "o10_e_c_p",      # no reference counterpart: 10th-order explicit periodic filter, blended
)
DIFF_PERIODIC = {"o4_e_c_p", "o4_i_c_p_pade", "o6_i_c_p", "o8_e_c_p"}


def diff_type(name: str) -> str:
    """'periodic' or 'open' as the ``diff_type`` parameter of each core module (e.g.
    src/diff/diff_pen_core_o4_e_c_p.f90:9, diff_pen_core_empty.f90:9)."""
    return "periodic" if name in DIFF_PERIODIC else "open"


# ------------------------------------------------------------------------------------------------
# LAPACK tridiagonal factors (the SAVE'd dl,dc,du,du2,ipiv of every compact core)
# ------------------------------------------------------------------------------------------------
@dataclasses.dataclass
class TriFactors:
    dl: np.ndarray
    d: np.ndarray
    du: np.ndarray
    du2: np.ndarray
    ipiv: np.ndarray          # 1-based, as LAPACK returns it
    fbnorm: Optional[np.ndarray] = None   # Sherman-Morrison correction (periodic cores)
    fbrat: float = 0.0

    def solve(self, b: np.ndarray) -> np.ndarray:
        """dgttrs('no transpose', n, nrhs, ...) on a (n, nrhs) array, then the cyclic correction
        ``q(:,i) = q(:,i) - fbnorm*(q(1,i) + fbrat*q(n1,i))`` (diff_pen_core_o6_i_c_p.f90:135-143)."""
        b = np.asfortranarray(b, dtype=np.float64)
        x, info = lapack.dgttrs(self.dl, self.d, self.du, self.du2, self.ipiv, b)
        if info != 0:
            raise RuntimeError(f"dgttrs info={info}")
        if self.fbnorm is not None:
            x = x - self.fbnorm[:, None] * (x[0:1, :] + self.fbrat * x[-1:, :])
        return x


def _dgttrf(dl, d, du) -> TriFactors:
    dl2, d2, du2_, du2, ipiv, info = lapack.dgttrf(np.array(dl, dtype=np.float64),
                                                   np.array(d, dtype=np.float64),
                                                   np.array(du, dtype=np.float64))
    if info != 0:
        raise RuntimeError(f"dgttrf info={info}")
    return TriFactors(dl2, d2, du2_, du2, ipiv)


def cyclic_factors(n: int, alpha: float, dc0: float) -> TriFactors:
    """Cyclic tridiagonal B (constant alpha off-diagonals, dc0 on the diagonal) reduced to a
    tridiagonal Btri plus a rank-one correction, as ``init_left_implicit_diff_part`` of
    src/diff/diff_pen_core_o6_i_c_p.f90:170-228 (also o4_i_c_p_pade.f90:167-225,
    filter_pen_core_o6_i_c_p.f90:184-249, o2_i_c_p, o2_i_c_o)."""
    dl = np.full(n - 1, alpha)
    dc = np.full(n, dc0)
    du = np.full(n - 1, alpha)
    fa = np.zeros(n)
    fb = np.zeros(n)
    fa[0] = -dc[0]
    fa[n - 1] = +alpha
    fb[0] = +1.0
    fb[n - 1] = -alpha / dc[0]
    dc[n - 1] = dc[n - 1] + (alpha * alpha / dc[0])
    dc[0] = dc[0] + dc[0]
    f = _dgttrf(dl, dc, du)
    y = f.solve(fa.reshape(n, 1))[:, 0]   # fbnorm is None here: plain dgttrs
    f.fbnorm = y * fb[0] / (1.0 + np.sum(fb * y))
    f.fbrat = fb[n - 1] / fb[0]
    return f


_FACTOR_CACHE: Dict[Tuple, TriFactors] = {}


def diff_factors(name: str, n: int) -> Optional[TriFactors]:
    key = ("diff", name, n)
    if key in _FACTOR_CACHE:
        return _FACTOR_CACHE[key]
    f = None
    if name == "o6_i_c_p":
        f = cyclic_factors(n, 1.0 / 3.0, 1.0)                    # o6_i_c_p.f90:195-226
    elif name == "o4_i_c_p_pade":
        f = cyclic_factors(n, 1.0 / 6.0, 2.0 / 3.0)              # o4_i_c_p_pade.f90:192-223
    elif name == "o6_i_c_o":                                     # o6_i_c_o.f90:180-197
        alpha = 1.0 / 3.0
        dl = np.full(n - 1, alpha)
        dc = np.full(n, 1.0)
        du = np.full(n - 1, alpha)
        du[0] = 3.00
        du[1] = 0.25
        du[n - 2] = 0.25
        dl[0] = 0.25
        dl[n - 2] = 3.00
        dl[n - 3] = 0.25
        f = _dgttrf(dl, dc, du)
    elif name == "o4_i_c_o_pade":                                # o4_i_c_o_pade.f90:168-182
        alpha = 1.0 / 6.0
        dl = np.full(n - 1, alpha)
        dc = np.full(n, 2.0 / 3.0)
        du = np.full(n - 1, alpha)
        dc[0] = 1.0 / 3.00
        dc[n - 1] = 1.0 / 3.00
        f = _dgttrf(dl, dc, du)
    _FACTOR_CACHE[key] = f
    return f


def filter_factors(name: str, n: int, alpha: float) -> Optional[TriFactors]:
    key = ("filter", name, n, float(alpha))
    if key in _FACTOR_CACHE:
        return _FACTOR_CACHE[key]
    f = None
    if name in ("o2_i_c_p", "o6_i_c_p", "o2_i_c_o"):
        f = cyclic_factors(n, alpha, 1.0)        # filter_pen_core_o6_i_c_p.f90:217-247
    elif name in ("o4_i_c_o", "o6_i_c_o", "o8_i_c_o", "o10_i_c_o"):
        dl = np.full(n - 1, alpha)               # filter_pen_core_o10_i_c_o.f90:284-294
        dc = np.full(n, 1.0)
        du = np.full(n - 1, alpha)
        du[0] = 0.0
        dl[n - 2] = 0.0
        f = _dgttrf(dl, dc, du)
    _FACTOR_CACHE[key] = f
    return f


# ------------------------------------------------------------------------------------------------
# derivative line cores: q is (n, m) with the derivative direction first ("fries"), returns q_x
# ------------------------------------------------------------------------------------------------
def _wrap(q: np.ndarray, s: int) -> np.ndarray:
    """q[i+s] with periodic wrap along axis 0."""
    return np.roll(q, -s, axis=0)


DIFF_MIN_POINTS = {"empty": 1, "o2_e_c_o": 4, "o4_e_c_p": 4, "o4_e_c_o": 6, "o4_i_c_p_pade": 3,
                   "o4_i_c_o_pade": 3, "o6_i_c_p": 5, "o6_i_c_o": 6, "o8_e_c_p": 8}


def diff_core(name: str, q: np.ndarray, dx: float) -> np.ndarray:
    q = np.asarray(q, dtype=np.float64)
    n = q.shape[0]
    if n < DIFF_MIN_POINTS[name]:
        raise ValueError(f"{name} needs at least {DIFF_MIN_POINTS[name]} points, got {n}")
    if name == "empty":
        # diff_pen_core_empty.f90:21 ``q = 0.0_rk * dx``; the reference builds with
        # -funsafe-math-optimizations, which folds 0*dx to 0 even for dx=inf (collapsed open direction)
        return np.zeros_like(q)
    if name == "o4_e_c_p":                       # diff_pen_core_o4_e_c_p.f90:68-80
        t = 8.0 * (_wrap(q, 1) - _wrap(q, -1)) - 1.0 * (_wrap(q, 2) - _wrap(q, -2))
        return t / (dx * 12.0)
    if name == "o8_e_c_p":                       # no reference counterpart (textbook 8th order)
        t = ((4.0 / 5.0) * (_wrap(q, 1) - _wrap(q, -1))
             + (-1.0 / 5.0) * (_wrap(q, 2) - _wrap(q, -2))
             + (4.0 / 105.0) * (_wrap(q, 3) - _wrap(q, -3))
             + (-1.0 / 280.0) * (_wrap(q, 4) - _wrap(q, -4)))
        return t / dx
    if name == "o4_e_c_o":                       # diff_pen_core_o4_e_c_o.f90:68-80
        t = np.empty_like(q)
        t[0] = -25.0 * q[0] + 48.0 * q[1] - 36.0 * q[2] + 16.0 * q[3] - 3.0 * q[4]
        t[1] = -3.0 * q[0] - 10.0 * q[1] + 18.0 * q[2] - 6.0 * q[3] + 1.0 * q[4]
        t[2:n - 2] = 8.0 * (q[3:n - 1] - q[1:n - 3]) - 1.0 * (q[4:n] - q[0:n - 4])
        t[n - 2] = -1.0 * q[n - 5] + 6.0 * q[n - 4] - 18.0 * q[n - 3] + 10.0 * q[n - 2] + 3.0 * q[n - 1]
        t[n - 1] = 3.0 * q[n - 5] - 16.0 * q[n - 4] + 36.0 * q[n - 3] - 48.0 * q[n - 2] + 25.0 * q[n - 1]
        return t / (dx * 12.0)
    if name == "o2_e_c_o":                       # diff_pen_core_o2_e_c_o.f90:68-80
        t = np.empty_like(q)
        t[0] = -1.5 * q[0] + 2.0 * q[1] - 0.5 * q[2]
        t[1] = -0.5 * q[0] + 0.5 * q[2]
        t[2:n - 2] = 0.5 * (q[3:n - 1] - q[1:n - 3])
        t[n - 2] = -0.5 * q[n - 3] + 0.5 * q[n - 1]
        t[n - 1] = +0.5 * q[n - 3] - 2.0 * q[n - 2] + 1.5 * q[n - 1]
        return t / dx
    if name == "o6_i_c_p":                       # diff_pen_core_o6_i_c_p.f90:115-143, stencil :160-162
        a = 14.00 / 9.0 / 2.0
        b = 1.00 / 9.0 / 4.0
        t = a * (_wrap(q, 1) - _wrap(q, -1)) + b * (_wrap(q, 2) - _wrap(q, -2))
        return diff_factors(name, n).solve(t / dx)
    if name == "o4_i_c_p_pade":                  # diff_pen_core_o4_i_c_p_pade.f90:115-141, :158
        a = 1.0 / 2.0
        t = a * (_wrap(q, 1) - _wrap(q, -1))
        return diff_factors(name, n).solve(t / dx)
    if name == "o6_i_c_o":                       # diff_pen_core_o6_i_c_o.f90:105-129, :148-153
        a = 14.00 / 9.0 / 2.0
        b = 1.00 / 9.0 / 4.0
        c = 17.00 / 6.0
        d = 1.50
        e = 1.00 / 6.0
        f = 0.75
        t = np.empty_like(q)
        t[0] = -c * q[0] + d * (q[1] + q[2]) - e * q[3]
        t[1] = -f * q[0] + f * q[2]
        t[2:n - 2] = a * (q[3:n - 1] - q[1:n - 3]) + b * (q[4:n] - q[0:n - 4])
        t[n - 2] = f * q[n - 1] - f * q[n - 3]
        t[n - 1] = c * q[n - 1] - d * (q[n - 2] + q[n - 3]) + e * q[n - 4]
        return diff_factors(name, n).solve(t / dx)
    if name == "o4_i_c_o_pade":                  # diff_pen_core_o4_i_c_o_pade.f90:104-124, :140
        a = 1.0 / 2.0
        t = np.empty_like(q)
        t[0] = -a * q[0] + a * (q[1])
        t[1:n - 1] = a * (q[2:n] - q[0:n - 2])
        t[n - 1] = a * q[n - 1] - a * (q[n - 2])
        return diff_factors(name, n).solve(t / dx)
    raise ValueError(f"unknown diff scheme {name}")


# ------------------------------------------------------------------------------------------------
# filter line cores
# ------------------------------------------------------------------------------------------------
def filter_interior_coeffs(name: str, alpha: float) -> List[float]:
    """Interior stencil a0..ar of the Gaitonde-Visbal filters, already halved as in the reference
    (e.g. filter_pen_core_o10_i_c_o.f90:182-199, o6_i_c_p.f90:167-178)."""
    if name in ("o2_i_c_p", "o2_i_c_o"):
        a0 = 1.0 / 2.0 + alpha
        a1 = (1.0 / 2.0 + alpha) / 2.0
        return [a0, a1]
    if name == "o4_i_c_o":
        a0 = 5.0 / 8.0 + 3.0 * alpha / 4.0
        a1 = (1.0 / 2.0 + alpha) / 2.0
        a2 = (-1.0 / 8.0 + alpha / 4.0) / 2.0
        return [a0, a1, a2]
    if name in ("o6_i_c_p", "o6_i_c_o"):
        a0 = 11.0 / 16.0 + 5.0 * alpha / 8.0
        a1 = (15.0 / 32.0 + 17.0 * alpha / 16.0) / 2.0
        a2 = (-3.0 / 16.0 + 3.0 * alpha / 8.0) / 2.0
        a3 = (1.0 / 32.0 - 1.0 * alpha / 16.0) / 2.0
        return [a0, a1, a2, a3]
    if name == "o8_i_c_o":
        a0 = 93.0 / 128.0 + 70.0 * alpha / 128.0
        a1 = (7.0 / 16.0 + 18.0 * alpha / 16.0) / 2.0
        a2 = (-7.0 / 32.0 + 14.0 * alpha / 32.0) / 2.0
        a3 = (1.0 / 16.0 - 1.0 * alpha / 8.0) / 2.0
        a4 = (-1.0 / 128.0 + 1.0 * alpha / 64.0) / 2.0
        return [a0, a1, a2, a3, a4]
    if name in ("o10_i_c_o", "o10_e_c_p"):
        a0 = 193.0 / 256.0 + 126.0 * alpha / 256.0
        a1 = (105.0 / 256.0 + 302.0 * alpha / 256.0) / 2.0
        a2 = (-15.0 / 64.0 + 30.0 * alpha / 64.0) / 2.0
        a3 = (45.0 / 512.0 - 90.0 * alpha / 512.0) / 2.0
        a4 = (-5.0 / 256.0 + 10.0 * alpha / 256.0) / 2.0
        a5 = (1.0 / 512.0 - 2.0 * alpha / 512.0) / 2.0
        return [a0, a1, a2, a3, a4, a5]
    raise ValueError(name)


def filter_boundary_coeffs(name: str, alpha: float) -> np.ndarray:
    """One-sided rows for points 2..(r+1) of the open filters (coefficients_for_boundary)."""
    al = alpha
    if name == "o4_i_c_o":                       # filter_pen_core_o4_i_c_o.f90
        return np.array([[1.0 / 16.0 + 7.0 * al / 8.0, 3.0 / 4.0 + 1.0 * al / 2.0, 3.0 / 8.0 + 1.0 * al / 4.0,
                          -1.0 / 4.0 + 1.0 * al / 2.0, 1.0 / 16.0 - 1.0 * al / 8.0]])
    if name == "o6_i_c_o":                       # filter_pen_core_o6_i_c_o.f90
        return np.array([
            [1.0 / 64.0 + 31.0 * al / 32.0, 29.0 / 32.0 + 3.0 * al / 16.0, 15.0 / 64.0 + 17.0 * al / 32.0,
             -5.0 / 16.0 + 5.0 * al / 8.0, 15.0 / 64.0 - 15.0 * al / 32.0, -3.0 / 32.0 + 3.0 * al / 16.0,
             1.0 / 64.0 - 1.0 * al / 32.0],
            [-1.0 / 64.0 + 1.0 * al / 32.0, 3.0 / 32.0 + 13.0 * al / 16.0, 49.0 / 64.0 + 15.0 * al / 32.0,
             5.0 / 16.0 + 3.0 * al / 8.0, -15.0 / 64.0 + 15.0 * al / 32.0, 3.0 / 32.0 - 3.0 * al / 16.0,
             -1.0 / 64.0 + 1.0 * al / 32.0]])
    if name == "o8_i_c_o":                       # filter_pen_core_o8_i_c_o.f90
        return np.array([
            [1.0 / 256.0 + 127.0 * al / 128.0, 31.0 / 32.0 + 1.0 * al / 16.0, 7.0 / 64.0 + 25.0 * al / 32.0,
             -7.0 / 32.0 + 7.0 * al / 16.0, 35.0 / 128.0 - 70.0 * al / 128.0, -7.0 / 32.0 + 7.0 * al / 16.0,
             7.0 / 64.0 - 7.0 * al / 32.0, -1.0 / 32.0 + 1.0 * al / 16.0, 1.0 / 256.0 - 1.0 * al / 128.0],
            [-1.0 / 256.0 + 1.0 * al / 128.0, 1.0 / 32.0 + 15.0 * al / 16.0, 57.0 / 64.0 + 7.0 * al / 32.0,
             7.0 / 32.0 + 9.0 * al / 16.0, -35.0 / 128.0 + 70.0 * al / 128.0, 7.0 / 32.0 - 7.0 * al / 16.0,
             -7.0 / 64.0 + 7.0 * al / 32.0, 1.0 / 32.0 - 1.0 * al / 16.0, -1.0 / 256.0 + 1.0 * al / 128.0],
            [1.0 / 256.0 - 1.0 * al / 128.0, -1.0 / 32.0 + 1.0 * al / 16.0, 7.0 / 64.0 + 25.0 * al / 32.0,
             25.0 / 32.0 + 7.0 * al / 16.0, 35.0 / 128.0 + 29.0 * al / 64.0, -7.0 / 32.0 + 7.0 * al / 16.0,
             7.0 / 64.0 - 7.0 * al / 32.0, -1.0 / 32.0 + 1.0 * al / 16.0, 1.0 / 256.0 - 1.0 * al / 128.0]])
    if name == "o10_i_c_o":                      # filter_pen_core_o10_i_c_o.f90:201-251
        return np.array([
            [1.0 / 1024.0 + 1022.0 * al / 1024.0, 507.0 / 512.0 + 10.0 * al / 512.0,
             45.0 / 1024.0 + 934.0 * al / 1024.0, -15.0 / 128.0 + 30.0 * al / 128.0,
             105.0 / 512.0 - 210.0 * al / 512.0, -63.0 / 256.0 + 126.0 * al / 256.0,
             105.0 / 512.0 - 210.0 * al / 512.0, -15.0 / 128.0 + 30.0 * al / 128.0,
             45.0 / 1024.0 - 90.0 * al / 1024.0, -5.0 / 512.0 + 10.0 * al / 512.0,
             1.0 / 1024.0 - 2.0 * al / 1024.0],
            [-1.0 / 1024.0 + 2.0 * al / 1024.0, 5.0 / 512.0 + 502.0 * al / 512.0,
             979.0 / 1024.0 + 90.0 * al / 1024.0, 15.0 / 128.0 + 98.0 * al / 128.0,
             -105.0 / 512.0 + 210.0 * al / 512.0, 63.0 / 256.0 - 126.0 * al / 256.0,
             -105.0 / 512.0 + 210.0 * al / 512.0, 15.0 / 128.0 - 30.0 * al / 128.0,
             -45.0 / 1024.0 + 90.0 * al / 1024.0, 5.0 / 512.0 - 10.0 * al / 512.0,
             -1.0 / 1024.0 + 2.0 * al / 1024.0],
            [1.0 / 1024.0 - 2.0 * al / 1024.0, -5.0 / 512.0 + 10.0 * al / 512.0,
             45.0 / 1024.0 + 934.0 * al / 1024.0, 113.0 / 128.0 + 30.0 * al / 128.0,
             105.0 / 512.0 + 302.0 * al / 512.0, -63.0 / 256.0 + 126.0 * al / 256.0,
             105.0 / 512.0 - 210.0 * al / 512.0, -15.0 / 128.0 + 30.0 * al / 128.0,
             45.0 / 1024.0 - 90.0 * al / 1024.0, -5.0 / 512.0 + 10.0 * al / 512.0,
             1.0 / 1024.0 - 2.0 * al / 1024.0],
            [-1.0 / 1024.0 + 2.0 * al / 1024.0, 5.0 / 512.0 - 10.0 * al / 512.0,
             -45.0 / 1024.0 + 90.0 * al / 1024.0, 15.0 / 128.0 + 98.0 * al / 128.0,
             407.0 / 512.0 + 210.0 * al / 512.0, 63.0 / 256.0 + 130.0 * al / 256.0,
             -105.0 / 512.0 + 210.0 * al / 512.0, 15.0 / 128.0 - 30.0 * al / 128.0,
             -45.0 / 1024.0 + 90.0 * al / 1024.0, 5.0 / 512.0 - 10.0 * al / 512.0,
             -1.0 / 1024.0 + 2.0 * al / 1024.0]])
    raise ValueError(name)


def _sym_stencil(q: np.ndarray, c: Sequence[float], lo: int, hi: int) -> np.ndarray:
    """a0*q(i) + a1*(q(i+1)+q(i-1)) + ... for i in [lo, hi) (no wrap), left-to-right sum."""
    t = c[0] * q[lo:hi]
    for m in range(1, len(c)):
        t = t + c[m] * (q[lo + m:hi + m] + q[lo - m:hi - m])
    return t


def filter_core(name: str, q: np.ndarray, alpha: float, strength: float = 0.2) -> np.ndarray:
    q = np.asarray(q, dtype=np.float64)
    n = q.shape[0]
    if name == "empty":                          # filter_pen_core_empty.f90: q = q
        return q.copy()
    c = filter_interior_coeffs(name, alpha if name != "o10_e_c_p" else 0.0)
    r = len(c) - 1
    if n < 2 * r + 1:
        raise ValueError(f"filter {name} needs at least {2 * r + 1} points, got {n}")
    if name in ("o2_i_c_p", "o6_i_c_p", "o10_e_c_p"):
        # periodic: interior formula with wrap (filter_pen_core_o6_i_c_p.f90:116-129)
        t = c[0] * q
        for m in range(1, r + 1):
            t = t + c[m] * (_wrap(q, m) + _wrap(q, -m))
        if name == "o10_e_c_p":
            # no reference counterpart: explicit (alpha = 0) 10th-order filter blended with strength s
            return q - strength * (q - t)
        return filter_factors(name, n, alpha).solve(t)
    t = np.empty_like(q)
    t[r:n - r] = _sym_stencil(q, c, r, n - r)
    t[0] = q[0]                                  # "do nothing at the boundary points" (o10:119-120)
    t[n - 1] = q[n - 1]
    if name != "o2_i_c_o":
        bc = filter_boundary_coeffs(name, alpha)
        w = bc.shape[1]
        for row in range(bc.shape[0]):           # points 2..r+1 and mirrors (o10:122-148)
            a = np.zeros_like(q[0])
            b = np.zeros_like(q[0])
            for i in range(w):
                a = a + bc[row, i] * q[i]
                b = b + bc[row, i] * q[n - 1 - i]
            t[1 + row] = a
            t[n - 2 - row] = b
    f = filter_factors(name, n, alpha)
    return f.solve(t)


# ------------------------------------------------------------------------------------------------
# configuration (the parameter.dat keys on the hot path, src/parameter/parameter.f90:100-170)
# ------------------------------------------------------------------------------------------------
@dataclasses.dataclass
class Config:
    n: Tuple[int, int, int]
    x0: Tuple[float, float, float] = (0.0, 0.0, 0.0)      # geom.x10, x20, x30
    x1: Tuple[float, float, float] = (1.0, 1.0, 1.0)      # geom.x11, x21, x31
    diff: Tuple[str, str, str] = ("o4_e_c_p", "o4_e_c_p", "o4_e_c_p")
    filt: Tuple[str, str, str] = ("empty", "empty", "empty")
    alpha: float = 0.35                                   # filter.alpha
    strength: float = 0.2                                 # o10_e_c_p blend strength
    di_freq: Tuple[int, int, int] = (2**31 - 1,) * 3      # filter.di{1,2,3}freq
    ai_freq: Tuple[int, int, int] = (2**31 - 1,) * 3      # filter.ai{1,2,3}freq
    gamma: float = 1.4                                    # material.gamma
    R: float = 8.3144598                                  # material.R (parameter.f90:160)
    W: float = 0.0289647                                  # material.W (ns_rho_rhou_p_trafos.f90:24)
    mu0: float = 0.0                                      # material.mu0
    T0: float = 273.0                                     # material.T0 (trafos.f90:133)
    Pr: float = 0.71                                      # material.Pr (trafos.f90:159)
    dt: float = 1e-3                                      # time.dt
    heat_flux_dx: bool = False   # False: reference behaviour, heat-flux Dx calls without h (dx=1)
    bc: Optional[np.ndarray] = None   # rows (type, is, ie, js, je, ks, ke, k1, k2, k3), 1-based
    sponge_length: Tuple[float, float, float] = (0.3, 0.3, 0.3)
    sponge_amplitude: float = 1.0
    sponge_shape: str = "quadratic"
    kvector: str = "diagonal"         # sponge.kvector: diagonal, orthogonal, hedgehog (zonal BC types)

    @property
    def npts(self) -> int:
        return self.n[0] * self.n[1] * self.n[2]

    def dx(self) -> Tuple[float, float, float]:
        """Grid spacing: periodic dx = L/n, open dx = L/(n-1) (src/geometry/grid_transform.f90:40-56)."""
        out = []
        for d in range(3):
            L = self.x1[d] - self.x0[d]
            m = self.n[d] if diff_type(self.diff[d]) == "periodic" else self.n[d] - 1
            out.append(L / m if m != 0 else math.inf)
        return tuple(out)

    def grid(self) -> List[np.ndarray]:
        """1-D grid vectors x_i = x0 + (i-1)*dx (grid_transform.f90:60-120; collapsed dims stay x0)."""
        dx = self.dx()
        out = []
        for d in range(3):
            if self.n[d] > 1:
                x = np.arange(self.n[d], dtype=np.float64) * dx[d]
            else:
                x = np.zeros(1)
            out.append(x + self.x0[d])
        return out

    def cp(self) -> float:
        return self.gamma * (self.R / self.W) / (self.gamma - 1.0)


# ------------------------------------------------------------------------------------------------
# directional operators Dx_d and filter_i_d (transpose -> core -> back-transpose)
# ------------------------------------------------------------------------------------------------
def _along(f: np.ndarray, d: int, fn: Callable[[np.ndarray], np.ndarray]) -> np.ndarray:
    g = np.moveaxis(f, d, 0)
    shp = g.shape
    r = fn(np.ascontiguousarray(g).reshape(shp[0], -1)).reshape(shp)
    return np.asfortranarray(np.moveaxis(r, 0, d))


def Dx(cfg: Config, d: int, f: np.ndarray, h: Optional[float] = None) -> np.ndarray:
    """Dx1/Dx2/Dx3 of one field; ``h`` defaults to 1.0 as in diff_i1_mpi_cartesian.f90:93-97."""
    dx = 1.0 if h is None else h
    return _along(f, d, lambda L: diff_core(cfg.diff[d], L, dx))


def filter_dir(cfg: Config, d: int, q: np.ndarray) -> np.ndarray:
    """filter_i1/2/3 of a state: loop over variables (filter_i1_mpi_cartesian.f90:83-97)."""
    out = np.empty_like(q)
    for v in range(q.shape[3]):
        out[..., v] = _along(q[..., v], d, lambda L: filter_core(cfg.filt[d], L, cfg.alpha, cfg.strength))
    return out


# ------------------------------------------------------------------------------------------------
# thermodynamics (src/equations/ns_rho_rhou_p_trafos.f90)
# ------------------------------------------------------------------------------------------------
def give_T(cfg: Config, q: np.ndarray) -> np.ndarray:
    return (cfg.W / cfg.R) * q[..., 4] / q[..., 0]                        # trafos.f90:51,57


def give_mu(cfg: Config, T: np.ndarray) -> np.ndarray:
    S1 = 110.4                                                              # trafos.f90:124
    return cfg.mu0 * (T / cfg.T0) ** 1.5 * ((cfg.T0 + S1) / (T + S1))      # trafos.f90:140


def give_lambda(cfg: Config, mu: np.ndarray) -> np.ndarray:
    return mu * cfg.cp() / cfg.Pr                                           # trafos.f90:163-169


def give_c(cfg: Config, q: np.ndarray) -> np.ndarray:
    return np.sqrt(cfg.gamma * q[..., 4] / q[..., 0])                      # trafos.f90:73


# ------------------------------------------------------------------------------------------------
# sponge shape (src/boundaries/shape_functions.f90:69-150)
# ------------------------------------------------------------------------------------------------
def sponge_shape_1d(cfg: Config) -> List[Tuple[np.ndarray, np.ndarray]]:
    """Per-direction (minus-side, plus-side) ramp factors.  A direction with length <= 0 has no
    sponge (factor 1); the reference would evaluate 0/0 there (no counterpart)."""
    out = []
    X = cfg.grid()
    for d in range(3):
        x = X[d]
        L = cfg.sponge_length[d]
        if L <= 0.0:
            out.append((np.ones_like(x), np.ones_like(x)))
            continue

        def fct(xx, x0):
            if cfg.sponge_shape == "quadratic":
                return 1.0 - ((xx - x0) / L) ** 2                          # :51
            pi = 4.0 * math.atan(1.0)
            return 0.5 + 0.5 * np.cos((xx - x0) * (pi / L))                 # :64

        x0 = cfg.x0[d] + L
        sm = fct(x, x0)
        sm = np.where(x > x0, 1.0, sm)
        x0 = cfg.x1[d] - L
        sp = fct(x, x0)
        sp = np.where(x < x0, 1.0, sp)
        out.append((sm, sp))
    return out


def sponge_shape(cfg: Config) -> np.ndarray:
    s = sponge_shape_1d(cfg)
    n1, n2, n3 = cfg.n
    phi = (s[0][0] * s[0][1])[:, None, None] * np.ones((1, n2, n3))          # xm*xp
    phi = phi * s[1][0][None, :, None]                                         # *ym
    phi = phi * s[1][1][None, :, None]                                         # *yp
    phi = phi * s[2][0][None, None, :]                                         # *zm
    phi = phi * s[2][1][None, None, :]                                         # *zp
    phi = 1.0 - phi                                                            # :142
    return np.asfortranarray(cfg.sponge_amplitude * phi)                       # :145


# ------------------------------------------------------------------------------------------------
# boundary conditions (src/boundaries/boundary_conditions.f90, nonreflecting.f90, sponge_layer_core.f90)
# ------------------------------------------------------------------------------------------------
def _box(row) -> Tuple[slice, slice, slice]:
    is_, ie, js, je, ks, ke = (int(round(v)) for v in row[1:7])
    return slice(is_ - 1, ie), slice(js - 1, je), slice(ks - 1, ke)


def kvector_field(cfg: Config) -> np.ndarray:
    """Boundary normal vectors (n1, n2, n3, 3) of the zonal BC types: init_orthogonal_and_diagonal_kvector,
    init_orthogonal_kvector, init_hedgehog_kvector and normalize_kvector (boundary_normal_vector.f90:37-261)."""
    x = cfg.grid()
    L = [cfg.x1[d] - cfg.x0[d] for d in range(3)]
    X = np.meshgrid(*x, indexing="ij")
    k = np.stack([X[d] - (cfg.x0[d] + 0.5 * L[d]) for d in range(3)], axis=-1)
    if cfg.kvector == "hedgehog":
        return k / np.sqrt(np.sum(k ** 2, axis=-1))[..., None]
    k = k / np.array(L)
    dx = cfg.dx()
    half = 0.5 * min(dx[d] / L[d] for d in range(3))
    a = np.abs(k)
    m = a.max(axis=-1)
    dom = np.where(m == a[..., 0], 0, np.where(m == a[..., 1], 1, 2))
    out = np.zeros_like(k)
    for d in range(3):
        sgn = np.copysign(1.0, k[..., d])
        keep = (dom == d)
        if cfg.kvector == "diagonal":
            keep = keep | (m - a[..., d] < half)
        out[..., d] = np.where(keep, sgn, 0.0)
    if cfg.kvector == "diagonal":
        out = out / np.sqrt(np.sum(out ** 2, axis=-1))[..., None]
    return out


def characteristic_q_k1d(cfg: Config, q: np.ndarray, aim: np.ndarray, kvec, shape=None) -> np.ndarray:
    """nonreflecting.f90:46-137 on a box (q, aim have shape (..., 5)); returns the new q.  With kvec of
    shape (..., 3) and an optional shape factor this is characteristic_q_k4d (:141-233)."""
    r = q[..., 0]
    u = q[..., 1:4] / r[..., None]
    p = q[..., 4]
    c = np.sqrt(cfg.gamma * q[..., 4] / q[..., 0])
    dq = np.empty_like(q)
    dq[..., 0] = aim[..., 0] - r
    dq[..., 1:4] = aim[..., 1:4] / aim[..., 0:1] - u
    dq[..., 4] = aim[..., 4] - p
    if shape is not None:
        dq = dq * shape[..., None]
    kvec = np.asarray(kvec)
    kx, ky, kz = -kvec[..., 0], -kvec[..., 1], -kvec[..., 2]
    c2 = c ** 2
    R1 = kx * dq[..., 0] + kz * dq[..., 2] - ky * dq[..., 3] - kx * dq[..., 4] / c2
    R2 = ky * dq[..., 0] - kz * dq[..., 1] + kx * dq[..., 3] - ky * dq[..., 4] / c2
    R3 = kz * dq[..., 0] + ky * dq[..., 1] - kx * dq[..., 2] - kz * dq[..., 4] / c2
    R4 = kx * dq[..., 1] + ky * dq[..., 2] + kz * dq[..., 3] + dq[..., 4] / (r * c)
    R5 = -kx * dq[..., 1] - ky * dq[..., 2] - kz * dq[..., 3] + dq[..., 4] / (r * c)
    lamS = kx * u[..., 0] + ky * u[..., 1] + kz * u[..., 2]
    lamP = lamS + c
    lamM = lamS - c
    R1 = np.where(lamS < 0.0, 0.0, R1)
    R2 = np.where(lamS < 0.0, 0.0, R2)
    R3 = np.where(lamS < 0.0, 0.0, R3)
    R4 = np.where(lamP < 0.0, 0.0, R4)
    R5 = np.where(lamM < 0.0, 0.0, R5)
    d1 = kx * R1 + ky * R2 + kz * R3 + r / (2.0 * c) * R4 + r / (2.0 * c) * R5
    d2 = -kz * R2 + ky * R3 + 0.5 * kx * R4 - 0.5 * kx * R5
    d3 = kz * R1 - kx * R3 + 0.5 * ky * R4 - 0.5 * ky * R5
    d4 = -ky * R1 + kx * R2 + 0.5 * kz * R4 - 0.5 * kz * R5
    d5 = +0.5 * r * c * R4 + 0.5 * r * c * R5
    r = r + d1
    u0 = u[..., 0] + d2
    u1 = u[..., 1] + d3
    u2 = u[..., 2] + d4
    p = p + d5
    out = np.empty_like(q)
    out[..., 0] = r
    out[..., 1] = r * u0
    out[..., 2] = r * u1
    out[..., 3] = r * u2
    out[..., 4] = p
    return out


def characteristic_rhs_k1d(cfg: Config, rhs, q, aim, kvec, shape=None) -> np.ndarray:
    """nonreflecting.f90:237-341 without shape (BC type 204); with kvec (..., 3) and shape it is
    characteristic_rhs_k4d (:345-449, types 205 and 206)."""
    dt = cfg.dt
    inv_dt = 1.0 / dt
    r = q[..., 0]
    u = q[..., 1:4] / r[..., None]
    c = np.sqrt(cfg.gamma * q[..., 4] / q[..., 0])
    dq = np.empty_like(q)
    dq[..., 0] = aim[..., 0] - r
    dq[..., 1:4] = aim[..., 1:4] / aim[..., 0:1] - u
    dq[..., 4] = aim[..., 4] - q[..., 4]
    tmp = dt / r
    dq[..., 0] = dq[..., 0] + rhs[..., 0] * dt
    dq[..., 1] = dq[..., 1] + rhs[..., 1] * tmp
    dq[..., 2] = dq[..., 2] + rhs[..., 2] * tmp
    dq[..., 3] = dq[..., 3] + rhs[..., 3] * tmp
    dq[..., 4] = dq[..., 4] + rhs[..., 4] * dt
    kvec = np.asarray(kvec)
    kx, ky, kz = -kvec[..., 0], -kvec[..., 1], -kvec[..., 2]
    c2 = c ** 2
    R1 = kx * dq[..., 0] + kz * dq[..., 2] - ky * dq[..., 3] - kx * dq[..., 4] / c2
    R2 = ky * dq[..., 0] - kz * dq[..., 1] + kx * dq[..., 3] - ky * dq[..., 4] / c2
    R3 = kz * dq[..., 0] + ky * dq[..., 1] - kx * dq[..., 2] - kz * dq[..., 4] / c2
    R4 = kx * dq[..., 1] + ky * dq[..., 2] + kz * dq[..., 3] + dq[..., 4] / (r * c)
    R5 = -kx * dq[..., 1] - ky * dq[..., 2] - kz * dq[..., 3] + dq[..., 4] / (r * c)
    lamS = kx * u[..., 0] + ky * u[..., 1] + kz * u[..., 2]
    lamP = lamS + c
    lamM = lamS - c
    R1 = np.where(lamS < 0.0, 0.0, R1)
    R2 = np.where(lamS < 0.0, 0.0, R2)
    R3 = np.where(lamS < 0.0, 0.0, R3)
    R4 = np.where(lamP < 0.0, 0.0, R4)
    R5 = np.where(lamM < 0.0, 0.0, R5)
    d1 = kx * R1 + ky * R2 + kz * R3 + r / (2.0 * c) * R4 + r / (2.0 * c) * R5
    d2 = -kz * R2 + ky * R3 + 0.5 * kx * R4 - 0.5 * kx * R5
    d3 = kz * R1 - kx * R3 + 0.5 * ky * R4 - 0.5 * ky * R5
    d4 = -ky * R1 + kx * R2 + 0.5 * kz * R4 - 0.5 * kz * R5
    d5 = +0.5 * r * c * R4 + 0.5 * r * c * R5
    r = r + d1
    out = np.empty_like(rhs)
    if shape is not None:                                       # :428-435
        tmp = shape * inv_dt
        out[..., 0] = (1.0 - shape) * rhs[..., 0] + d1 * tmp
        out[..., 4] = (1.0 - shape) * rhs[..., 4] + d5 * tmp
        tmp = tmp * r
        out[..., 1] = (1.0 - shape) * rhs[..., 1] + d2 * tmp
        out[..., 2] = (1.0 - shape) * rhs[..., 2] + d3 * tmp
        out[..., 3] = (1.0 - shape) * rhs[..., 3] + d4 * tmp
        return out
    out[..., 0] = d1 * inv_dt
    tmp = inv_dt * r
    out[..., 1] = d2 * tmp
    out[..., 2] = d3 * tmp
    out[..., 3] = d4 * tmp
    out[..., 4] = d5 * inv_dt
    return out


def characteristic_qs_k1d(cfg: Config, qs, q, kvec, shape=None) -> np.ndarray:
    """nonreflecting.f90:453-554 (adjoint, target zero); with kvec (..., 3) and shape it is
    characteristic_qs_k4d (:558-661)."""
    ds = -qs
    if shape is not None:
        ds = ds * shape[..., None]
    kvec = np.asarray(kvec)
    kx, ky, kz = -kvec[..., 0], -kvec[..., 1], -kvec[..., 2]
    gm1 = cfg.gamma - 1.0
    c = np.sqrt(cfg.gamma * (q[..., 4] / q[..., 0]))
    g_c = gm1 / c
    u = q[..., 1] / q[..., 0]
    v = q[..., 2] / q[..., 0]
    w = q[..., 3] / q[..., 0]
    ku = kx * u + ky * v + kz * w
    kus = kx * ds[..., 1] + ky * ds[..., 2] + kz * ds[..., 3]
    ruus = (ds[..., 0] + u * ds[..., 1] + v * ds[..., 2] + w * ds[..., 3]) / c
    rups = ruus + ds[..., 4] / g_c
    S = ku < 0.0
    P = ku + c < 0.0
    M = ku - c < 0.0
    z = np.zeros_like(u)
    drs = np.where(S, ds[..., 0] + ku * kus, z)
    dus = np.where(S, ds[..., 1] - kx * kus, z)
    dvs = np.where(S, ds[..., 2] - ky * kus, z)
    dws = np.where(S, ds[..., 3] - kz * kus, z)
    dps = np.where(S, -g_c * ruus, z)
    tmp = 0.5 * (kus + rups)
    drs = np.where(P, drs - ku * tmp, drs)
    dus = np.where(P, dus + kx * tmp, dus)
    dvs = np.where(P, dvs + ky * tmp, dvs)
    dws = np.where(P, dws + kz * tmp, dws)
    dps = np.where(P, dps + g_c * tmp, dps)
    tmp = 0.5 * (kus - rups)
    drs = np.where(M, drs - ku * tmp, drs)
    dus = np.where(M, dus + kx * tmp, dus)
    dvs = np.where(M, dvs + ky * tmp, dvs)
    dws = np.where(M, dws + kz * tmp, dws)
    dps = np.where(M, dps - g_c * tmp, dps)
    out = np.empty_like(qs)
    out[..., 0] = qs[..., 0] + drs
    out[..., 1] = qs[..., 1] + dus
    out[..., 2] = qs[..., 2] + dvs
    out[..., 3] = qs[..., 3] + dws
    out[..., 4] = qs[..., 4] + dps
    return out


def _zonal_active(row, outside_rhs: bool) -> bool:
    """Type 203 inside / outside the RHS: column 8 = -1 applies outside only, 1 inside only
    (boundary_conditions.f90:96-107, :436-438)."""
    only = int(round(row[7]))
    return (only != 1) if outside_rhs else (only != -1)


def _zero_grad_shift(row) -> Tuple[int, int, int]:
    """characteristic_zero_grad_init (nonreflecting.f90:665-700): unit step towards the inside."""
    k = np.array(row[7:10], dtype=np.float64)
    k = k / np.sqrt(np.sum(k ** 2))
    return tuple(-1 if k[i] > 0 else (1 if k[i] < 0 else 0) for i in range(3))


class Solver:
    """The CRUNA hot path on one block: RHS, RK4, BCs, filters and the step loops."""

    def __init__(self, cfg: Config, qref: Optional[np.ndarray] = None,
                 force: Optional[np.ndarray] = None):
        self.cfg = cfg
        self.dx = cfg.dx()
        self.qref = qref
        self.force = force
        self.bc = np.zeros((0, 10)) if cfg.bc is None else np.asarray(cfg.bc, dtype=np.float64)
        need_shape = any(int(round(r[0])) in (203, 206, 400, 401) for r in self.bc)
        self.shape = sponge_shape(cfg) if need_shape else None
        zonal = any(int(round(r[0])) in (202, 203, 205, 206) for r in self.bc)
        self.kvec = kvector_field(cfg) if zonal else None
        for r in self.bc:
            t = int(round(r[0]))
            if t not in (0, 100, 200, 201, 202, 203, 204, 205, 206, 400, 401):
                raise NotImplementedError(f"boundary type {t} is not on this path")

    # --------------------------------------------------------------------------------------------
    def set_boundary_condition_q(self, q: np.ndarray, outside_rhs: bool = False) -> np.ndarray:
        """boundary_conditions.f90:52-136 (types 0,100,200,201,400,401)."""
        q = q.copy(order="F")
        for row in self.bc:
            t = int(round(row[0]))
            b = _box(row)
            if t == 200:
                sh = _zero_grad_shift(row)
                b2 = tuple(slice(s.start + o, s.stop + o) for s, o in zip(b, sh))
                q[b] = characteristic_q_k1d(self.cfg, q[b], q[b2], row[7:10])
            elif t == 201:
                q[b] = characteristic_q_k1d(self.cfg, q[b], self.qref[b], row[7:10])
            elif t == 202:                                          # boundary_conditions.f90:89-91
                q[b] = characteristic_q_k1d(self.cfg, q[b], self.qref[b], self.kvec[b])
            elif t == 203 and _zonal_active(row, outside_rhs):     # :93-107, whole block
                q = characteristic_q_k1d(self.cfg, q, self.qref, self.kvec, self.shape)
            elif t == 401:
                for v in range(5):                                  # sponge_layer_core.f90:80-84
                    q[..., v] = q[..., v] - self.shape * (q[..., v] - self.qref[..., v])
        return q

    def set_boundary_condition_qs(self, qs, q, outside_rhs: bool = False) -> np.ndarray:
        """boundary_conditions.f90:140-224."""
        qs = qs.copy(order="F")
        for row in self.bc:
            t = int(round(row[0]))
            b = _box(row)
            if t == 200:
                sh = _zero_grad_shift(row)
                b2 = tuple(slice(s.start + o, s.stop + o) for s, o in zip(b, sh))
                qs[b] = characteristic_qs_k1d(self.cfg, qs[b], q[b2], row[7:10])
            elif t == 201:
                qs[b] = characteristic_qs_k1d(self.cfg, qs[b], q[b], row[7:10])
            elif t == 202:                                          # boundary_conditions.f90:176-179
                qs[b] = characteristic_qs_k1d(self.cfg, qs[b], q[b], self.kvec[b])
            elif t == 203 and _zonal_active(row, outside_rhs):     # :181-195
                qs = characteristic_qs_k1d(self.cfg, qs, q, self.kvec, self.shape)
            elif t == 401:
                for v in range(5):                                  # sponge_layer_core.f90:163-165
                    qs[..., v] = qs[..., v] - self.shape * qs[..., v]
        return qs

    def set_boundary_condition_rhs(self, rhs, q) -> np.ndarray:
        """boundary_conditions.f90:228-298 (types 100, 204, 400)."""
        rhs = rhs.copy(order="F")
        for row in self.bc:
            t = int(round(row[0]))
            b = _box(row)
            if t == 100:                                            # wall_boundary_conditions.f90:13-23
                comp = int(round(row[7]))
                rhs[b + (comp - 1,)] = 0.0
            elif t == 204:
                rhs[b] = characteristic_rhs_k1d(self.cfg, rhs[b], q[b], self.qref[b], row[7:10])
            elif t == 205:                                          # boundary_conditions.f90:272-274
                rhs[b] = characteristic_rhs_k1d(self.cfg, rhs[b], q[b], self.qref[b], self.kvec[b])
            elif t == 206:                                          # :276-279, whole block
                rhs = characteristic_rhs_k1d(self.cfg, rhs, q, self.qref, self.kvec, self.shape)
            elif t == 400:                                          # sponge_layer_core.f90:45-48
                for v in range(5):
                    rhs[..., v] = rhs[..., v] - self.shape * (q[..., v] - self.qref[..., v])
        return rhs

    def set_boundary_condition_rhss(self, rhss, qs, q=None) -> np.ndarray:
        """boundary_conditions.f90:302-377.  The NS adjoint calls it without q, which makes a type 400
        sponge a printed warning only (sponge_layer_core.f90:194-199)."""
        rhss = rhss.copy(order="F")
        for row in self.bc:
            t = int(round(row[0]))
            b = _box(row)
            if t == 100:
                comp = int(round(row[7]))
                rhss[b + (comp - 1,)] = 0.0
            elif t == 400 and q is not None:                        # sponge_layer_core.f90:107-151
                rho = q[..., 0]
                ui = q[..., 1:4] / rho[..., None]
                s = np.empty_like(qs)
                s[..., 0] = (1.0 * qs[..., 0] - ui[..., 0] / rho * qs[..., 1]
                             - ui[..., 1] / rho * qs[..., 2] - ui[..., 2] / rho * qs[..., 3])
                s[..., 1] = 1.0 / rho * qs[..., 1]
                s[..., 2] = 1.0 / rho * qs[..., 2]
                s[..., 3] = 1.0 / rho * qs[..., 3]
                s[..., 4] = (self.cfg.gamma - 1.0) * qs[..., 4]
                for v in range(5):
                    rhss[..., v] = rhss[..., v] + self.shape * s[..., v]
        return rhss

    # --------------------------------------------------------------------------------------------
    def rhs_direct(self, q_in: np.ndarray, t: float = 0.0) -> np.ndarray:
        """right_hand_side_direct_3d, src/equations/ns_rho_rhou_p.f90:31-253."""
        cfg = self.cfg
        d1, d2, d3 = self.dx
        D = lambda d, f, h=None: Dx(cfg, d, f, h)
        q = self.set_boundary_condition_q(q_in)                                # :89-92
        u = [q[..., 1] / q[..., 0], q[..., 2] / q[..., 0], q[..., 3] / q[..., 0]]   # :95-99
        u_x, u_y, u_z = D(0, u[0], d1), D(1, u[0], d2), D(2, u[0], d3)        # :102-112
        v_x, v_y, v_z = D(0, u[1], d1), D(1, u[1], d2), D(2, u[1], d3)
        w_x, w_y, w_z = D(0, u[2], d1), D(1, u[2], d2), D(2, u[2], d3)
        temp = give_T(cfg, q)                                                  # :115-116
        mu = give_mu(cfg, temp)
        mu_div = -(2.0 / 3.0 * mu * (u_x + v_y + w_z))                         # :118
        tau_11 = mu_div + 2 * mu * u_x
        tau_22 = mu_div + 2 * mu * v_y
        tau_33 = mu_div + 2 * mu * w_z
        tau_12 = mu * (u_y + v_x)
        tau_13 = mu * (u_z + w_x)
        tau_23 = mu * (v_z + w_y)
        rhs = np.zeros(q.shape, order="F")
        a_x, a_y, a_z = D(0, q[..., 1], d1), D(1, q[..., 2], d2), D(2, q[..., 3], d3)
        rhs[..., 0] = -a_x - a_y - a_z                                         # :131-135
        a_x = D(0, q[..., 1] * u[0], d1)                                        # :138-149
        a_y = D(1, q[..., 2] * u[0], d2)
        a_z = D(2, q[..., 3] * u[0], d3)
        p_x = D(0, q[..., 4], d1)
        rhs[..., 1] = -a_x - a_y - a_z - p_x
        a_x, a_y, a_z = D(0, tau_11, d1), D(1, tau_12, d2), D(2, tau_13, d3)
        rhs[..., 1] = rhs[..., 1] + a_x + a_y + a_z
        a_x = D(0, q[..., 1] * u[1], d1)                                        # :152-163
        a_y = D(1, q[..., 2] * u[1], d2)
        a_z = D(2, q[..., 3] * u[1], d3)
        p_y = D(1, q[..., 4], d2)
        rhs[..., 2] = -a_x - a_y - a_z - p_y
        a_x, a_y, a_z = D(0, tau_12, d1), D(1, tau_22, d2), D(2, tau_23, d3)
        rhs[..., 2] = rhs[..., 2] + a_x + a_y + a_z
        a_x = D(0, q[..., 1] * u[2], d1)                                        # :166-177
        a_y = D(1, q[..., 2] * u[2], d2)
        a_z = D(2, q[..., 3] * u[2], d3)
        p_z = D(2, q[..., 4], d3)
        rhs[..., 3] = -a_x - a_y - a_z - p_z
        a_x, a_y, a_z = D(0, tau_13, d1), D(1, tau_23, d2), D(2, tau_33, d3)
        rhs[..., 3] = rhs[..., 3] + a_x + a_y + a_z
        a_x = D(0, q[..., 4] * u[0], d1)                                        # :180-186
        a_y = D(1, q[..., 4] * u[1], d2)
        a_z = D(2, q[..., 4] * u[2], d3)
        gamma_term = cfg.gamma / (cfg.gamma - 1.0)
        rhs[..., 4] = gamma_term * (-a_x - a_y - a_z)
        rhs[..., 4] = rhs[..., 4] + u[0] * p_x + u[1] * p_y + u[2] * p_z
        hh = self.dx if cfg.heat_flux_dx else (None, None, None)               # :189-197 (no h)
        a_x, a_y, a_z = D(0, temp, hh[0]), D(1, temp, hh[1]), D(2, temp, hh[2])
        lam = give_lambda(cfg, mu)
        a_x = D(0, lam * a_x, hh[0])
        a_y = D(1, lam * a_y, hh[1])
        a_z = D(2, lam * a_z, hh[2])
        rhs[..., 4] = rhs[..., 4] + a_x + a_y + a_z                             # :200
        rhs[..., 4] = (rhs[..., 4] + tau_11 * u_x + tau_12 * u_y + tau_13 * u_z  # :204-206
                       + tau_12 * v_x + tau_22 * v_y + tau_23 * v_z
                       + tau_13 * w_x + tau_23 * w_y + tau_33 * w_z)
        rhs[..., 4] = (cfg.gamma - 1.0) * rhs[..., 4]                          # :208-209
        if self.force is not None:                                             # :212 apply_force
            rhs = rhs + self.force
        # :215 sponge(rhs,q,qref) is empty_sponge_inrhs_warning in src (sponge_layer.f90:15)
        return self.set_boundary_condition_rhs(rhs, q)                         # :218

    # --------------------------------------------------------------------------------------------
    def rhs_adjoint(self, qs_in, q, g, t: float = 0.0) -> np.ndarray:
        """right_hand_side_adjoint_3d, ns_rho_rhou_p.f90:257-536 (continuous inviscid adjoint)."""
        cfg = self.cfg
        D = lambda d, f: Dx(cfg, d, f, self.dx[d])
        qs = self.set_boundary_condition_qs(qs_in, q)                          # :287-290
        gm1 = cfg.gamma - 1.0
        gpr = cfg.gamma * q[..., 4] / (q[..., 0] * gm1)                        # :292-294
        inv_rho = 1.0 / q[..., 0]
        rhs = np.zeros(qs.shape, order="F")
        u1 = q[..., 1] / q[..., 0]
        u2 = q[..., 2] / q[..., 0]
        u3 = q[..., 3] / q[..., 0]
        # D_x1 part (:304-370)
        a, b, c, d, e = (D(0, qs[..., v]) for v in range(5))
        rhs[..., 0] = rhs[..., 0] + (u1 ** 2) * b + (u1 * u2) * c + (u1 * u3) * d + gpr * u1 * e
        rhs[..., 1] = rhs[..., 1] - a - 2.0 * u1 * b - u2 * c - u3 * d - gpr * e
        rhs[..., 2] = rhs[..., 2] - u1 * c
        rhs[..., 3] = rhs[..., 3] - u1 * d
        rhs[..., 4] = rhs[..., 4] - gm1 * b - cfg.gamma * u1 * e
        a = D(0, -u1 * qs[..., 4])
        rhs[..., 4] = rhs[..., 4] - gm1 * a
        a = D(0, q[..., 4])
        rhs[..., 0] = rhs[..., 0] + qs[..., 4] * u1 * inv_rho * a
        rhs[..., 1] = rhs[..., 1] - qs[..., 4] * inv_rho * a
        # D_x2 part (:380-440)
        a, b, c, d, e = (D(1, qs[..., v]) for v in range(5))
        rhs[..., 0] = rhs[..., 0] + (u2 * u1) * b + (u2 ** 2) * c + (u2 * u3) * d + gpr * u2 * e
        rhs[..., 1] = rhs[..., 1] - u2 * b
        rhs[..., 2] = rhs[..., 2] - a - u1 * b - 2 * u2 * c - u3 * d - gpr * e
        rhs[..., 3] = rhs[..., 3] - u2 * d
        rhs[..., 4] = rhs[..., 4] - gm1 * c - cfg.gamma * u2 * e
        a = D(1, -u2 * qs[..., 4])
        rhs[..., 4] = rhs[..., 4] - gm1 * a
        a = D(1, q[..., 4])
        rhs[..., 0] = rhs[..., 0] + qs[..., 4] * u2 * inv_rho * a
        rhs[..., 2] = rhs[..., 2] - qs[..., 4] * inv_rho * a
        # D_x3 part (:450-509)
        a, b, c, d, e = (D(2, qs[..., v]) for v in range(5))
        rhs[..., 0] = rhs[..., 0] + (u3 * u1) * b + (u3 * u2) * c + (u3 ** 2) * d + gpr * u3 * e
        rhs[..., 1] = rhs[..., 1] - u3 * b
        rhs[..., 2] = rhs[..., 2] - u3 * c
        rhs[..., 3] = rhs[..., 3] - a - u1 * b - u2 * c - 2 * u3 * d - gpr * e
        rhs[..., 4] = rhs[..., 4] - gm1 * d - cfg.gamma * u3 * e
        a = D(2, -u3 * qs[..., 4])
        rhs[..., 4] = rhs[..., 4] - gm1 * a
        a = D(2, q[..., 4])
        rhs[..., 0] = rhs[..., 0] + qs[..., 4] * u3 * inv_rho * a
        rhs[..., 3] = rhs[..., 3] - qs[..., 4] * inv_rho * a
        rhs = rhs + g                                                          # :512
        # :515 sponge_adjoint is empty_sponge_inrhs_warning (sponge_layer.f90:16)
        return self.set_boundary_condition_rhss(rhs, qs)                       # :518 (no q)

    # --------------------------------------------------------------------------------------------
    def time_stepper_direct(self, q0, t: float = 0.0) -> np.ndarray:
        """rk_o4_e.f90:17-58."""
        dt = self.cfg.dt
        dth = dt * 0.5
        k1 = self.rhs_direct(q0, t)
        k2 = self.rhs_direct(q0 + dth * k1, t + dth)
        k3 = self.rhs_direct(q0 + dth * k2, t + dth)
        k4 = self.rhs_direct(q0 + dt * k3, t + dt)
        return np.asfortranarray(q0 + dt / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4))

    def time_stepper_adjoint(self, qs0, q0, g, t: float = 0.0) -> np.ndarray:
        """rk_o4_e.f90:62-105 (dt -> -dt, direct state frozen)."""
        dt = -self.cfg.dt
        dth = -self.cfg.dt * 0.5
        k1 = self.rhs_adjoint(qs0, q0, g, t)
        k2 = self.rhs_adjoint(qs0 + dth * k1, q0, g, t + dth)
        k3 = self.rhs_adjoint(qs0 + dth * k2, q0, g, t + dth)
        k4 = self.rhs_adjoint(qs0 + dt * k3, q0, g, t + dt)
        return np.asfortranarray(qs0 + dt / 6.0 * (k1 + 2 * k2 + 2 * k3 + k4))

    def filter_i(self, d: int, q: np.ndarray) -> np.ndarray:
        return filter_dir(self.cfg, d, q)

    # --------------------------------------------------------------------------------------------
    def calc_direct(self, q0: np.ndarray, steps: int, store: bool = False, nt0: int = 0):
        """Loop body of calc_direct (src/main/computation_direct.f90:64-107): step, BC q outside the
        RHS, filters i1, i2, i3 when mod(nt, freq) == 0, keep Q(nt)."""
        cfg = self.cfg
        qn = np.asfortranarray(q0.copy())
        Q = [qn.copy()] if store else None
        for it in range(1, steps + 1):
            nt = nt0 + it
            t = nt * cfg.dt
            qn = self.time_stepper_direct(qn, t)
            qn = self.set_boundary_condition_q(qn, outside_rhs=True)
            for d in range(3):
                if nt % cfg.di_freq[d] == 0:
                    qn = self.filter_i(d, qn)
            if store:
                Q.append(qn.copy())
        return (qn, Q) if store else qn

    def calc_adjoint(self, qs0: np.ndarray, Q: Sequence[np.ndarray],
                     g_fn: Optional[Callable[[np.ndarray, int], np.ndarray]] = None):
        """Loop body of calc_adjoint (src/main/computation_adjoint.f90:60-108): backwards over nt,
        q0 = Q(nt), g = calc_objective_g(q0), adjoint step, BC qs outside, filters ai freq."""
        cfg = self.cfg
        steps = len(Q) - 1
        qsn = np.asfortranarray(qs0.copy())
        out = [None] * (steps + 1)
        out[steps] = qsn.copy()
        for nt in range(steps, 0, -1):
            t = nt * cfg.dt
            q0 = Q[nt]
            g = np.zeros_like(q0) if g_fn is None else g_fn(q0, nt)
            qsn = self.time_stepper_adjoint(qsn, q0, g, t)
            qsn = self.set_boundary_condition_qs(qsn, q0, outside_rhs=True)
            for d in range(3):
                if nt % cfg.ai_freq[d] == 0:
                    qsn = self.filter_i(d, qsn)
            out[nt - 1] = qsn.copy()
        return qsn, out


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """Relative L2 difference ||a-b|| / ||b||."""
    nb = float(np.linalg.norm(b.ravel()))
    return float(np.linalg.norm((a - b).ravel())) / (nb if nb > 0 else 1.0)


# ------------------------------------------------------------------------------------------------
# objectives and the gradient of CRUNA's optimisation loop (src/main/cruna.f90:78-179):
# calc_direct -> calc_objective -> calc_adjoint (with calc_objective_g as the adjoint source) ->
# calc_grad.  The reference leaves the objective and the gradient assembly to each case
# (src/opt/objective.f90:19-45, force.f90:41-45); these are the library's built-in choices.
# ------------------------------------------------------------------------------------------------
def plane_weight(cfg: Config, normal: int) -> float:
    """Area element of a grid plane with the given normal direction (0, 1, 2): product of the other
    two grid spacings (a collapsed direction contributes 1)."""
    dx = cfg.dx()
    w = 1.0
    for d in range(3):
        if d != normal and cfg.n[d] > 1:
            w *= dx[d]
    return w


def objective_plane_p2(cfg: Config, q: np.ndarray, normal: int, index: int, p_inf: float):
    """j(q) = sum over the plane x_normal = index (0-based) of w (p - p_inf)^2 and its gradient
    g = dj/dq (only the pressure component of the plane points is non-zero)."""
    w = plane_weight(cfg, normal)
    sl = [slice(None)] * 3
    sl[normal] = index
    p = q[..., 4][tuple(sl)]
    dp = p - p_inf
    j = float(np.sum(w * dp * dp))
    g = np.zeros_like(q)
    gp = g[..., 4]
    gp[tuple(sl)] = 2.0 * w * dp
    return j, g


def objective_kinetic_energy(cfg: Config, q: np.ndarray):
    """E(q) = sum dV * 0.5 |rho u|^2 / rho and dE/dq = dV * (-0.5|u|^2, u, v, w, 0)."""
    dx = cfg.dx()
    dV = 1.0
    for d in range(3):
        if cfg.n[d] > 1:
            dV *= dx[d]
    rho = q[..., 0]
    m2 = q[..., 1] ** 2 + q[..., 2] ** 2 + q[..., 3] ** 2
    E = float(np.sum(dV * 0.5 * m2 / rho))
    g = np.zeros_like(q)
    u = q[..., 1:4] / rho[..., None]
    g[..., 0] = dV * (-0.5 * np.sum(u * u, axis=-1))
    g[..., 1:4] = dV * u
    return E, g


def cell_volume(cfg: Config) -> float:
    """Volume element dV: product of the grid spacings of the non-collapsed directions."""
    dx = cfg.dx()
    dV = 1.0
    for d in range(3):
        if cfg.n[d] > 1:
            dV *= dx[d]
    return dV


def vorticity(cfg: Config, q: np.ndarray):
    """curl u with the solver's own derivative operators (Dx with h = dx; a collapsed direction's
    empty core contributes zero): (D_y w - D_z v, D_z u - D_x w, D_x v - D_y u)."""
    dx = cfg.dx()
    rho = q[..., 0]
    u = [np.asfortranarray(q[..., 1 + i] / rho) for i in range(3)]
    D = lambda d, f: Dx(cfg, d, f, dx[d])
    return (D(1, u[2]) - D(2, u[1]), D(2, u[0]) - D(0, u[2]), D(0, u[1]) - D(1, u[0])), u


def objective_enstrophy(cfg: Config, q: np.ndarray):
    """Z(q) = sum dV * 0.5 |curl u|^2 (discrete curl of the solver's derivative operators) and dZ/dq:
    dZ/du = dV curl^T(omega) with the transposed line operators, then through u_i = (rho u_i) / rho."""
    from . import discrete_adjoint as DA       # transposed operators (imported here: DA imports this module)
    dV = cell_volume(cfg)
    (wx, wy, wz), u = vorticity(cfg, q)
    Z = float(np.sum(dV * 0.5 * (wx * wx + wy * wy + wz * wz)))
    dx = cfg.dx()
    DT = lambda d, f: DA.DT(cfg, d, np.asfortranarray(f), dx[d])
    gu = [dV * (DT(2, wy) - DT(1, wz)), dV * (DT(0, wz) - DT(2, wx)), dV * (DT(1, wx) - DT(0, wy))]
    rho = q[..., 0]
    g = np.zeros_like(q)
    g[..., 0] = -(u[0] * gu[0] + u[1] * gu[1] + u[2] * gu[2]) / rho
    for i in range(3):
        g[..., 1 + i] = gu[i] / rho
    return Z, g


def terminal_objective(cfg: Config, q: np.ndarray, kind: str):
    """The final-time objectives: kinetic energy or enstrophy, value and gradient."""
    if kind == "kinetic_energy":
        return objective_kinetic_energy(cfg, q)
    if kind == "enstrophy":
        return objective_enstrophy(cfg, q)
    raise ValueError(f"unknown terminal objective {kind}")


def gradient_store_all(S: "Solver", q0: np.ndarray, steps: int, objective: dict):
    """J, dJ/df (time-constant forcing) and dJ/dq0 with the whole trajectory stored.

    objective = {"kind": "plane_p2", "normal": d, "index": i, "p_inf": p} gives
    J = sum_{nt=1..steps} dt * j(Q(nt)) with the adjoint source -dj/dq(Q(nt)) at adjoint step nt (the
    order of computation_adjoint.f90:66-81); {"kind": "kinetic_energy"} gives J = E(Q(steps)) with
    qs(T) = dE/dq, {"kind": "enstrophy"} J = Z(Q(steps)) with qs(T) = dZ/dq.  dJ/df = integral of qs dt (trapezoid over the adjoint trajectory), dJ/dq0 = qs(0).
    """
    cfg = S.cfg
    qT, Q = S.calc_direct(q0, steps, store=True)
    J = 0.0
    qs = np.zeros_like(q0)
    gfn = None
    if objective["kind"] == "plane_p2":
        def gfn(qq, nt):
            # rk_o4_e.f90:62-105 integrates dqs/dt = rhs_adjoint + g backwards: g = -dj/dq makes qs ~ dJ/dq
            return -objective_plane_p2(cfg, qq, objective["normal"], objective["index"], objective["p_inf"])[1]
        for nt in range(1, steps + 1):
            J += cfg.dt * objective_plane_p2(cfg, Q[nt], objective["normal"], objective["index"],
                                             objective["p_inf"])[0]
    else:
        J, qs = terminal_objective(cfg, Q[steps], objective["kind"])
    qs_end, traj = S.calc_adjoint(qs, Q, g_fn=gfn)
    gf = 0.5 * cfg.dt * traj[steps]
    for nt in range(steps - 1, 0, -1):
        gf = gf + cfg.dt * traj[nt]
    gf = gf + 0.5 * cfg.dt * traj[0]
    return J, np.asfortranarray(gf), qs_end


def max_states(s: int, t: int) -> int:
    """Most states rev() can reverse with s free snapshots and t sweeps: C(s+1+t, t) - 1."""
    return math.comb(s + 1 + t, t) - 1


def checkpoint_table(n: int, S: int):
    """Minimal number of direct steps to reverse m <= n states with s <= S free snapshots, and the
    first-checkpoint distance achieving it, searched within the binomial bounds."""
    W = S + 1
    cost = [[0] * W for _ in range(n + 1)]
    kbest = [[1] * W for _ in range(n + 1)]
    for s in range(W):
        for m in range(1, n + 1):
            if s == 0:
                cost[m][s] = m * (m + 1) // 2
                continue
            t = 0
            while max_states(s, t) < m:
                t += 1
            lo = max(1, m - max_states(s - 1, t))
            hi = min(m, max_states(s, t - 1) + 1)
            best, bk = None, lo
            for k in range(lo, hi + 1):
                v = k + cost[m - k][s - 1] + cost[k - 1][s]
                if best is None or v < best:
                    best, bk = v, k
            cost[m][s], kbest[m][s] = best, bk
    return cost, kbest


def treeverse_schedule(steps: int, slots: int):
    """Binomial checkpoint schedule to reverse `steps` time steps with `slots` snapshots (the state
    Q(0) occupies one of them).  The adjoint step nt consumes Q(nt), nt = steps .. 1.  rev(a, b, s)
    produces Q(b), ..., Q(a+1) from the stored Q(a) with s free slots: it advances to a checkpoint
    a + k, reverses the right part with s - 1 slots, runs the adjoint step at the checkpoint from its
    slot, then reverses the left part with s slots; k minimises the advanced steps.
    Returns (actions, direct steps advanced)."""
    if slots < 1:
        raise ValueError("need at least one snapshot slot (for the initial state)")
    S = min(slots - 1, steps)
    _, kbest = checkpoint_table(steps, S)
    acts = []

    def rec(a, b, s):
        n = b - a
        if n <= 0:
            return
        if s == 0:
            for nt in range(b, a, -1):
                acts.append(("restore", a))
                acts.append(("advance", a, nt))
                acts.append(("adjoint", nt))
            return
        m = a + kbest[n][s]
        acts.append(("restore", a))
        acts.append(("advance", a, m))
        acts.append(("store", m))
        rec(m, b, s - 1)
        acts.append(("restore", m))
        acts.append(("adjoint", m))
        acts.append(("free", m))
        rec(a, m - 1, s)

    rec(0, steps, S)
    advanced = sum(r[1] - r[0] for (k, *r) in acts if k == "advance")
    return acts, advanced
