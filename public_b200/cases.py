"""Seeded / analytic initial states for the workloads the solver is run on.

A state is a Fortran-ordered float64 array (n1, n2, n3, 5) holding (rho, rho*u, rho*v, rho*w, p).
Nondimensional cases map onto CRUNA's dimensional parameters with R = W = 1 (so T = p/rho),
T0 = the free-stream temperature and mu0 = rho*U*L/Re; Sutherland's constant stays 110.4 as in
src/equations/ns_rho_rhou_p_trafos.f90:124.

Each builder returns ``(settings, q0)`` where ``settings`` is a dict of solver settings (the same keys
as ``public_b200.cruna.Settings``) and ``q0`` the initial state.
"""
from __future__ import annotations

import math
from typing import Dict, Tuple

import numpy as np

GAMMA = 1.4
PR = 0.71


def _state(n1, n2, n3) -> np.ndarray:
    return np.zeros((n1, n2, n3, 5), order="F")


def _dt_cfl(q: np.ndarray, dx_min: float, cfl: float, gamma: float) -> float:
    """dt = CFL * dx_min / max(|u| + c) over the initial field (src/helper/check_state.f90 formula)."""
    rho = q[..., 0]
    u = np.sqrt((q[..., 1] ** 2 + q[..., 2] ** 2 + q[..., 3] ** 2)) / rho
    c = np.sqrt(gamma * q[..., 4] / rho)
    return cfl * dx_min / float(np.max(u + c))


def isentropic_vortex(n: int = 256, steps_cfl: float = 0.5, mach: float = 0.5, strength: float = 5.0,
                      reynolds: float = 1000.0) -> Tuple[Dict, np.ndarray]:
    """2-D isentropic vortex (radius 1, strength 5) advected at Mach 0.5 along x in the periodic box
    [-5,5]^2 on n x n x 1 points; 8th-order explicit differences, 10th-order explicit filter
    (strength 0.2) every step, z collapsed (empty derivative core)."""
    L = 10.0
    dx = L / n
    x = -5.0 + np.arange(n) * dx
    X, Y = np.meshgrid(x, x, indexing="ij")
    r2 = X ** 2 + Y ** 2
    g = GAMMA
    Tinf = 1.0
    cinf = math.sqrt(g * Tinf)
    uinf = mach * cinf
    f = np.exp(0.5 * (1.0 - r2))
    du = -strength / (2 * math.pi) * Y * f
    dv = strength / (2 * math.pi) * X * f
    T = Tinf - (g - 1.0) * strength ** 2 / (8.0 * g * math.pi ** 2) * f ** 2
    rho = T ** (1.0 / (g - 1.0))
    p = rho * T
    q = _state(n, n, 1)
    q[:, :, 0, 0] = rho
    q[:, :, 0, 1] = rho * (uinf + du)
    q[:, :, 0, 2] = rho * dv
    q[:, :, 0, 3] = 0.0
    q[:, :, 0, 4] = p
    settings = dict(
        n=(n, n, 1), x0=(-5.0, -5.0, 0.0), x1=(5.0, 5.0, 1.0),
        diff=("o8_e_c_p", "o8_e_c_p", "empty"), filt=("o10_e_c_p", "o10_e_c_p", "empty"),
        alpha=0.0, strength=0.2, di_freq=(1, 1, 1), gamma=g, R=1.0, W=1.0,
        mu0=1.0 * uinf * 1.0 / reynolds, T0=Tinf, Pr=PR,
        dt=_dt_cfl(q, dx, steps_cfl, g))
    return settings, q


def taylor_green(n: int = 256, mach: float = 0.1, reynolds: float = 1600.0, seed: int = 0,
                 noise: float = 1e-4, cfl: float = 0.5) -> Tuple[Dict, np.ndarray]:
    """3-D Taylor-Green vortex in the periodic box [0, 2pi]^3 on n^3 points at Mach 0.1, Re 1600; the
    density carries a 1e-4 relative N(0,1) perturbation drawn from numpy PCG64(seed)."""
    L = 2.0 * math.pi
    dx = L / n
    x = np.arange(n) * dx
    g = GAMMA
    rho0, U0 = 1.0, 1.0
    p0 = rho0 * U0 ** 2 / (g * mach ** 2)
    sx, cx = np.sin(x), np.cos(x)
    q = _state(n, n, n)
    rng = np.random.Generator(np.random.PCG64(seed))
    xi = rng.standard_normal((n, n, n)).reshape((n, n, n), order="F")
    rho = rho0 * (1.0 + noise * xi)
    u = U0 * sx[:, None, None] * cx[None, :, None] * cx[None, None, :]
    v = -U0 * cx[:, None, None] * sx[None, :, None] * cx[None, None, :]
    c2x = np.cos(2 * x)
    p = p0 + rho0 * U0 ** 2 / 16.0 * (c2x[:, None, None] + c2x[None, :, None]) * (c2x[None, None, :] + 2.0)
    q[..., 0] = rho
    q[..., 1] = rho * u
    q[..., 2] = rho * v
    q[..., 3] = 0.0
    q[..., 4] = p
    T0 = p0 / rho0
    settings = dict(
        n=(n, n, n), x0=(0.0, 0.0, 0.0), x1=(L, L, L),
        diff=("o8_e_c_p",) * 3, filt=("o10_e_c_p",) * 3, alpha=0.0, strength=0.2,
        di_freq=(1, 1, 1), gamma=g, R=1.0, W=1.0, mu0=rho0 * U0 * 1.0 / reynolds, T0=T0, Pr=PR,
        dt=_dt_cfl(q, dx, cfl, g))
    return settings, q


def gaussian_pulse(n=(60, 65, 70), steps_dt: float = 5e-05) -> Tuple[Dict, np.ndarray]:
    """Gaussian pressure pulse of usr/unit_test/grid_transform_ns_and_euler/05_ns_pulse
    (initial_condition.f90:15-59, parameter.dat): rho0 = 1.193847801511275, p0 = 101325,
    amplitude 0.1 (a default-real literal there, i.e. float32(0.1)), fwhm 10 grid cells,
    centre (3.14, 3.14, 3.14), domain [0, 6.283185307]^3, o4_e_c_o differences, non-reflecting
    type 201 boundaries on all six faces, mu0 = 0, dt = 5e-5."""
    n1, n2, n3 = n
    L = 6.283185307
    dxs = [L / (m - 1) for m in n]
    xs = [np.arange(m) * dxs[i] for i, m in enumerate(n)]
    rho0 = 1.193847801511275
    p0 = 101325.0
    g = 1.4
    sigma = 10.0 / 2.3548 * dxs[0]
    r2 = ((xs[0][:, None, None] - 3.14) ** 2 + (xs[1][None, :, None] - 3.14) ** 2
          + (xs[2][None, None, :] - 3.14) ** 2)
    q = _state(n1, n2, n3)
    p = p0 + float(np.float32(0.1)) * np.exp(-r2 / (2.0 * sigma ** 2))
    q[..., 4] = p
    q[..., 0] = rho0 * (p / p0) ** (1.0 / g)
    inf1, inf2, inf3 = n
    bc = np.array([
        [201, 1, 1, 1, inf2, 1, inf3, -1, 0, 0],
        [201, inf1, inf1, 1, inf2, 1, inf3, 1, 0, 0],
        [201, 1, inf1, 1, 1, 1, inf3, 0, -1, 0],
        [201, 1, inf1, inf2, inf2, 1, inf3, 0, 1, 0],
        [201, 1, inf1, 1, inf2, 1, 1, 0, 0, -1],
        [201, 1, inf1, 1, inf2, inf3, inf3, 0, 0, 1]], dtype=np.float64)
    settings = dict(
        n=n, x0=(0.0, 0.0, 0.0), x1=(L, L, L), diff=("o4_e_c_o",) * 3, filt=("empty",) * 3,
        alpha=0.0, gamma=g, R=8.3144598, W=0.0289647, mu0=0.0, T0=273.0, Pr=0.71, dt=steps_dt, bc=bc)
    return settings, q


def mixing_layer(n=(512, 384, 256), mach_c: float = 0.4, reynolds: float = 500.0, seed: int = 1,
                 noise: float = 1e-3, sponge_points: int = 20, cfl: float = 0.5,
                 y_scheme: str = "o6_i_c_o") -> Tuple[Dict, np.ndarray]:
    """Temporal mixing layer: tanh profile of thickness 1 in the box 80 x 60 x 40, periodic in x and z,
    open in y with type-201 characteristic boundaries and a sponge of ``sponge_points`` cells at both
    y ends; convective Mach 0.4 (velocity difference 2*Mc*c0); white-noise velocity seeding of
    amplitude 1e-3 from PCG64(seed)."""
    n1, n2, n3 = n
    Lx, Ly, Lz = 80.0, 60.0, 40.0
    g = GAMMA
    rho0, T0 = 1.0, 1.0
    p0 = rho0 * T0
    c0 = math.sqrt(g * T0)
    dU = 2.0 * mach_c * c0
    x = np.arange(n1) * (Lx / n1)
    y = -Ly / 2 + np.arange(n2) * (Ly / (n2 - 1))
    z = np.arange(n3) * (Lz / n3)
    rng = np.random.Generator(np.random.PCG64(seed))
    q = _state(n1, n2, n3)
    u = 0.5 * dU * np.tanh(y)[None, :, None] * np.ones((n1, 1, n3))
    u = u + noise * dU * rng.standard_normal((n1, n2, n3))
    v = noise * dU * rng.standard_normal((n1, n2, n3))
    w = noise * dU * rng.standard_normal((n1, n2, n3))
    q[..., 0] = rho0
    q[..., 1] = rho0 * u
    q[..., 2] = rho0 * v
    q[..., 3] = rho0 * w
    q[..., 4] = p0
    dy = Ly / (n2 - 1)
    bc = np.array([
        [201, 1, n1, 1, 1, 1, n3, 0, -1, 0],
        [201, 1, n1, n2, n2, 1, n3, 0, 1, 0],
        [400, 1, n1, 1, n2, 1, n3, 0, 0, 0]], dtype=np.float64)
    settings = dict(
        n=n, x0=(0.0, -Ly / 2, 0.0), x1=(Lx, Ly / 2, Lz),
        diff=("o8_e_c_p", y_scheme, "o8_e_c_p"), filt=("o10_e_c_p", "o10_i_c_o", "o10_e_c_p"),
        alpha=0.0, strength=0.2, di_freq=(1, 1, 1), ai_freq=(1, 1, 1), gamma=g, R=1.0, W=1.0,
        mu0=rho0 * dU * 1.0 / reynolds, T0=T0, Pr=PR, bc=bc,
        sponge_length=(0.0, sponge_points * dy, 0.0), sponge_amplitude=1.0,
        dt=_dt_cfl(q, min(Lx / n1, dy, Lz / n3), cfl, g))
    return settings, q


def isotropic_turbulence(n: int = 256, seed: int = 3, mach_t: float = 0.3, k0: float = 4.0,
                         re_lambda: float = 100.0, cfl: float = 0.5) -> Tuple[Dict, np.ndarray]:
    """Decaying isotropic turbulence in the periodic box [0, 2pi]^3: a solenoidal velocity field with
    energy spectrum E(k) ~ k^4 exp(-2 (k/k0)^2) and random phases from PCG64(seed), scaled to the
    turbulent Mach number sqrt(<u.u>)/c = mach_t; uniform rho = 1, p = 1/gamma (c = 1, R = W = 1, so
    T = p / rho).  The viscosity gives Re_lambda = u' lambda / nu with u' = sqrt(<u.u>/3) and the
    Taylor microscale lambda = sqrt(<u_x^2> / <(du_x/dx)^2>) of the initial field (spectral
    derivatives); Sutherland's law is referenced to the initial temperature."""
    g = GAMMA
    L = 2.0 * math.pi
    dx = L / n
    rng = np.random.Generator(np.random.PCG64(seed))
    k1 = np.fft.fftfreq(n, d=1.0 / n)
    KX, KY, KZ = np.meshgrid(k1, k1, k1, indexing="ij")
    K2 = KX ** 2 + KY ** 2 + KZ ** 2
    Kmag = np.sqrt(K2)
    with np.errstate(divide="ignore", invalid="ignore"):
        E = np.where(Kmag > 0, Kmag ** 4 * np.exp(-2.0 * (Kmag / k0) ** 2), 0.0)
        amp = np.where(Kmag > 0, np.sqrt(E / (4.0 * math.pi * np.maximum(K2, 1e-30))), 0.0)
    xi = [rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n)) for _ in range(3)]
    kdx = (KX * xi[0] + KY * xi[1] + KZ * xi[2]) / np.where(K2 > 0, K2, 1.0)
    uh = [amp * (xi[0] - KX * kdx), amp * (xi[1] - KY * kdx), amp * (xi[2] - KZ * kdx)]
    u = [np.real(np.fft.ifftn(c)) for c in uh]
    scale = mach_t / math.sqrt(float(np.mean(u[0] ** 2 + u[1] ** 2 + u[2] ** 2)))
    u = [scale * c for c in u]
    dudx = np.real(np.fft.ifftn(1j * KX * np.fft.fftn(u[0])))
    lam = math.sqrt(float(np.mean(u[0] ** 2)) / float(np.mean(dudx ** 2)))
    uprime = mach_t / math.sqrt(3.0)
    nu = uprime * lam / re_lambda
    rho0, p0 = 1.0, 1.0 / g
    q = _state(n, n, n)
    q[..., 0] = rho0
    for v in range(3):
        q[..., 1 + v] = rho0 * u[v]
    q[..., 4] = p0
    settings = dict(
        n=(n, n, n), x0=(0.0, 0.0, 0.0), x1=(L, L, L),
        diff=("o8_e_c_p",) * 3, filt=("o10_e_c_p",) * 3, alpha=0.0, strength=0.2,
        di_freq=(1, 1, 1), gamma=g, R=1.0, W=1.0, mu0=rho0 * nu, T0=p0 / rho0, Pr=PR,
        dt=_dt_cfl(q, dx, cfl, g))
    return settings, q


def smooth_random_state(n=(16, 12, 10), seed: int = 0, p0: float = 1.0, rho0: float = 1.0,
                        amp: float = 0.05, x1=(1.0, 1.0, 1.0)) -> np.ndarray:
    """A smooth positive state built from a few random Fourier modes (test input)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n1, n2, n3 = n
    xs = [np.arange(m) / m * 2 * math.pi for m in n]
    q = _state(n1, n2, n3)
    base = [rho0, 0.0, 0.0, 0.0, p0]
    for v in range(5):
        f = np.zeros((n1, n2, n3))
        for _ in range(3):
            k = rng.integers(0, 3, size=3)
            ph = rng.uniform(0, 2 * math.pi, size=3)
            f += (np.cos(k[0] * xs[0] + ph[0])[:, None, None] * np.cos(k[1] * xs[1] + ph[1])[None, :, None]
                  * np.cos(k[2] * xs[2] + ph[2])[None, None, :])
        q[..., v] = base[v] + amp * f * (1.0 if v in (0, 4) else 4.0)
    q[..., 1] *= q[..., 0]
    q[..., 2] *= q[..., 0]
    q[..., 3] *= q[..., 0]
    return q
