// Point-wise characteristic boundary treatments, written once for any scalar type: double for the
// direct kernels, the forward-mode Dual of dual.cuh for their exact Jacobians in the discrete adjoint.
#pragma once

namespace cruna {

// characteristic_q_k1d (src/boundaries/nonreflecting.f90:46-137): q (rho, rho u, rho v, rho w, p) is
// relaxed towards aim along the waves whose eigenvalue points into the domain; returns the new q.
// With per-point normal vectors (characteristic_q_k4d, nonreflecting.f90:141-233) the change towards
// aim is first weighted by the sponge shape sh (1 for the box types).
template <class S, class A>
__host__ __device__ __forceinline__ void char_q_point(const S q[5], const A aim[5], double k1, double k2,
                                                      double k3, double gamma, S out[5], double sh = 1.0) {
  const S r = q[0], u0 = q[1] / r, u1 = q[2] / r, u2 = q[3] / r, pp = q[4];
  const S c = sqrt(gamma * q[4] / q[0]);
  const A ar = aim[0];
  S d0 = ar - r;
  S d1 = aim[1] / ar - u0;
  S d2 = aim[2] / ar - u1;
  S d3 = aim[3] / ar - u2;
  S d4 = aim[4] - pp;
  if (sh != 1.0) {
    d0 = d0 * sh; d1 = d1 * sh; d2 = d2 * sh; d3 = d3 * sh; d4 = d4 * sh;
  }
  const double kx = -k1, ky = -k2, kz = -k3;
  const S c2 = c * c;
  S R1 = kx * d0 + kz * d2 - ky * d3 - kx * d4 / c2;
  S R2 = ky * d0 - kz * d1 + kx * d3 - ky * d4 / c2;
  S R3 = kz * d0 + ky * d1 - kx * d2 - kz * d4 / c2;
  S R4 = kx * d1 + ky * d2 + kz * d3 + d4 / (r * c);
  S R5 = -kx * d1 - ky * d2 - kz * d3 + d4 / (r * c);
  const S lamS = kx * u0 + ky * u1 + kz * u2;
  const S lamP = lamS + c, lamM = lamS - c;
  if (lamS < 0.0) { R1 = 0.0; R2 = 0.0; R3 = 0.0; }
  if (lamP < 0.0) R4 = 0.0;
  if (lamM < 0.0) R5 = 0.0;
  const S e1 = kx * R1 + ky * R2 + kz * R3 + r / (2.0 * c) * R4 + r / (2.0 * c) * R5;
  const S e2 = -kz * R2 + ky * R3 + 0.5 * kx * R4 - 0.5 * kx * R5;
  const S e3 = kz * R1 - kx * R3 + 0.5 * ky * R4 - 0.5 * ky * R5;
  const S e4 = -ky * R1 + kx * R2 + 0.5 * kz * R4 - 0.5 * kz * R5;
  const S e5 = +0.5 * r * c * R4 + 0.5 * r * c * R5;
  const S rn = r + e1;
  out[0] = rn;
  out[1] = rn * (u0 + e2);
  out[2] = rn * (u1 + e3);
  out[3] = rn * (u2 + e4);
  out[4] = pp + e5;
}

// characteristic_rhs_k1d without shape (nonreflecting.f90:237-341), BC type 204: the RHS at the point
// is replaced by the rate that relaxes q + dt*rhs towards aim along the incoming waves.
// With shape (characteristic_rhs_k4d with shape, nonreflecting.f90:345-449, type 206) the result is
// blended with the incoming RHS: (1 - sh) rhs + sh * (characteristic rate).
template <class S>
__host__ __device__ __forceinline__ void char_rhs_point(const S rhs[5], const S q[5], const double aim[5],
                                                        double k1, double k2, double k3, double gamma,
                                                        double dt, S out[5], bool shaped = false,
                                                        double sh = 0.0) {
  const double inv_dt = 1.0 / dt;
  const S r = q[0], u0 = q[1] / r, u1 = q[2] / r, u2 = q[3] / r;
  const S c = sqrt(gamma * q[4] / q[0]);
  const double ar = aim[0];
  S d0 = ar - r, d1 = aim[1] / ar - u0, d2 = aim[2] / ar - u1, d3 = aim[3] / ar - u2, d4 = aim[4] - q[4];
  const S tmp = dt / r;
  d0 = d0 + rhs[0] * dt;
  d1 = d1 + rhs[1] * tmp;
  d2 = d2 + rhs[2] * tmp;
  d3 = d3 + rhs[3] * tmp;
  d4 = d4 + rhs[4] * dt;
  const double kx = -k1, ky = -k2, kz = -k3;
  const S c2 = c * c;
  S R1 = kx * d0 + kz * d2 - ky * d3 - kx * d4 / c2;
  S R2 = ky * d0 - kz * d1 + kx * d3 - ky * d4 / c2;
  S R3 = kz * d0 + ky * d1 - kx * d2 - kz * d4 / c2;
  S R4 = kx * d1 + ky * d2 + kz * d3 + d4 / (r * c);
  S R5 = -kx * d1 - ky * d2 - kz * d3 + d4 / (r * c);
  const S lamS = kx * u0 + ky * u1 + kz * u2;
  if (lamS < 0.0) { R1 = 0.0; R2 = 0.0; R3 = 0.0; }
  if (lamS + c < 0.0) R4 = 0.0;
  if (lamS - c < 0.0) R5 = 0.0;
  const S e1 = kx * R1 + ky * R2 + kz * R3 + r / (2.0 * c) * R4 + r / (2.0 * c) * R5;
  const S e2 = -kz * R2 + ky * R3 + 0.5 * kx * R4 - 0.5 * kx * R5;
  const S e3 = kz * R1 - kx * R3 + 0.5 * ky * R4 - 0.5 * ky * R5;
  const S e4 = -ky * R1 + kx * R2 + 0.5 * kz * R4 - 0.5 * kz * R5;
  const S e5 = +0.5 * r * c * R4 + 0.5 * r * c * R5;
  const S rn = r + e1;
  if (shaped) {
    const double t1 = sh * inv_dt;
    out[0] = (1.0 - sh) * rhs[0] + e1 * t1;
    out[4] = (1.0 - sh) * rhs[4] + e5 * t1;
    const S t2 = t1 * rn;
    out[1] = (1.0 - sh) * rhs[1] + e2 * t2;
    out[2] = (1.0 - sh) * rhs[2] + e3 * t2;
    out[3] = (1.0 - sh) * rhs[3] + e4 * t2;
    return;
  }
  out[0] = e1 * inv_dt;
  const S t2 = inv_dt * rn;
  out[1] = e2 * t2;
  out[2] = e3 * t2;
  out[3] = e4 * t2;
  out[4] = e5 * inv_dt;
}

// characteristic_qs_k1d / _k4d (nonreflecting.f90:453-554, :558-661): adjoint, target zero; the
// change -qs is weighted by sh (1 for the box types)
template <class S, class Q>
__host__ __device__ __forceinline__ void char_qs_point(const S qs[5], const Q q[5], double k1, double k2,
                                                       double k3, double gamma, S out[5], double sh = 1.0) {
  S ds[5];
  for (int v = 0; v < 5; ++v) ds[v] = -qs[v];
  if (sh != 1.0)
    for (int v = 0; v < 5; ++v) ds[v] = ds[v] * sh;
  const double kx = -k1, ky = -k2, kz = -k3;
  const double gm1 = gamma - 1.0;
  const Q c = sqrt(gamma * (q[4] / q[0]));
  const Q g_c = gm1 / c;
  const Q u = q[1] / q[0], v = q[2] / q[0], w = q[3] / q[0];
  const Q ku = kx * u + ky * v + kz * w;
  const S kus = kx * ds[1] + ky * ds[2] + kz * ds[3];
  const S ruus = (ds[0] + u * ds[1] + v * ds[2] + w * ds[3]) / c;
  const S rups = ruus + ds[4] / g_c;
  S drs = 0.0, dus = 0.0, dvs = 0.0, dws = 0.0, dps = 0.0;
  if (ku < 0.0) {
    drs = ds[0] + ku * kus;
    dus = ds[1] - kx * kus;
    dvs = ds[2] - ky * kus;
    dws = ds[3] - kz * kus;
    dps = -g_c * ruus;
  }
  if (ku + c < 0.0) {
    const S tmp = 0.5 * (kus + rups);
    drs = drs - ku * tmp; dus = dus + kx * tmp; dvs = dvs + ky * tmp; dws = dws + kz * tmp;
    dps = dps + g_c * tmp;
  }
  if (ku - c < 0.0) {
    const S tmp = 0.5 * (kus - rups);
    drs = drs - ku * tmp; dus = dus + kx * tmp; dvs = dvs + ky * tmp; dws = dws + kz * tmp;
    dps = dps - g_c * tmp;
  }
  out[0] = qs[0] + drs;
  out[1] = qs[1] + dus;
  out[2] = qs[2] + dvs;
  out[3] = qs[3] + dws;
  out[4] = qs[4] + dps;
}

}  // namespace cruna
