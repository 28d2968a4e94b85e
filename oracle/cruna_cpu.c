/*
 * CPU restatement (C + OpenMP) of the CRUNA direct + adjoint time step for periodic explicit schemes
 * -- TEST INFRASTRUCTURE and the timed CPU baseline of bench.py, never the product.
 *
 * It follows the reference's call structure rather than the GPU's: every Dx_d call of
 * right_hand_side_direct_3d (src/equations/ns_rho_rhou_p.f90:31-253) and
 * right_hand_side_adjoint_3d (:257-536) fills a full-field temporary, the point-wise assembly follows
 * the reference's statement order, RK4 follows src/time/rk_o4_e.f90:17-105, and the loop bodies
 * follow src/main/computation_direct.f90:64-107 / computation_adjoint.f90:60-108 (step, filters
 * i1 -> i2 -> i3).  Loops over grid planes are parallelised with OpenMP.  Derivative cores: periodic
 * explicit central stencils a_m (f[i+m] - f[i-m]) / (h*div) (o4_e_c_p, o8_e_c_p); filter: the
 * blended explicit periodic o10 stencil.  Checked against the numpy oracle (cruna_oracle.py) by the
 * test-suite.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  int n[3];
  double dx[3];
  int r[3];           /* stencil half-width per direction (0: empty core -> derivative 0) */
  double c[3][5];     /* c[d][1..r] */
  double div[3];      /* 12 for o4_e_c_p, 1 for o8_e_c_p */
  int fon[3];         /* filter direction active */
  double fa[6];       /* filter a0..a5 */
  double blend;       /* filter strength */
  double gamma, R, W, mu0, T0, Pr, dt;
  int heat_flux_dx;
} ccpu_cfg;

static long long npts(const ccpu_cfg *c) { return (long long)c->n[0] * c->n[1] * c->n[2]; }

static inline int wrap(int i, int n) { return ((i % n) + n) % n; }

/* Dx_d(f) or Dx_d(f*g), h = grid spacing (or 1 when h is absent) */
static void dxd(const ccpu_cfg *c, int d, const double *f, const double *g, double *out, double h) {
  const int n1 = c->n[0], n2 = c->n[1], n3 = c->n[2], r = c->r[d], nd = c->n[d];
  const long long s = d == 0 ? 1 : (d == 1 ? n1 : (long long)n1 * n2);
  const double sc = 1.0 / (h * c->div[d]);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < n3; ++k)
    for (int j = 0; j < n2; ++j)
      for (int i = 0; i < n1; ++i) {
        const long long p = i + (long long)n1 * (j + (long long)n2 * k);
        if (r == 0) {
          out[p] = 0.0;
          continue;
        }
        const int pos = d == 0 ? i : (d == 1 ? j : k);
        const long long base = p - pos * s;
        double t = 0.0;
        for (int m = 1; m <= r; ++m) {
          const long long ip = base + wrap(pos + m, nd) * s, im = base + wrap(pos - m, nd) * s;
          const double dd = g ? (f[ip] * g[ip] - f[im] * g[im]) : (f[ip] - f[im]);
          t = (m == 1) ? c->c[d][1] * dd : t + c->c[d][m] * dd;
        }
        out[p] = t * sc;
      }
}

enum { U1, U2, U3, TT, UX, UY, UZ, VX, VY, VZ, WX, WY, WZ, T11, T22, T33, T12, T13, T23, MU,
       AX, AY, AZ, PX, PY, PZ, HX, HY, HZ, NTMP };

static void rhs_direct(const ccpu_cfg *c, const double *q, double *rhs, double *t) {
  const long long N = npts(c);
  double *F[NTMP];
  for (int f = 0; f < NTMP; ++f) F[f] = t + f * N;
  const double *r = q, *ru = q + N, *rv = q + 2 * N, *rw = q + 3 * N, *p = q + 4 * N;
  const double WoR = c->W / c->R, gam = c->gamma;
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < N; ++i) {                     /* ns_rho_rhou_p.f90:95-99, :115 */
    F[U1][i] = ru[i] / r[i];
    F[U2][i] = rv[i] / r[i];
    F[U3][i] = rw[i] / r[i];
    F[TT][i] = WoR * p[i] / r[i];
  }
  for (int v = 0; v < 3; ++v)                             /* :102-112 */
    for (int d = 0; d < 3; ++d) dxd(c, d, F[U1 + v], NULL, F[UX + 3 * v + d], c->dx[d]);
  const double cp = gam * (c->R / c->W) / (gam - 1.0);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < N; ++i) {                     /* :116-128 */
    const double T = F[TT][i];
    const double mu = c->mu0 * pow(T / c->T0, 1.5) * ((c->T0 + 110.4) / (T + 110.4));
    const double md = -(2.0 / 3.0 * mu * (F[UX][i] + F[VY][i] + F[WZ][i]));
    F[MU][i] = mu;
    F[T11][i] = md + 2 * mu * F[UX][i];
    F[T22][i] = md + 2 * mu * F[VY][i];
    F[T33][i] = md + 2 * mu * F[WZ][i];
    F[T12][i] = mu * (F[UY][i] + F[VX][i]);
    F[T13][i] = mu * (F[UZ][i] + F[WX][i]);
    F[T23][i] = mu * (F[VZ][i] + F[WY][i]);
  }
  /* mass (:131-135) */
  dxd(c, 0, ru, NULL, F[AX], c->dx[0]);
  dxd(c, 1, rv, NULL, F[AY], c->dx[1]);
  dxd(c, 2, rw, NULL, F[AZ], c->dx[2]);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < N; ++i) rhs[i] = -F[AX][i] - F[AY][i] - F[AZ][i];
  /* momentum (:138-177) */
  const double *flux[3] = {ru, rv, rw};
  const int tau[3][3] = {{T11, T12, T13}, {T12, T22, T23}, {T13, T23, T33}};
  for (int v = 0; v < 3; ++v) {
    double *rr = rhs + (v + 1) * N;
    for (int d = 0; d < 3; ++d) dxd(c, d, flux[d], F[U1 + v], F[AX + d], c->dx[d]);
    dxd(c, v, p, NULL, F[PX + v], c->dx[v]);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i) rr[i] = -F[AX][i] - F[AY][i] - F[AZ][i] - F[PX + v][i];
    for (int d = 0; d < 3; ++d) dxd(c, d, F[tau[v][d]], NULL, F[AX + d], c->dx[d]);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i) rr[i] = rr[i] + F[AX][i] + F[AY][i] + F[AZ][i];
  }
  /* pressure equation (:180-209) */
  double *r5 = rhs + 4 * N;
  for (int d = 0; d < 3; ++d) dxd(c, d, p, F[U1 + d], F[AX + d], c->dx[d]);
  const double gt = gam / (gam - 1.0);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < N; ++i) {
    r5[i] = gt * (-F[AX][i] - F[AY][i] - F[AZ][i]);
    r5[i] = r5[i] + F[U1][i] * F[PX][i] + F[U2][i] * F[PY][i] + F[U3][i] * F[PZ][i];
  }
  for (int d = 0; d < 3; ++d)
    dxd(c, d, F[TT], NULL, F[HX + d], c->heat_flux_dx ? c->dx[d] : 1.0);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < N; ++i) {
    const double lam = F[MU][i] * cp / c->Pr;
    F[HX][i] = lam * F[HX][i];
    F[HY][i] = lam * F[HY][i];
    F[HZ][i] = lam * F[HZ][i];
  }
  for (int d = 0; d < 3; ++d) dxd(c, d, F[HX + d], NULL, F[AX + d], c->heat_flux_dx ? c->dx[d] : 1.0);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < N; ++i) {
    double e = r5[i] + F[AX][i] + F[AY][i] + F[AZ][i];
    e = e + F[T11][i] * F[UX][i] + F[T12][i] * F[UY][i] + F[T13][i] * F[UZ][i] + F[T12][i] * F[VX][i] +
        F[T22][i] * F[VY][i] + F[T23][i] * F[VZ][i] + F[T13][i] * F[WX][i] + F[T23][i] * F[WY][i] +
        F[T33][i] * F[WZ][i];
    r5[i] = (gam - 1.0) * e;
  }
}

enum { A_U1, A_U2, A_U3, A_GPR, A_IR, A_D0, A_S = A_D0 + 5, A_P, A_NTMP };

static void rhs_adjoint(const ccpu_cfg *c, const double *qs, const double *q, double *rhs, double *t) {
  const long long N = npts(c);
  double *F[A_NTMP];
  for (int f = 0; f < A_NTMP; ++f) F[f] = t + f * N;
  const double gam = c->gamma, gm1 = gam - 1.0;
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < N; ++i) {                    /* :292-301 */
    F[A_GPR][i] = gam * q[i + 4 * N] / (q[i] * gm1);
    F[A_IR][i] = 1.0 / q[i];
    F[A_U1][i] = q[i + N] / q[i];
    F[A_U2][i] = q[i + 2 * N] / q[i];
    F[A_U3][i] = q[i + 3 * N] / q[i];
  }
  memset(rhs, 0, sizeof(double) * 5 * N);
  for (int d = 0; d < 3; ++d) {
    for (int v = 0; v < 5; ++v) dxd(c, d, qs + v * N, NULL, F[A_D0 + v], c->dx[d]);
    dxd(c, d, qs + 4 * N, F[A_U1 + d], F[A_S], c->dx[d]);
    dxd(c, d, q + 4 * N, NULL, F[A_P], c->dx[d]);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i) {
      const double u1 = F[A_U1][i], u2 = F[A_U2][i], u3 = F[A_U3][i], gpr = F[A_GPR][i], ir = F[A_IR][i];
      const double a = F[A_D0][i], b = F[A_D0 + 1][i], cc = F[A_D0 + 2][i], dd = F[A_D0 + 3][i],
                   e = F[A_D0 + 4][i], sx = F[A_S][i], px = F[A_P][i], qs5 = qs[i + 4 * N];
      double r1 = rhs[i], r2 = rhs[i + N], r3 = rhs[i + 2 * N], r4 = rhs[i + 3 * N], r5 = rhs[i + 4 * N];
      const double ud = d == 0 ? u1 : (d == 1 ? u2 : u3);
      if (d == 0) {
        r1 = r1 + (u1 * u1) * b + (u1 * u2) * cc + (u1 * u3) * dd + gpr * u1 * e;
        r2 = r2 - a - 2.0 * u1 * b - u2 * cc - u3 * dd - gpr * e;
        r3 = r3 - u1 * cc;
        r4 = r4 - u1 * dd;
        r5 = r5 - gm1 * b - gam * u1 * e;
      } else if (d == 1) {
        r1 = r1 + (u2 * u1) * b + (u2 * u2) * cc + (u2 * u3) * dd + gpr * u2 * e;
        r2 = r2 - u2 * b;
        r3 = r3 - a - u1 * b - 2 * u2 * cc - u3 * dd - gpr * e;
        r4 = r4 - u2 * dd;
        r5 = r5 - gm1 * cc - gam * u2 * e;
      } else {
        r1 = r1 + (u3 * u1) * b + (u3 * u2) * cc + (u3 * u3) * dd + gpr * u3 * e;
        r2 = r2 - u3 * b;
        r3 = r3 - u3 * cc;
        r4 = r4 - a - u1 * b - u2 * cc - 2 * u3 * dd - gpr * e;
        r5 = r5 - gm1 * dd - gam * u3 * e;
      }
      r5 = r5 - gm1 * (-sx);
      r1 = r1 + qs5 * ud * ir * px;
      if (d == 0) r2 = r2 - qs5 * ir * px;
      else if (d == 1) r3 = r3 - qs5 * ir * px;
      else r4 = r4 - qs5 * ir * px;
      rhs[i] = r1; rhs[i + N] = r2; rhs[i + 2 * N] = r3; rhs[i + 3 * N] = r4; rhs[i + 4 * N] = r5;
    }
  }
}

/* blended explicit periodic o10 filter along d, for 5 variables, out of place */
static void filter_dir(const ccpu_cfg *c, int d, const double *in, double *out) {
  const int n1 = c->n[0], n2 = c->n[1], n3 = c->n[2], nd = c->n[d];
  const long long N = npts(c), s = d == 0 ? 1 : (d == 1 ? n1 : (long long)n1 * n2);
  for (int v = 0; v < 5; ++v) {
    const double *f = in + v * N;
    double *o = out + v * N;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < n3; ++k)
      for (int j = 0; j < n2; ++j)
        for (int i = 0; i < n1; ++i) {
          const long long p = i + (long long)n1 * (j + (long long)n2 * k);
          const int pos = d == 0 ? i : (d == 1 ? j : k);
          const long long base = p - pos * s;
          double t = c->fa[0] * f[p];
          for (int m = 1; m <= 5; ++m) t = t + c->fa[m] * (f[base + wrap(pos + m, nd) * s] + f[base + wrap(pos - m, nd) * s]);
          o[p] = f[p] - c->blend * (f[p] - t);
        }
  }
}

/* classical RK4 (rk_o4_e.f90); adjoint: dtv < 0 and q frozen */
static void rk4(const ccpu_cfg *c, double *x, const double *q, double dtv, double *w) {
  const long long M = 5 * npts(c);
  double *k = w, *acc = w + M, *xs = w + 2 * M, *tmp = w + 3 * M;
  const double dth = dtv * 0.5;
  for (int s = 1; s <= 4; ++s) {
    const double *in = s == 1 ? x : xs;
    if (q) rhs_adjoint(c, in, q, k, tmp);
    else rhs_direct(c, in, k, tmp);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < M; ++i) {
      if (s == 1) { acc[i] = k[i]; xs[i] = x[i] + dth * k[i]; }
      else if (s == 2) { acc[i] = acc[i] + 2.0 * k[i]; xs[i] = x[i] + dth * k[i]; }
      else if (s == 3) { acc[i] = acc[i] + 2.0 * k[i]; xs[i] = x[i] + dtv * k[i]; }
      else { x[i] = x[i] + dtv / 6.0 * (acc[i] + k[i]); }
    }
  }
}

static void filters(const ccpu_cfg *c, double *x, double *buf) {
  const long long M = 5 * npts(c);
  for (int d = 0; d < 3; ++d)
    if (c->fon[d]) {
      filter_dir(c, d, x, buf);
      memcpy(x, buf, sizeof(double) * M);
    }
}

/* nsteps of (direct step + filters) followed by (adjoint step on the new direct state + filters);
   qs may be NULL (direct only).  threads <= 0 keeps the OpenMP default.  Returns 0 or -1 (memory). */
int ccpu_run(const ccpu_cfg *c, double *q, double *qs, int nsteps, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  const long long N = npts(c);
  const long long words = 3 * 5 * N + (NTMP > A_NTMP ? NTMP : A_NTMP) * N + 5 * N;
  double *w = (double *)malloc(sizeof(double) * (size_t)words);
  if (!w) return -1;
  for (int s = 0; s < nsteps; ++s) {
    rk4(c, q, NULL, c->dt, w);
    filters(c, q, w);
    if (qs) {
      rk4(c, qs, q, -c->dt, w);
      filters(c, qs, w);
    }
  }
  free(w);
  return 0;
}

int ccpu_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
