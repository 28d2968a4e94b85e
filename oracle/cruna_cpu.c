/*
 * CPU restatement (C + OpenMP) of the CRUNA direct + adjoint time step -- TEST INFRASTRUCTURE and the
 * timed CPU baseline of bench.py, never the product.  Schemes: periodic explicit derivative cores and
 * the periodic explicit o10 filter (the Taylor-Green and vortex configurations), and the mixing-layer
 * set: the o6 compact open derivative core (diff_pen_core_o6_i_c_o.f90:105-153 with LAPACK's dgttrs on
 * the dgttrf factors the caller passes), the o10 compact open filter (filter_pen_core_o10_i_c_o.f90),
 * type-201 characteristic rows (nonreflecting.f90:46-137, 453-554) and the type-400 sponge
 * (sponge_layer_core.f90:45-48).
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
  /* open / compact schemes and boundaries */
  int dkind[3];              /* 0: r/c/div above (explicit periodic, r = 0 empty); 1: o6_i_c_o compact */
  const double *dfac[3][4];  /* dgttrf factors dl, d, du, du2 of the compact derivative (kind 1) */
  const int *dpiv[3];        /* their 1-based pivots */
  int fkind[3];              /* 0: fon / o10_e_c_p above; 1: o10_i_c_o compact open filter */
  double fo[6];              /* o10_i_c_o interior a0..a5 (filter.alpha) */
  double fbrow[4][11];       /* o10_i_c_o closure rows for points 2..5 (filter_pen_core_o10_i_c_o.f90:201-251) */
  const double *ffac[3][4];  /* dgttrf factors of the compact filter */
  const int *fpiv[3];
  int nbc;                   /* boundary rows (type, is, ie, js, je, ks, ke, k1, k2, k3), 1-based */
  const double *bc;
  const double *qref;        /* 5N reference state (types 201, 400) */
  const double *shape;       /* N sponge shape (type 400) */
} ccpu_cfg;

static long long npts(const ccpu_cfg *c) { return (long long)c->n[0] * c->n[1] * c->n[2]; }

static inline int wrap(int i, int n) { return ((i % n) + n) % n; }

/* LAPACK dgttrs('N', n, 1) on one strided line b[0], b[s], ... (dgtts2: L solve with the row
   interchanges of dgttrf, then U back substitution) */
static void gttrs_line(int n, const double *const fac[4], const int *ipiv, double *b, long long s) {
  const double *dl = fac[0], *dd = fac[1], *du = fac[2], *du2 = fac[3];
  for (int i = 0; i < n - 1; ++i) {
    const int ip = ipiv[i] - 1;
    const double temp = b[(long long)(i + 1 - ip + i) * s] - dl[i] * b[(long long)ip * s];
    b[(long long)i * s] = b[(long long)ip * s];
    b[(long long)(i + 1) * s] = temp;
  }
  b[(long long)(n - 1) * s] = b[(long long)(n - 1) * s] / dd[n - 1];
  if (n > 1) b[(long long)(n - 2) * s] = (b[(long long)(n - 2) * s] - du[n - 2] * b[(long long)(n - 1) * s]) / dd[n - 2];
  for (int i = n - 3; i >= 0; --i)
    b[(long long)i * s] = (b[(long long)i * s] - du[i] * b[(long long)(i + 1) * s] - du2[i] * b[(long long)(i + 2) * s]) / dd[i];
}

/* o6_i_c_o derivative of f (or f*g) along d: explicit part divided by h, then the tridiagonal solve
   (diff_pen_core_o6_i_c_o.f90:105-153, the oracle's diff_core) */
static void dxd_compact(const ccpu_cfg *c, int d, const double *f, const double *g, double *out, double h) {
  const int n1 = c->n[0], n2 = c->n[1], n3 = c->n[2], nd = c->n[d];
  const long long s = d == 0 ? 1 : (d == 1 ? n1 : (long long)n1 * n2);
  const double a = 14.00 / 9.0 / 2.0, b = 1.00 / 9.0 / 4.0, cc = 17.00 / 6.0, dd = 1.50, e = 1.00 / 6.0, ff = 0.75;
  const int m1 = d == 0 ? n2 : n1, m2 = d == 2 ? n2 : n3;   /* the two other directions */
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < m2; ++k)
    for (int j = 0; j < m1; ++j) {
      long long base;
      if (d == 0) base = (long long)n1 * (j + (long long)n2 * k);
      else if (d == 1) base = j + (long long)n1 * n2 * k;
      else base = j + (long long)n1 * k;
#define V(i) (g ? f[base + (long long)(i) * s] * g[base + (long long)(i) * s] : f[base + (long long)(i) * s])
      double *o = out + base;
      const int n = nd;
      o[0] = (-cc * V(0) + dd * (V(1) + V(2)) - e * V(3)) / h;
      o[s] = (-ff * V(0) + ff * V(2)) / h;
      for (int i = 2; i < n - 2; ++i) o[(long long)i * s] = (a * (V(i + 1) - V(i - 1)) + b * (V(i + 2) - V(i - 2))) / h;
      o[(long long)(n - 2) * s] = (ff * V(n - 1) - ff * V(n - 3)) / h;
      o[(long long)(n - 1) * s] = (cc * V(n - 1) - dd * (V(n - 2) + V(n - 3)) + e * V(n - 4)) / h;
#undef V
      gttrs_line(n, c->dfac[d], c->dpiv[d], o, s);
    }
}

/* Dx_d(f) or Dx_d(f*g), h = grid spacing (or 1 when h is absent) */
static void dxd(const ccpu_cfg *c, int d, const double *f, const double *g, double *out, double h) {
  if (c->dkind[d] == 1) {
    dxd_compact(c, d, f, g, out, h);
    return;
  }
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

/* ---- boundary rows (boundary_conditions.f90:52-377 for the types of the mixing layer) ---- */

/* characteristic_q_k1d (nonreflecting.f90:46-137) at one point: q[v*N] updated towards aim */
static void char_q_point(const ccpu_cfg *c, double *q, const double *aim, long long N, const double *kv) {
  const double r = q[0], u0 = q[N] / r, u1 = q[2 * N] / r, u2 = q[3 * N] / r, p = q[4 * N];
  const double cs = sqrt(c->gamma * q[4 * N] / q[0]);
  double dq[5];
  dq[0] = aim[0] - r;
  dq[1] = aim[N] / aim[0] - u0;
  dq[2] = aim[2 * N] / aim[0] - u1;
  dq[3] = aim[3 * N] / aim[0] - u2;
  dq[4] = aim[4 * N] - p;
  const double kx = -kv[0], ky = -kv[1], kz = -kv[2];
  const double c2 = cs * cs;
  double R1 = kx * dq[0] + kz * dq[2] - ky * dq[3] - kx * dq[4] / c2;
  double R2 = ky * dq[0] - kz * dq[1] + kx * dq[3] - ky * dq[4] / c2;
  double R3 = kz * dq[0] + ky * dq[1] - kx * dq[2] - kz * dq[4] / c2;
  double R4 = kx * dq[1] + ky * dq[2] + kz * dq[3] + dq[4] / (r * cs);
  double R5 = -kx * dq[1] - ky * dq[2] - kz * dq[3] + dq[4] / (r * cs);
  const double lamS = kx * u0 + ky * u1 + kz * u2, lamP = lamS + cs, lamM = lamS - cs;
  if (lamS < 0.0) R1 = R2 = R3 = 0.0;
  if (lamP < 0.0) R4 = 0.0;
  if (lamM < 0.0) R5 = 0.0;
  const double d1 = kx * R1 + ky * R2 + kz * R3 + r / (2.0 * cs) * R4 + r / (2.0 * cs) * R5;
  const double d2 = -kz * R2 + ky * R3 + 0.5 * kx * R4 - 0.5 * kx * R5;
  const double d3 = kz * R1 - kx * R3 + 0.5 * ky * R4 - 0.5 * ky * R5;
  const double d4 = -ky * R1 + kx * R2 + 0.5 * kz * R4 - 0.5 * kz * R5;
  const double d5 = +0.5 * r * cs * R4 + 0.5 * r * cs * R5;
  const double rn = r + d1;
  q[0] = rn;
  q[N] = rn * (u0 + d2);
  q[2 * N] = rn * (u1 + d3);
  q[3 * N] = rn * (u2 + d4);
  q[4 * N] = p + d5;
}

/* characteristic_qs_k1d (nonreflecting.f90:453-554) at one point, target zero */
static void char_qs_point(const ccpu_cfg *c, double *qs, const double *q, long long N, const double *kv) {
  double ds[5];
  for (int v = 0; v < 5; ++v) ds[v] = -qs[v * N];
  const double kx = -kv[0], ky = -kv[1], kz = -kv[2];
  const double gm1 = c->gamma - 1.0;
  const double cs = sqrt(c->gamma * (q[4 * N] / q[0]));
  const double g_c = gm1 / cs;
  const double u = q[N] / q[0], v = q[2 * N] / q[0], w = q[3 * N] / q[0];
  const double ku = kx * u + ky * v + kz * w;
  const double kus = kx * ds[1] + ky * ds[2] + kz * ds[3];
  const double ruus = (ds[0] + u * ds[1] + v * ds[2] + w * ds[3]) / cs;
  const double rups = ruus + ds[4] / g_c;
  double drs = 0.0, dus = 0.0, dvs = 0.0, dws = 0.0, dps = 0.0;
  if (ku < 0.0) {
    drs = ds[0] + ku * kus;
    dus = ds[1] - kx * kus;
    dvs = ds[2] - ky * kus;
    dws = ds[3] - kz * kus;
    dps = -g_c * ruus;
  }
  if (ku + cs < 0.0) {
    const double tmp = 0.5 * (kus + rups);
    drs = drs - ku * tmp;
    dus = dus + kx * tmp;
    dvs = dvs + ky * tmp;
    dws = dws + kz * tmp;
    dps = dps + g_c * tmp;
  }
  if (ku - cs < 0.0) {
    const double tmp = 0.5 * (kus - rups);
    drs = drs - ku * tmp;
    dus = dus + kx * tmp;
    dvs = dvs + ky * tmp;
    dws = dws + kz * tmp;
    dps = dps - g_c * tmp;
  }
  qs[0] += drs;
  qs[N] += dus;
  qs[2 * N] += dvs;
  qs[3 * N] += dws;
  qs[4 * N] += dps;
}

/* the 1-based index box of a row as [lo, hi) per direction */
static void row_box(const double *row, int lo[3], int hi[3]) {
  for (int d = 0; d < 3; ++d) {
    lo[d] = (int)lround(row[1 + 2 * d]) - 1;
    hi[d] = (int)lround(row[2 + 2 * d]);
  }
}

/* set_boundary_condition_q (types 201; rows in table order) */
static void bc_q(const ccpu_cfg *c, double *q) {
  const long long N = npts(c), n1 = c->n[0], n12 = (long long)c->n[0] * c->n[1];
  for (int b = 0; b < c->nbc; ++b) {
    const double *row = c->bc + 10 * b;
    if ((int)lround(row[0]) != 201) continue;
    int lo[3], hi[3];
    row_box(row, lo, hi);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = lo[2]; k < hi[2]; ++k)
      for (int j = lo[1]; j < hi[1]; ++j)
        for (int i = lo[0]; i < hi[0]; ++i) {
          const long long p = i + n1 * j + n12 * k;
          char_q_point(c, q + p, c->qref + p, N, row + 7);
        }
  }
}

/* set_boundary_condition_qs (type 201) */
static void bc_qs(const ccpu_cfg *c, double *qs, const double *q) {
  const long long N = npts(c), n1 = c->n[0], n12 = (long long)c->n[0] * c->n[1];
  for (int b = 0; b < c->nbc; ++b) {
    const double *row = c->bc + 10 * b;
    if ((int)lround(row[0]) != 201) continue;
    int lo[3], hi[3];
    row_box(row, lo, hi);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = lo[2]; k < hi[2]; ++k)
      for (int j = lo[1]; j < hi[1]; ++j)
        for (int i = lo[0]; i < hi[0]; ++i) {
          const long long p = i + n1 * j + n12 * k;
          char_qs_point(c, qs + p, q + p, N, row + 7);
        }
  }
}

/* set_boundary_condition_rhs (type 400: rhs -= shape (q - qref) on the whole block) */
static void bc_rhs(const ccpu_cfg *c, double *rhs, const double *q) {
  const long long N = npts(c);
  for (int b = 0; b < c->nbc; ++b) {
    if ((int)lround(c->bc[10 * b]) != 400) continue;
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < N; ++i)
      for (int v = 0; v < 5; ++v)
        rhs[i + v * N] = rhs[i + v * N] - c->shape[i] * (q[i + v * N] - c->qref[i + v * N]);
  }
}

enum { U1, U2, U3, TT, UX, UY, UZ, VX, VY, VZ, WX, WY, WZ, T11, T22, T33, T12, T13, T23, MU,
       AX, AY, AZ, PX, PY, PZ, HX, HY, HZ, NTMP };

static void rhs_direct(const ccpu_cfg *c, const double *q_in, double *rhs, double *t) {
  const long long N = npts(c);
  double *F[NTMP];
  for (int f = 0; f < NTMP; ++f) F[f] = t + f * N;
  const double *q = q_in;
  if (c->nbc > 0) {                                       /* ns_rho_rhou_p.f90:89-92 on a copy */
    double *qb = t + NTMP * N;
    memcpy(qb, q_in, sizeof(double) * 5 * N);
    bc_q(c, qb);
    q = qb;
  }
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
  if (c->nbc > 0) bc_rhs(c, rhs, q);                      /* :218 */
}

enum { A_U1, A_U2, A_U3, A_GPR, A_IR, A_D0, A_S = A_D0 + 5, A_P, A_NTMP };

static void rhs_adjoint(const ccpu_cfg *c, const double *qs_in, const double *q, double *rhs, double *t) {
  const long long N = npts(c);
  double *F[A_NTMP];
  for (int f = 0; f < A_NTMP; ++f) F[f] = t + f * N;
  const double *qs = qs_in;
  if (c->nbc > 0) {                                       /* :287-290 on a copy; rhss (:518, no q) leaves
                                                             types 201 / 400 alone */
    double *qb = t + A_NTMP * N;
    memcpy(qb, qs_in, sizeof(double) * 5 * N);
    bc_qs(c, qb, q);
    qs = qb;
  }
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

/* o10_i_c_o filter along d, out of place: interior stencil, end points copied, closure rows for
   points 2..5 and mirrors, tridiagonal solve (filter_pen_core_o10_i_c_o.f90, the oracle's filter_core) */
static void filter_dir_compact(const ccpu_cfg *c, int d, const double *in, double *out) {
  const int n1 = c->n[0], n2 = c->n[1], n3 = c->n[2], nd = c->n[d];
  const long long N = npts(c), s = d == 0 ? 1 : (d == 1 ? n1 : (long long)n1 * n2);
  const int m1 = d == 0 ? n2 : n1, m2 = d == 2 ? n2 : n3;
  for (int v = 0; v < 5; ++v) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < m2; ++k)
      for (int j = 0; j < m1; ++j) {
        long long base;
        if (d == 0) base = (long long)n1 * (j + (long long)n2 * k);
        else if (d == 1) base = j + (long long)n1 * n2 * k;
        else base = j + (long long)n1 * k;
        const double *f = in + v * N + base;
        double *o = out + v * N + base;
        const int n = nd;
        for (int i = 5; i < n - 5; ++i) {
          double t = c->fo[0] * f[(long long)i * s];
          for (int m = 1; m <= 5; ++m) t = t + c->fo[m] * (f[(long long)(i + m) * s] + f[(long long)(i - m) * s]);
          o[(long long)i * s] = t;
        }
        o[0] = f[0];
        o[(long long)(n - 1) * s] = f[(long long)(n - 1) * s];
        for (int row = 0; row < 4; ++row) {
          double a = 0.0, b = 0.0;
          for (int i = 0; i < 11; ++i) {
            a = a + c->fbrow[row][i] * f[(long long)i * s];
            b = b + c->fbrow[row][i] * f[(long long)(n - 1 - i) * s];
          }
          o[(long long)(1 + row) * s] = a;
          o[(long long)(n - 2 - row) * s] = b;
        }
        gttrs_line(n, c->ffac[d], c->fpiv[d], o, s);
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
      if (c->fkind[d] == 1) filter_dir_compact(c, d, x, buf);
      else filter_dir(c, d, x, buf);
      memcpy(x, buf, sizeof(double) * M);
    }
}

/* nsteps of (direct step + filters) followed by (adjoint step on the new direct state + filters);
   qs may be NULL (direct only).  threads <= 0 uses the OpenMP default the first call found.  Returns 0 or
   -1 (memory). */
#ifdef _OPENMP
/* the OpenMP thread count of the process before any call here changed it */
static int default_threads(void) {
  static int n = 0;
  if (n <= 0) n = omp_get_max_threads();
  return n;
}
#endif

int ccpu_run(const ccpu_cfg *c, double *q, double *qs, int nsteps, int threads) {
#ifdef _OPENMP
  /* the thread count set here persists in the process: a later call with threads <= 0 returns to the
     count the first call found */
  omp_set_num_threads(threads > 0 ? threads : default_threads());
#else
  (void)threads;
#endif
  const long long N = npts(c);
  const long long words = 3 * 5 * N + ((NTMP > A_NTMP ? NTMP : A_NTMP) + 5) * N + 5 * N;
  double *w = (double *)malloc(sizeof(double) * (size_t)words);
  if (!w) return -1;
  for (int s = 0; s < nsteps; ++s) {
    rk4(c, q, NULL, c->dt, w);
    if (c->nbc > 0) bc_q(c, q);                           /* computation_direct.f90: BC q outside the RHS */
    filters(c, q, w);
    if (qs) {
      rk4(c, qs, q, -c->dt, w);
      if (c->nbc > 0) bc_qs(c, qs, q);                    /* computation_adjoint.f90 */
      filters(c, qs, w);
    }
  }
  free(w);
  return 0;
}

/* the thread count a call with threads <= 0 uses (the process default, whatever an earlier call set) */
int ccpu_threads(void) {
#ifdef _OPENMP
  return default_threads();
#else
  return 1;
#endif
}
