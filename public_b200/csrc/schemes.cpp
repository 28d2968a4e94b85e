// Host-side set-up of the line operators: stencil coefficients of every derivative and filter core
// and the LAPACK tridiagonal factorisation they solve with.
//
// The coefficient tables follow the reference modules cited beside each case; the factorisation is a
// restatement of LAPACK's published dgttrf algorithm (partial pivoting LU of a tridiagonal matrix)
// so the pivots and multipliers are those the reference obtains from its LAPACK.
#include <cmath>
#include <cstring>
#include <string>

#include "cruna_internal.cuh"

namespace cruna {

// LAPACK dgttrf: LU factorisation of a tridiagonal matrix with row interchanges.
// dl(n-1) sub-diagonal, d(n) diagonal, du(n-1) super-diagonal are overwritten; du2(n-2) receives the
// second super-diagonal of U; ipiv(n) the 1-based pivot rows.  Returns info (0 = ok, i>0 = U(i,i)=0).
int lapack_dgttrf(int n, double *dl, double *d, double *du, double *du2, int *ipiv) {
  if (n < 0) return -1;
  if (n == 0) return 0;
  for (int i = 0; i < n; ++i) ipiv[i] = i + 1;
  for (int i = 0; i < n - 2; ++i) du2[i] = 0.0;
  auto eliminate = [&](int i, bool last) {
    if (std::fabs(d[i]) >= std::fabs(dl[i])) {
      // no row interchange
      if (d[i] != 0.0) {
        double fact = dl[i] / d[i];
        dl[i] = fact;
        d[i + 1] = d[i + 1] - fact * du[i];
      }
    } else {
      // interchange rows i and i+1
      double fact = d[i] / dl[i];
      d[i] = dl[i];
      dl[i] = fact;
      double temp = du[i];
      du[i] = d[i + 1];
      d[i + 1] = temp - fact * d[i + 1];
      if (!last) {
        du2[i] = du[i + 1];
        du[i + 1] = -fact * du[i + 1];
      }
      ipiv[i] = i + 2;
    }
  };
  for (int i = 0; i < n - 2; ++i) eliminate(i, false);
  if (n > 1) eliminate(n - 2, true);
  for (int i = 0; i < n; ++i)
    if (d[i] == 0.0) return i + 1;
  return 0;
}

// LAPACK dgttrs('N') for one right-hand side, using the factors of lapack_dgttrf.
void lapack_dgttrs(int n, const double *dl, const double *d, const double *du, const double *du2,
                   const int *ipiv, double *b) {
  for (int i = 0; i < n - 1; ++i) {
    if (ipiv[i] == i + 1) {
      b[i + 1] = b[i + 1] - dl[i] * b[i];
    } else {
      double temp = b[i];
      b[i] = b[i + 1];
      b[i + 1] = temp - dl[i] * b[i];
    }
  }
  b[n - 1] = b[n - 1] / d[n - 1];
  if (n > 1) b[n - 2] = (b[n - 2] - du[n - 2] * b[n - 1]) / d[n - 2];
  for (int i = n - 3; i >= 0; --i) b[i] = (b[i] - du[i] * b[i + 1] - du2[i] * b[i + 2]) / d[i];
}

static void factor(HostFactors &hf, int n) {
  hf.raw_dl = hf.dl;
  hf.raw_d = hf.d;
  hf.raw_du = hf.du;
  hf.du2.assign(n > 2 ? n - 2 : 1, 0.0);
  hf.ipiv.assign(n, 0);
  hf.info = lapack_dgttrf(n, hf.dl.data(), hf.d.data(), hf.du.data(), hf.du2.data(), hf.ipiv.data());
}

// Cyclic tridiagonal matrix (alpha off-diagonals, dc0 diagonal) as tridiagonal + rank-one correction,
// as init_left_implicit_diff_part of src/diff/diff_pen_core_o6_i_c_p.f90:170-228.
static void cyclic_factors(HostFactors &hf, int n, double alpha, double dc0) {
  hf.dl.assign(n - 1, alpha);
  hf.d.assign(n, dc0);
  hf.du.assign(n - 1, alpha);
  std::vector<double> fa(n, 0.0), fb(n, 0.0);
  fa[0] = -hf.d[0];
  fa[n - 1] = +alpha;
  fb[0] = +1.0;
  fb[n - 1] = -alpha / hf.d[0];
  hf.d[n - 1] = hf.d[n - 1] + (alpha * alpha / hf.d[0]);
  hf.d[0] = hf.d[0] + hf.d[0];
  factor(hf, n);
  lapack_dgttrs(n, hf.dl.data(), hf.d.data(), hf.du.data(), hf.du2.data(), hf.ipiv.data(), fa.data());
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += fb[i] * fa[i];
  hf.fbnorm.resize(n);
  for (int i = 0; i < n; ++i) hf.fbnorm[i] = fa[i] * fb[0] / (1.0 + s);
  hf.fbrat = fb[n - 1] / fb[0];
}

bool diff_is_periodic(int scheme) {
  return scheme == CRUNA_DIFF_O4_E_C_P || scheme == CRUNA_DIFF_O4_I_C_P_PADE ||
         scheme == CRUNA_DIFF_O6_I_C_P || scheme == CRUNA_DIFF_O8_E_C_P;
}

static void set_row(LineOp &op, int row, std::initializer_list<double> w) {
  int m = 0;
  for (double v : w) op.brow[row][m++] = v;
}

bool build_diff_op(int scheme, int n, LineOp &op, HostFactors &hf, std::string &err) {
  op = LineOp();
  op.n = n;
  op.antisym = 1;
  op.kind = OP_STENCIL;
  auto need = [&](int m) {
    if (n < m) {
      err = "derivative scheme " + std::to_string(scheme) + " needs at least " + std::to_string(m) +
            " points, got " + std::to_string(n);
      return false;
    }
    return true;
  };
  switch (scheme) {
    case CRUNA_DIFF_EMPTY:                     // diff_pen_core_empty.f90:21
      op.kind = OP_ZERO;
      return true;
    case CRUNA_DIFF_O4_E_C_P:                  // diff_pen_core_o4_e_c_p.f90:68-80
      if (!need(4)) return false;
      op.periodic = 1; op.r = 2; op.c[1] = 8.0; op.c[2] = -1.0; op.div = 12.0;
      return true;
    case CRUNA_DIFF_O8_E_C_P:                  // no reference counterpart
      if (!need(8)) return false;
      op.periodic = 1; op.r = 4;
      op.c[1] = 4.0 / 5.0; op.c[2] = -1.0 / 5.0; op.c[3] = 4.0 / 105.0; op.c[4] = -1.0 / 280.0;
      return true;
    case CRUNA_DIFF_O4_E_C_O:                  // diff_pen_core_o4_e_c_o.f90:68-80
      if (!need(6)) return false;
      op.r = 2; op.c[1] = 8.0; op.c[2] = -1.0; op.div = 12.0; op.nb = 2; op.bw = 5;
      set_row(op, 0, {-25.0, 48.0, -36.0, 16.0, -3.0});
      set_row(op, 1, {-3.0, -10.0, 18.0, -6.0, 1.0});
      return true;
    case CRUNA_DIFF_O2_E_C_O:                  // diff_pen_core_o2_e_c_o.f90:68-80
      if (!need(4)) return false;
      op.r = 1; op.c[1] = 0.5; op.nb = 2; op.bw = 3;
      set_row(op, 0, {-1.5, 2.0, -0.5});
      set_row(op, 1, {-0.5, 0.0, 0.5});
      return true;
    case CRUNA_DIFF_O6_I_C_P:                  // diff_pen_core_o6_i_c_p.f90:115-143, 160-226
      if (!need(5)) return false;
      op.periodic = 1; op.r = 2; op.c[1] = 14.00 / 9.0 / 2.0; op.c[2] = 1.00 / 9.0 / 4.0;
      op.solve = 1; op.cyclic = 1;
      cyclic_factors(hf, n, 1.0 / 3.0, 1.0);
      break;
    case CRUNA_DIFF_O4_I_C_P_PADE:             // diff_pen_core_o4_i_c_p_pade.f90:115-141, 158-223
      if (!need(3)) return false;
      op.periodic = 1; op.r = 1; op.c[1] = 1.0 / 2.0;
      op.solve = 1; op.cyclic = 1;
      cyclic_factors(hf, n, 1.0 / 6.0, 2.0 / 3.0);
      break;
    case CRUNA_DIFF_O6_I_C_O: {                // diff_pen_core_o6_i_c_o.f90:105-129, 148-197
      if (!need(6)) return false;
      const double a = 14.00 / 9.0 / 2.0, b = 1.00 / 9.0 / 4.0, c = 17.00 / 6.0, d = 1.50,
                   e = 1.00 / 6.0, f = 0.75;
      op.r = 2; op.c[1] = a; op.c[2] = b; op.nb = 2; op.bw = 4;
      set_row(op, 0, {-c, d, d, -e});
      set_row(op, 1, {-f, 0.0, f});
      op.solve = 1;
      const double alpha = 1.0 / 3.0;
      hf.dl.assign(n - 1, alpha);
      hf.d.assign(n, 1.0);
      hf.du.assign(n - 1, alpha);
      hf.du[0] = 3.00; hf.du[1] = 0.25; hf.du[n - 2] = 0.25;
      hf.dl[0] = 0.25; hf.dl[n - 2] = 3.00; hf.dl[n - 3] = 0.25;
      factor(hf, n);
      break;
    }
    case CRUNA_DIFF_O4_I_C_O_PADE: {           // diff_pen_core_o4_i_c_o_pade.f90:104-182
      if (!need(3)) return false;
      const double a = 1.0 / 2.0;
      op.r = 1; op.c[1] = a; op.nb = 1; op.bw = 2;
      set_row(op, 0, {-a, a});
      op.solve = 1;
      const double alpha = 1.0 / 6.0;
      hf.dl.assign(n - 1, alpha);
      hf.d.assign(n, 2.0 / 3.0);
      hf.du.assign(n - 1, alpha);
      hf.d[0] = 1.0 / 3.00; hf.d[n - 1] = 1.0 / 3.00;
      factor(hf, n);
      break;
    }
    default:
      err = "unknown derivative scheme " + std::to_string(scheme);
      return false;
  }
  if (hf.info != 0) {
    err = "dgttrf failed (info=" + std::to_string(hf.info) + ")";
    return false;
  }
  return true;
}

static void filter_interior(int scheme, double al, LineOp &op) {
  double *c = op.c;
  switch (scheme) {
    case CRUNA_FILTER_O2_I_C_P:
    case CRUNA_FILTER_O2_I_C_O:                // filter_pen_core_o2_i_c_p.f90 init_right
      op.r = 1;
      c[0] = 1.0 / 2.0 + al;
      c[1] = (1.0 / 2.0 + al) / 2.0;
      break;
    case CRUNA_FILTER_O4_I_C_O:                // filter_pen_core_o4_i_c_o.f90
      op.r = 2;
      c[0] = 5.0 / 8.0 + 3.0 * al / 4.0;
      c[1] = (1.0 / 2.0 + al) / 2.0;
      c[2] = (-1.0 / 8.0 + al / 4.0) / 2.0;
      break;
    case CRUNA_FILTER_O6_I_C_P:
    case CRUNA_FILTER_O6_I_C_O:                // filter_pen_core_o6_i_c_p.f90:167-178
      op.r = 3;
      c[0] = 11.0 / 16.0 + 5.0 * al / 8.0;
      c[1] = (15.0 / 32.0 + 17.0 * al / 16.0) / 2.0;
      c[2] = (-3.0 / 16.0 + 3.0 * al / 8.0) / 2.0;
      c[3] = (1.0 / 32.0 - 1.0 * al / 16.0) / 2.0;
      break;
    case CRUNA_FILTER_O8_I_C_O:                // filter_pen_core_o8_i_c_o.f90
      op.r = 4;
      c[0] = 93.0 / 128.0 + 70.0 * al / 128.0;
      c[1] = (7.0 / 16.0 + 18.0 * al / 16.0) / 2.0;
      c[2] = (-7.0 / 32.0 + 14.0 * al / 32.0) / 2.0;
      c[3] = (1.0 / 16.0 - 1.0 * al / 8.0) / 2.0;
      c[4] = (-1.0 / 128.0 + 1.0 * al / 64.0) / 2.0;
      break;
    case CRUNA_FILTER_O10_I_C_O:
    case CRUNA_FILTER_O10_E_C_P:               // filter_pen_core_o10_i_c_o.f90:182-199
      op.r = 5;
      c[0] = 193.0 / 256.0 + 126.0 * al / 256.0;
      c[1] = (105.0 / 256.0 + 302.0 * al / 256.0) / 2.0;
      c[2] = (-15.0 / 64.0 + 30.0 * al / 64.0) / 2.0;
      c[3] = (45.0 / 512.0 - 90.0 * al / 512.0) / 2.0;
      c[4] = (-5.0 / 256.0 + 10.0 * al / 256.0) / 2.0;
      c[5] = (1.0 / 512.0 - 2.0 * al / 512.0) / 2.0;
      break;
  }
}

static void filter_rows(int scheme, double al, LineOp &op) {
  // row 0 keeps the end point ("do nothing at the boundary points"); rows 1.. are the one-sided
  // coefficients_for_boundary of each open core
  op.keep_ends = 1;
  switch (scheme) {
    case CRUNA_FILTER_O2_I_C_O:
      op.nb = 1; op.bw = 1;
      break;
    case CRUNA_FILTER_O4_I_C_O:                // filter_pen_core_o4_i_c_o.f90
      op.nb = 2; op.bw = 5;
      set_row(op, 1, {1.0 / 16.0 + 7.0 * al / 8.0, 3.0 / 4.0 + 1.0 * al / 2.0, 3.0 / 8.0 + 1.0 * al / 4.0,
                      -1.0 / 4.0 + 1.0 * al / 2.0, 1.0 / 16.0 - 1.0 * al / 8.0});
      break;
    case CRUNA_FILTER_O6_I_C_O:                // filter_pen_core_o6_i_c_o.f90
      op.nb = 3; op.bw = 7;
      set_row(op, 1, {1.0 / 64.0 + 31.0 * al / 32.0, 29.0 / 32.0 + 3.0 * al / 16.0,
                      15.0 / 64.0 + 17.0 * al / 32.0, -5.0 / 16.0 + 5.0 * al / 8.0,
                      15.0 / 64.0 - 15.0 * al / 32.0, -3.0 / 32.0 + 3.0 * al / 16.0,
                      1.0 / 64.0 - 1.0 * al / 32.0});
      set_row(op, 2, {-1.0 / 64.0 + 1.0 * al / 32.0, 3.0 / 32.0 + 13.0 * al / 16.0,
                      49.0 / 64.0 + 15.0 * al / 32.0, 5.0 / 16.0 + 3.0 * al / 8.0,
                      -15.0 / 64.0 + 15.0 * al / 32.0, 3.0 / 32.0 - 3.0 * al / 16.0,
                      -1.0 / 64.0 + 1.0 * al / 32.0});
      break;
    case CRUNA_FILTER_O8_I_C_O:                // filter_pen_core_o8_i_c_o.f90
      op.nb = 4; op.bw = 9;
      set_row(op, 1, {1.0 / 256.0 + 127.0 * al / 128.0, 31.0 / 32.0 + 1.0 * al / 16.0,
                      7.0 / 64.0 + 25.0 * al / 32.0, -7.0 / 32.0 + 7.0 * al / 16.0,
                      35.0 / 128.0 - 70.0 * al / 128.0, -7.0 / 32.0 + 7.0 * al / 16.0,
                      7.0 / 64.0 - 7.0 * al / 32.0, -1.0 / 32.0 + 1.0 * al / 16.0,
                      1.0 / 256.0 - 1.0 * al / 128.0});
      set_row(op, 2, {-1.0 / 256.0 + 1.0 * al / 128.0, 1.0 / 32.0 + 15.0 * al / 16.0,
                      57.0 / 64.0 + 7.0 * al / 32.0, 7.0 / 32.0 + 9.0 * al / 16.0,
                      -35.0 / 128.0 + 70.0 * al / 128.0, 7.0 / 32.0 - 7.0 * al / 16.0,
                      -7.0 / 64.0 + 7.0 * al / 32.0, 1.0 / 32.0 - 1.0 * al / 16.0,
                      -1.0 / 256.0 + 1.0 * al / 128.0});
      set_row(op, 3, {1.0 / 256.0 - 1.0 * al / 128.0, -1.0 / 32.0 + 1.0 * al / 16.0,
                      7.0 / 64.0 + 25.0 * al / 32.0, 25.0 / 32.0 + 7.0 * al / 16.0,
                      35.0 / 128.0 + 29.0 * al / 64.0, -7.0 / 32.0 + 7.0 * al / 16.0,
                      7.0 / 64.0 - 7.0 * al / 32.0, -1.0 / 32.0 + 1.0 * al / 16.0,
                      1.0 / 256.0 - 1.0 * al / 128.0});
      break;
    case CRUNA_FILTER_O10_I_C_O:               // filter_pen_core_o10_i_c_o.f90:201-251
      op.nb = 5; op.bw = 11;
      set_row(op, 1, {1.0 / 1024.0 + 1022.0 * al / 1024.0, 507.0 / 512.0 + 10.0 * al / 512.0,
                      45.0 / 1024.0 + 934.0 * al / 1024.0, -15.0 / 128.0 + 30.0 * al / 128.0,
                      105.0 / 512.0 - 210.0 * al / 512.0, -63.0 / 256.0 + 126.0 * al / 256.0,
                      105.0 / 512.0 - 210.0 * al / 512.0, -15.0 / 128.0 + 30.0 * al / 128.0,
                      45.0 / 1024.0 - 90.0 * al / 1024.0, -5.0 / 512.0 + 10.0 * al / 512.0,
                      1.0 / 1024.0 - 2.0 * al / 1024.0});
      set_row(op, 2, {-1.0 / 1024.0 + 2.0 * al / 1024.0, 5.0 / 512.0 + 502.0 * al / 512.0,
                      979.0 / 1024.0 + 90.0 * al / 1024.0, 15.0 / 128.0 + 98.0 * al / 128.0,
                      -105.0 / 512.0 + 210.0 * al / 512.0, 63.0 / 256.0 - 126.0 * al / 256.0,
                      -105.0 / 512.0 + 210.0 * al / 512.0, 15.0 / 128.0 - 30.0 * al / 128.0,
                      -45.0 / 1024.0 + 90.0 * al / 1024.0, 5.0 / 512.0 - 10.0 * al / 512.0,
                      -1.0 / 1024.0 + 2.0 * al / 1024.0});
      set_row(op, 3, {1.0 / 1024.0 - 2.0 * al / 1024.0, -5.0 / 512.0 + 10.0 * al / 512.0,
                      45.0 / 1024.0 + 934.0 * al / 1024.0, 113.0 / 128.0 + 30.0 * al / 128.0,
                      105.0 / 512.0 + 302.0 * al / 512.0, -63.0 / 256.0 + 126.0 * al / 256.0,
                      105.0 / 512.0 - 210.0 * al / 512.0, -15.0 / 128.0 + 30.0 * al / 128.0,
                      45.0 / 1024.0 - 90.0 * al / 1024.0, -5.0 / 512.0 + 10.0 * al / 512.0,
                      1.0 / 1024.0 - 2.0 * al / 1024.0});
      set_row(op, 4, {-1.0 / 1024.0 + 2.0 * al / 1024.0, 5.0 / 512.0 - 10.0 * al / 512.0,
                      -45.0 / 1024.0 + 90.0 * al / 1024.0, 15.0 / 128.0 + 98.0 * al / 128.0,
                      407.0 / 512.0 + 210.0 * al / 512.0, 63.0 / 256.0 + 130.0 * al / 256.0,
                      -105.0 / 512.0 + 210.0 * al / 512.0, 15.0 / 128.0 - 30.0 * al / 128.0,
                      -45.0 / 1024.0 + 90.0 * al / 1024.0, 5.0 / 512.0 - 10.0 * al / 512.0,
                      -1.0 / 1024.0 + 2.0 * al / 1024.0});
      break;
  }
}

bool build_filter_op(int scheme, int n, double alpha, double strength, LineOp &op, HostFactors &hf,
                     std::string &err) {
  op = LineOp();
  op.n = n;
  op.antisym = 0;
  if (scheme == CRUNA_FILTER_EMPTY) {          // filter_pen_core_empty.f90: q = q
    op.kind = OP_COPY;
    return true;
  }
  if (scheme < 0 || scheme > CRUNA_FILTER_O10_E_C_P) {
    err = "unknown filter scheme " + std::to_string(scheme);
    return false;
  }
  op.kind = OP_STENCIL;
  filter_interior(scheme, scheme == CRUNA_FILTER_O10_E_C_P ? 0.0 : alpha, op);
  const int minn = 2 * op.r + 1;
  if (n < minn) {
    err = "filter scheme " + std::to_string(scheme) + " needs at least " + std::to_string(minn) +
          " points, got " + std::to_string(n);
    return false;
  }
  switch (scheme) {
    case CRUNA_FILTER_O10_E_C_P:               // no reference counterpart: explicit + blend
      op.periodic = 1;
      op.blend = strength;
      return true;
    case CRUNA_FILTER_O2_I_C_P:
    case CRUNA_FILTER_O6_I_C_P:                // filter_pen_core_o6_i_c_p.f90:184-249
      op.periodic = 1; op.solve = 1; op.cyclic = 1;
      cyclic_factors(hf, n, alpha, 1.0);
      break;
    case CRUNA_FILTER_O2_I_C_O:                // filter_pen_core_o2_i_c_o.f90 (cyclic correction)
      filter_rows(scheme, alpha, op);
      op.solve = 1; op.cyclic = 1;
      cyclic_factors(hf, n, alpha, 1.0);
      break;
    default:                                   // o4/o6/o8/o10 open: filter_pen_core_o10_i_c_o.f90:284-294
      filter_rows(scheme, alpha, op);
      op.solve = 1;
      hf.dl.assign(n - 1, alpha);
      hf.d.assign(n, 1.0);
      hf.du.assign(n - 1, alpha);
      hf.du[0] = 0.0;
      hf.dl[n - 2] = 0.0;
      factor(hf, n);
      break;
  }
  if (hf.info != 0) {
    err = "dgttrf failed (info=" + std::to_string(hf.info) + ")";
    return false;
  }
  return true;
}

}  // namespace cruna
