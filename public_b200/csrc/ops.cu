// Generic kernels of the CRUNA B200 library: line operators (derivatives and filters of any
// reference scheme along any direction), boundary conditions, RK4 stage updates and the generic
// RHS sequences that mirror src/equations/ns_rho_rhou_p.f90 call by call.
#include <cmath>
#include <stdexcept>
#include <string>

#include "bc_point.cuh"
#include "cruna_internal.cuh"
#include "ops_common.cuh"

namespace cruna {

__global__ void k_line_stencil(LineOp op, Grid g, int dir, const double *__restrict__ f1,
                               const double *__restrict__ f2, double *__restrict__ out, double scale,
                               double sign, int nfields) {
  const long long total = g.N * nfields;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long fld = t / g.N, p = t - fld * g.N;
    long long base, s;
    int i;
    line_geom(g, dir, p, base, s, i);
    const double *a = f1 + fld * g.N;
    const double *b = f2 ? f2 + fld * g.N : nullptr;
    out[t] = sign * line_point(op, a, b, base, s, i, scale);
  }
}

// one thread per line: dgttrs('N') sweeps (pivots as LAPACK) + cyclic correction, in place
__global__ void k_line_solve(LineOp op, Grid g, int dir, double *__restrict__ data, int nfields) {
  const int n = op.n;
  const long long nlines = g.N / n;
  const long long total = nlines * nfields;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long fld = t / nlines, l = t - fld * nlines;
    long long base, s;
    if (dir == 0) { base = l * g.n1; s = 1; }
    else if (dir == 1) { const long long i = l % g.n1, k = l / g.n1; base = i + k * (long long)g.n1 * g.n2; s = g.n1; }
    else { base = l; s = (long long)g.n1 * g.n2; }
    double *b = data + fld * g.N + base;
    for (int i = 0; i < n - 1; ++i) {
      if (op.ipiv[i] == i + 1) {
        b[(i + 1) * s] = b[(i + 1) * s] - op.dl[i] * b[i * s];
      } else {
        const double temp = b[i * s];
        const double nxt = b[(i + 1) * s];
        b[i * s] = nxt;
        b[(i + 1) * s] = temp - op.dl[i] * nxt;
      }
    }
    double x2 = b[(n - 1) * s] * op.inv_d[n - 1];
    b[(n - 1) * s] = x2;
    double x1 = x2;
    if (n > 1) {
      x1 = (b[(n - 2) * s] - op.du[n - 2] * x2) * op.inv_d[n - 2];
      b[(n - 2) * s] = x1;
    }
    for (int i = n - 3; i >= 0; --i) {
      const double x0 = (b[i * s] - op.du[i] * x1 - op.du2[i] * x2) * op.inv_d[i];
      b[i * s] = x0;
      x2 = x1;
      x1 = x0;
    }
    if (op.cyclic) {
      const double corr = b[0] + op.fbrat * b[(n - 1) * s];
      for (int i = 0; i < n; ++i) b[i * s] = b[i * s] - op.fbnorm[i] * corr;
    }
  }
}

// ------------------------------------------------------------------------------------------------
// fast line operators: the same arithmetic as k_line_stencil / k_line_solve (identical expressions in
// identical order, so identical results), with the interior radius a compile-time constant, no
// integer division per tap, and for compact operators along y and z the explicit part and the
// dgttrs sweeps fused in one pass over each line
// ------------------------------------------------------------------------------------------------

// interior explicit part from values v(m) = f(i + m), m = -R..R, in explicit_part's order
template <int R, bool ANTI, class V>
__device__ __forceinline__ double interior_part(const LineOp &op, V v) {
  if (ANTI) {
    double t = op.c[1] * (v(1) - v(-1));
#pragma unroll
    for (int m = 2; m <= R; ++m) t = t + op.c[m] * (v(m) - v(-m));
    return t;
  }
  double t = op.c[0] * v(0);
#pragma unroll
  for (int m = 1; m <= R; ++m) t = t + op.c[m] * (v(m) + v(-m));
  return t;
}

// line_point's epilogue: derivative scale, filter blend, sign
__device__ __forceinline__ double point_epilogue(const LineOp &op, double v, double q, double scale,
                                                 double sign) {
  if (op.antisym) v = v * scale;  // every OP_STENCIL derivative
  if (op.blend > 0.0) v = q - op.blend * (q - v);
  return sign * v;
}

// one thread per KB points stacked in z: x from the block's x range, j = blockIdx.y, the field and
// the z chunk from blockIdx.z (strided).  DIR and F2 (f1 * f2 operand) are compile-time, so a chunk
// whose taps all lie on its line (no periodic wrap, no closure row) reads them at fixed offsets from
// one pointer; the KB results are formed before any is stored, so the loads of all KB points are in
// flight together (and along z the shared taps are loaded once).  Other chunks take the generic path.
template <int R, bool ANTI, int DIR, bool F2>
__global__ void __launch_bounds__(128) k_line_stencil_r(LineOp op, Grid g, const __grid_constant__ FieldSet fs,
                                                        double scale, double sign) {
  const int nfields = fs.n;
  constexpr int KB = 4;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= g.n1) return;
  const long long n12 = (long long)g.n1 * g.n2;
  const int j = blockIdx.y;
  const int nkb = (g.n3 + KB - 1) / KB;
  const int n = op.n;
  const long long s = DIR == 0 ? 1 : (DIR == 1 ? (long long)g.n1 : n12);
  for (int zf = blockIdx.z; zf < nkb * nfields; zf += gridDim.z) {
    const int fld = zf / nkb, k0 = (zf - fld * nkb) * KB;
    const long long p0 = x + (long long)g.n1 * j + n12 * k0;
    const double *__restrict__ fa = fs.f1[fld];
    const double *__restrict__ fb = F2 ? fs.f2[fld] : nullptr;
    double *__restrict__ o = fs.out[fld] + p0;
    const int ilo = DIR == 0 ? x : (DIR == 1 ? j : k0), ihi = DIR == 2 ? k0 + KB - 1 : ilo;
    const int lo = op.periodic ? 0 : op.nb, hi = op.periodic ? n - 1 : n - 1 - op.nb;
    if (k0 + KB <= g.n3 && ilo - R >= 0 && ihi + R <= n - 1 && ilo >= lo && ihi <= hi) {
      const double *a = fa + p0;
      const double *b = F2 ? fb + p0 : nullptr;
      double r[KB];
#pragma unroll
      for (int u = 0; u < KB; ++u) {
        const double *au = a + u * n12;
        const double *bu = F2 ? b + u * n12 : nullptr;
        auto val = [&](int m) { return F2 ? au[m * s] * bu[m * s] : au[m * s]; };
        const double v = interior_part<R, ANTI>(op, val);
        r[u] = point_epilogue(op, v, op.blend > 0.0 ? val(0) : 0.0, scale, sign);
      }
#pragma unroll
      for (int u = 0; u < KB; ++u) o[u * n12] = r[u];
      continue;
    }
    const int kend = min(k0 + KB, g.n3);
    for (int k = k0; k < kend; ++k) {
      const long long p = p0 + (k - k0) * n12;
      const int i = DIR == 0 ? x : (DIR == 1 ? j : k);
      const long long base = p - (long long)i * s;
      const double *a = fa + base;
      const double *b = F2 ? fb + base : nullptr;
      double v;
      if (op.periodic) {
        v = interior_part<R, ANTI>(op, [&](int m) {
          int ii = i + m;
          ii = ii < 0 ? ii + n : (ii >= n ? ii - n : ii);
          return ldv(a, b, ii * s);
        });
      } else if (i >= op.nb && i < n - op.nb) {
        v = interior_part<R, ANTI>(op, [&](int m) { return ldv(a, b, (i + m) * s); });
      } else {
        v = explicit_part(op, a, b, 0, s, i);
      }
      o[(k - k0) * n12] = point_epilogue(op, v, op.blend > 0.0 ? ldv(a, b, i * s) : 0.0, scale, sign);
    }
  }
}

// Compact operators along y or z: one thread per line, consecutive threads on consecutive x (every
// load and store coalesced).  The operator's factors sit in shared memory (the same for every line).
// EXPL: the explicit part comes from a sliding window of f over the interior (one new load per point;
// the closure rows of open lines use explicit_part) and dgttrs's forward sweep runs on the fly;
// otherwise the line of `out` is solved in place.  Then the backward sweep and the cyclic correction
// over the stored forward values.  Every sweep reads its line CH points at a time and issues the next
// chunk's loads before it works through the current one, so two chunks' loads are in flight.
constexpr int kCompactMaxN = 1024;  // factors in shared memory: 44 bytes per line point

template <int R, bool ANTI, bool EXPL, bool NOPIV>
__global__ void __launch_bounds__(64) k_line_compact_yz(LineOp op, Grid g, int dir,
                                                        const double *__restrict__ f1,
                                                        const double *__restrict__ f2, double *out,
                                                        double scale, double sign, int nfields) {
  constexpr int CH = 8;
  constexpr int W = 2 * R + 1;
  extern __shared__ double cs[];
  const int n = op.n;
  double *s_dl = cs, *s_du = cs + n, *s_du2 = cs + 2 * n, *s_inv = cs + 3 * n, *s_fb = cs + 4 * n;
  int *s_piv = reinterpret_cast<int *>(cs + 5 * n);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    s_dl[i] = i < n - 1 ? op.dl[i] : 0.0;
    s_du[i] = i < n - 1 ? op.du[i] : 0.0;
    s_du2[i] = i < n - 2 ? op.du2[i] : 0.0;
    s_inv[i] = op.inv_d[i];
    s_fb[i] = op.cyclic ? op.fbnorm[i] : 0.0;
    s_piv[i] = NOPIV ? i + 1 : op.ipiv[i];
  }
  __syncthreads();
  const long long n12 = (long long)g.n1 * g.n2;
  const long long nlines = g.N / n;
  const long long total = nlines * nfields;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long fld = t / nlines, l = t - fld * nlines;
    long long base, s;
    if (dir == 1) { const long long i = l % g.n1, k = l / g.n1; base = i + k * n12; s = g.n1; }
    else { base = l; s = n12; }
    double *o = out + fld * g.N + base;
    double *po = o;  // o[(i - 1) * s] for the forward step at i
    double cur = 0.0;
    // dgttrs forward sweep (L with LAPACK's row interchanges) on the pair (i - 1, i); v = b[i]
    auto fwd = [&](int i, double v) {
      if (i == 0) {
        cur = v;
        return;
      }
      if (NOPIV || s_piv[i - 1] == i) {
        *po = cur;
        cur = v - s_dl[i - 1] * cur;
      } else {
        *po = v;
        cur = cur - s_dl[i - 1] * v;
      }
      po += s;
    };
    if (EXPL) {
      const double *a = f1 + fld * g.N + base;
      const double *b = f2 ? f2 + fld * g.N + base : nullptr;
      const int ib = op.periodic ? 0 : op.nb, ie = op.periodic ? n : n - op.nb;
      for (int i = 0; i < ib; ++i)
        fwd(i, point_epilogue(op, explicit_part(op, a, b, 0, s, i), ldv(a, b, i * s), scale, sign));
      auto wrap = [&](int idx) { return op.periodic ? (idx < 0 ? idx + n : (idx >= n ? idx - n : idx)) : idx; };
      double w[W];  // w[R + m] = f(i + m)
#pragma unroll
      for (int m = 0; m < W; ++m) w[m] = ldv(a, b, wrap(ib + m - R) * s);
      auto step = [&](int i, double next) {  // position i from the window, then slide it by one
        const double v = interior_part<R, ANTI>(op, [&](int m) { return w[R + m]; });
        fwd(i, point_epilogue(op, v, w[R], scale, sign));
#pragma unroll
        for (int m = 0; m < W - 1; ++m) w[m] = w[m + 1];
        w[W - 1] = next;
      };
      // chunk at i0 needs f(i0 + u + 1 + R), u < CH, while i0 + u + 1 < ie
      int i0 = ib;
      double nx[CH];
      if (i0 + CH <= ie) {
#pragma unroll
        for (int u = 0; u < CH; ++u) nx[u] = (i0 + u + 1 < ie) ? ldv(a, b, wrap(i0 + u + 1 + R) * s) : 0.0;
      }
      for (; i0 + CH <= ie; i0 += CH) {
        double cb[CH];
#pragma unroll
        for (int u = 0; u < CH; ++u) cb[u] = nx[u];
        if (i0 + 2 * CH <= ie) {
#pragma unroll
          for (int u = 0; u < CH; ++u)
            nx[u] = (i0 + CH + u + 1 < ie) ? ldv(a, b, wrap(i0 + CH + u + 1 + R) * s) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < CH; ++u) step(i0 + u, cb[u]);
      }
      for (; i0 < ie; ++i0) step(i0, (i0 + 1 < ie) ? ldv(a, b, wrap(i0 + 1 + R) * s) : 0.0);
      for (int i = ie; i < n; ++i)
        fwd(i, point_epilogue(op, explicit_part(op, a, b, 0, s, i), ldv(a, b, i * s), scale, sign));
    } else {
      cur = o[0];
      const double *pl = o + s;  // o[i0 * s]
      int i0 = 1;
      double nx[CH];
      if (i0 + CH <= n) {
#pragma unroll
        for (int u = 0; u < CH; ++u) nx[u] = pl[(long long)u * s];
      }
      for (; i0 + CH <= n; i0 += CH) {
        double cb[CH];
#pragma unroll
        for (int u = 0; u < CH; ++u) cb[u] = nx[u];
        pl += CH * s;
        if (i0 + 2 * CH <= n) {
#pragma unroll
          for (int u = 0; u < CH; ++u) nx[u] = pl[(long long)u * s];
        }
#pragma unroll
        for (int u = 0; u < CH; ++u) fwd(i0 + u, cb[u]);
      }
      for (; i0 < n; ++i0, pl += s) fwd(i0, *pl);
    }
    // backward sweep with U (diagonal inverted, du, du2); po now points at o[(n - 1) * s]
    double x2 = cur * s_inv[n - 1];
    *po = x2;
    const double xlast = x2;
    double x1 = (po[-s] - s_du[n - 2] * x2) * s_inv[n - 2];  // n > 2R + 2 >= 4
    po -= s;
    *po = x1;
    auto back = [&](int i, double bi) {
      const double x0 = (bi - s_du[i] * x1 - s_du2[i] * x2) * s_inv[i];
      po -= s;
      *po = x0;
      x2 = x1;
      x1 = x0;
    };
    int i0 = n - 3;  // chunk at i0 reads positions i0 - u = po[-(u + 1) s]
    double nb[CH];
    if (i0 >= CH - 1) {
#pragma unroll
      for (int u = 0; u < CH; ++u) nb[u] = po[-(long long)(u + 1) * s];
    }
    for (; i0 >= CH - 1; i0 -= CH) {
      double cb[CH];
#pragma unroll
      for (int u = 0; u < CH; ++u) cb[u] = nb[u];
      if (i0 - CH >= CH - 1) {
#pragma unroll
        for (int u = 0; u < CH; ++u) nb[u] = po[-(long long)(CH + u + 1) * s];
      }
#pragma unroll
      for (int u = 0; u < CH; ++u) back(i0 - u, cb[u]);
    }
    for (; i0 >= 0; --i0) back(i0, po[-s]);
    if (op.cyclic) {  // Sherman-Morrison: x1 is the solution's first value, xlast its last
      const double corr = x1 + op.fbrat * xlast;
      for (int j0 = 0; j0 < n; j0 += CH) {
        double bv[CH];
#pragma unroll
        for (int u = 0; u < CH; ++u) bv[u] = (j0 + u < n) ? o[(long long)(j0 + u) * s] : 0.0;
#pragma unroll
        for (int u = 0; u < CH; ++u)
          if (j0 + u < n) o[(long long)(j0 + u) * s] = bv[u] - s_fb[j0 + u] * corr;
      }
    }
  }
}

static size_t compact_smem(const LineOp &op) { return (size_t)op.n * (5 * sizeof(double) + sizeof(int)); }


// the fast kernels handle interior radii 1..6 on lines longer than 2R + 2 (every periodic wrap then
// stays within one period) whose open ends have at least R closure rows and an interior between them
// (interior taps stay on the line)
static bool fast_ok(const LineOp &op) {
  return op.kind == OP_STENCIL && op.r >= 1 && op.r <= 6 && op.n > 2 * op.r + 2 &&
         (op.periodic || (op.nb >= op.r && op.n >= 2 * op.nb + 2 * op.r + 1));
}

template <int R, bool ANTI, int DIR>
static void launch_stencil_dir(cruna_ctx *c, const LineOp &op, const FieldSet &fs, double scale, double sign) {
  const int bx = c->g.n1 >= 128 ? 128 : (c->g.n1 >= 64 ? 64 : 32);
  const dim3 grid((c->g.n1 + bx - 1) / bx, c->g.n2, std::min((c->g.n3 + 3) / 4 * fs.n, 65535));
  if (fs.f2[0])
    k_line_stencil_r<R, ANTI, DIR, true><<<grid, bx, 0, c->stream>>>(op, c->g, fs, scale, sign);
  else
    k_line_stencil_r<R, ANTI, DIR, false><<<grid, bx, 0, c->stream>>>(op, c->g, fs, scale, sign);
}

template <int R, bool ANTI>
static void launch_stencil_rr(cruna_ctx *c, const LineOp &op, int dir, const FieldSet &fs, double scale,
                              double sign) {
  if (dir == 0) launch_stencil_dir<R, ANTI, 0>(c, op, fs, scale, sign);
  else if (dir == 1) launch_stencil_dir<R, ANTI, 1>(c, op, fs, scale, sign);
  else launch_stencil_dir<R, ANTI, 2>(c, op, fs, scale, sign);
}

template <bool ANTI>
static void launch_stencil_r(cruna_ctx *c, const LineOp &op, int dir, const FieldSet &fs, double scale,
                             double sign) {
  switch (op.r) {
    case 1: launch_stencil_rr<1, ANTI>(c, op, dir, fs, scale, sign); break;
    case 2: launch_stencil_rr<2, ANTI>(c, op, dir, fs, scale, sign); break;
    case 3: launch_stencil_rr<3, ANTI>(c, op, dir, fs, scale, sign); break;
    case 4: launch_stencil_rr<4, ANTI>(c, op, dir, fs, scale, sign); break;
    case 5: launch_stencil_rr<5, ANTI>(c, op, dir, fs, scale, sign); break;
    case 6: launch_stencil_rr<6, ANTI>(c, op, dir, fs, scale, sign); break;
  }
}

template <bool ANTI>
static void launch_compact_r(cruna_ctx *c, const LineOp &op, int dir, const double *f1, const double *f2,
                             double *out, double scale, double sign, int nfields) {
  const long long lines = (c->g.N / op.n) * nfields;
  const int blocks = nblocks(lines, 64);  // one line per thread: small blocks spread few lines over all SMs
  const size_t sm = compact_smem(op);
  switch (op.r) {
#define CRUNA_COMPACT_CASE(RR)                                                                          \
  case RR:                                                                                              \
    if (op.nopiv)                                                                                       \
      k_line_compact_yz<RR, ANTI, true, true><<<blocks, 64, sm, c->stream>>>(op, c->g, dir, f1, f2, out, scale, \
                                                                             sign, nfields);            \
    else                                                                                                \
      k_line_compact_yz<RR, ANTI, true, false><<<blocks, 64, sm, c->stream>>>(op, c->g, dir, f1, f2, out, scale, \
                                                                              sign, nfields);           \
    break;
    CRUNA_COMPACT_CASE(1) CRUNA_COMPACT_CASE(2) CRUNA_COMPACT_CASE(3)
    CRUNA_COMPACT_CASE(4) CRUNA_COMPACT_CASE(5) CRUNA_COMPACT_CASE(6)
#undef CRUNA_COMPACT_CASE
  }
}

// contiguous fields f1 + k N (f2 + k N), out + k N, k < nfields, as field sets of at most kMax
template <class F>
static void for_sets(const cruna_ctx *c, const double *f1, const double *f2, double *out, int nfields, F &&fn) {
  for (int k0 = 0; k0 < nfields; k0 += FieldSet::kMax) {
    FieldSet fs;
    for (int k = k0; k < std::min(nfields, k0 + FieldSet::kMax); ++k)
      fs.add(f1 + (long long)k * c->g.N, f2 ? f2 + (long long)k * c->g.N : nullptr, out + (long long)k * c->g.N);
    fn(fs);
  }
}

static const char *const kStencilNames[2][3] = {{"line_filter_x", "line_filter_y", "line_filter_z"},
                                                {"line_diff_x", "line_diff_y", "line_diff_z"}};

static bool stencil_fast(const cruna_ctx *c, const LineOp &op) { return fast_ok(op) && c->g.n2 <= 65535; }
static bool compact_fast(const LineOp &op, int dir) {
  return op.kind == OP_STENCIL && op.solve && dir > 0 && fast_ok(op) && op.n <= kCompactMaxN;
}

static void launch_stencil_set(cruna_ctx *c, const LineOp &op, int dir, const FieldSet &fs, double scale,
                               double sign) {
  ProfScope ps(c, kStencilNames[op.antisym ? 1 : 0][dir]);
  if (op.antisym) launch_stencil_r<true>(c, op, dir, fs, scale, sign);
  else launch_stencil_r<false>(c, op, dir, fs, scale, sign);
  CRUNA_LAUNCH_CHECK(c);
}

void launch_line_stencil(cruna_ctx *c, const LineOp &op, int dir, const double *f1, const double *f2,
                         double *out, double scale, int nfields, double sign) {
  if (stencil_fast(c, op)) {
    for_sets(c, f1, f2, out, nfields, [&](const FieldSet &fs) { launch_stencil_set(c, op, dir, fs, scale, sign); });
    return;
  }
  ProfScope ps(c, kStencilNames[op.antisym ? 1 : 0][dir]);
  const long long work = c->g.N * nfields;
  const int blocks = (int)std::min<long long>(nblocks(work), 148LL * 64);
  k_line_stencil<<<blocks, kThreads, 0, c->stream>>>(op, c->g, dir, f1, f2, out, scale, sign, nfields);
  CRUNA_LAUNCH_CHECK(c);
}

void launch_line_solve(cruna_ctx *c, const LineOp &op, int dir, double *data, int nfields) {
  static const char *names[3] = {"line_solve_x", "line_solve_y", "line_solve_z"};
  ProfScope ps(c, names[dir]);
  const long long lines = (c->g.N / op.n) * nfields;
  if (dir > 0 && op.n >= 4 && op.n <= kCompactMaxN) {
    if (op.nopiv)
      k_line_compact_yz<1, false, false, true><<<nblocks(lines, 64), 64, compact_smem(op), c->stream>>>(
          op, c->g, dir, nullptr, nullptr, data, 1.0, 1.0, nfields);
    else
      k_line_compact_yz<1, false, false, false><<<nblocks(lines, 64), 64, compact_smem(op), c->stream>>>(
          op, c->g, dir, nullptr, nullptr, data, 1.0, 1.0, nfields);
    CRUNA_LAUNCH_CHECK(c);
    return;
  }
  k_line_solve<<<nblocks(lines, 128), 128, 0, c->stream>>>(op, c->g, dir, data, nfields);
  CRUNA_LAUNCH_CHECK(c);
}

// explicit part and compact solve of op along y or z in one pass (compact_fast(op, dir)) on nfields
// contiguous fields
static void launch_line_compact(cruna_ctx *c, const LineOp &op, int dir, const double *f1, const double *f2,
                                double *out, double scale, int nfields) {
  static const char *names[2][3] = {{"", "compact_filter_y", "compact_filter_z"},
                                    {"", "compact_diff_y", "compact_diff_z"}};
  ProfScope ps(c, names[op.antisym ? 1 : 0][dir]);
  if (op.antisym) launch_compact_r<true>(c, op, dir, f1, f2, out, scale, 1.0, nfields);
  else launch_compact_r<false>(c, op, dir, f1, f2, out, scale, 1.0, nfields);
  CRUNA_LAUNCH_CHECK(c);
}

// Dx_d of each field of a set (f1, or f1*f2 when every f2 is given), all with the same spacing h:
// explicit operators take one launch per set; compact ones (whose kernel keeps one line per thread in
// flight, so more fields per launch do not shorten it) and the fallbacks one apply_diff per field
void apply_diff_set(cruna_ctx *c, int dir, const FieldSet &fs, double h) {
  const LineOp &op = c->dop[dir];
  const double scale = 1.0 / (h * op.div);
  bool uniform = true;
  for (int k = 1; k < fs.n; ++k) uniform = uniform && ((fs.f2[k] != nullptr) == (fs.f2[0] != nullptr));
  if (uniform && !op.solve && stencil_fast(c, op)) {
    launch_stencil_set(c, op, dir, fs, scale, 1.0);
  } else {
    for (int k = 0; k < fs.n; ++k) apply_diff(c, dir, fs.f1[k], fs.f2[k], fs.out[k], h, 1);
  }
}

// Dx_d of f1 (or of f1*f2): explicit part scaled by 1/(h*div), then the compact solve if any
void apply_diff(cruna_ctx *c, int dir, const double *f1, const double *f2, double *out, double h,
                int nfields) {
  const LineOp &op = c->dop[dir];
  const double scale = 1.0 / (h * op.div);
  if (compact_fast(op, dir)) {
    launch_line_compact(c, op, dir, f1, f2, out, scale, nfields);
    return;
  }
  launch_line_stencil(c, op, dir, f1, f2, out, scale, nfields);
  if (op.kind == OP_STENCIL && op.solve) launch_line_solve(c, op, dir, out, nfields);
}

// filter_i_d in place: out-of-place stencil into scratch, solve, copy back
void apply_filter(cruna_ctx *c, int dir, double *q, double *scratch, int nfields) {
  const LineOp &op = c->fop[dir];
  if (op.kind == OP_COPY) return;
  if (compact_fast(op, dir)) {
    launch_line_compact(c, op, dir, q, nullptr, scratch, 1.0, nfields);
  } else {
    launch_line_stencil(c, op, dir, q, nullptr, scratch, 1.0, nfields);
    if (op.solve) launch_line_solve(c, op, dir, scratch, nfields);
  }
  CRUNA_CUDA_CHECK(cudaMemcpyAsync(q, scratch, sizeof(double) * c->g.N * nfields,
                                   cudaMemcpyDeviceToDevice, c->stream));
}

// ------------------------------------------------------------------------------------------------
// boundary kernels
// ------------------------------------------------------------------------------------------------

// characteristic_q_k1d (src/boundaries/nonreflecting.f90:46-137) -- aim from `aim` at p + aim_off
__global__ void k_char_q(Box b, Grid g, double k1, double k2, double k3, double gamma, double *q,
                         const double *aim, long long aim_off) {
  const long long tot = b.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const long long p = box_point(b, g, t, i, j, k);
    const long long N = g.N, pa = p + aim_off;
    double qv[5], av[5], out[5];
    for (int v = 0; v < 5; ++v) {
      qv[v] = q[p + v * N];
      av[v] = aim[pa + v * N];
    }
    char_q_point(qv, av, k1, k2, k3, gamma, out);
    for (int v = 0; v < 5; ++v) q[p + v * N] = out[v];
  }
}

// characteristic_qs_k1d (nonreflecting.f90:453-554); q sampled at p + q_off
__global__ void k_char_qs(Box b, Grid g, double k1, double k2, double k3, double gamma, double *qs,
                          const double *q, long long q_off) {
  const long long tot = b.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const long long p = box_point(b, g, t, i, j, k);
    const long long N = g.N, pq = p + q_off;
    double sv[5], qv[5], out[5];
    for (int v = 0; v < 5; ++v) {
      sv[v] = qs[p + v * N];
      qv[v] = q[pq + v * N];
    }
    char_qs_point(sv, qv, k1, k2, k3, gamma, out);
    for (int v = 0; v < 5; ++v) qs[p + v * N] = out[v];
  }
}

// characteristic_rhs_k1d without shape (nonreflecting.f90:237-341), BC type 204
__global__ void k_char_rhs(Box b, Grid g, double k1, double k2, double k3, double gamma, double dt,
                           double *rhs, const double *q, const double *aim) {
  const long long tot = b.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const long long p = box_point(b, g, t, i, j, k);
    const long long N = g.N;
    double rv[5], qv[5], av[5], out[5];
    for (int v = 0; v < 5; ++v) {
      rv[v] = rhs[p + v * N];
      qv[v] = q[p + v * N];
      av[v] = aim[p + v * N];
    }
    char_rhs_point(rv, qv, av, k1, k2, k3, gamma, dt, out);
    for (int v = 0; v < 5; ++v) rhs[p + v * N] = out[v];
  }
}

// zonal variants with a normal vector per point (nonreflecting.f90:141-233, :345-449, :558-661): types
// 202 / 205 on their box, 203 / 206 on the whole block weighted by the sponge shape
__global__ void k_char_q4(Box b, Grid g, const double *__restrict__ kv, SpongeDev sp, int shaped, double gamma,
                          double *q, const double *aim) {
  const long long tot = b.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const long long p = box_point(b, g, t, i, j, k);
    const long long N = g.N;
    double qv[5], av[5], out[5];
    for (int v = 0; v < 5; ++v) {
      qv[v] = q[p + v * N];
      av[v] = aim[p + v * N];
    }
    char_q_point(qv, av, kv[p], kv[p + N], kv[p + 2 * N], gamma, out, shaped ? sponge_at(sp, g, p) : 1.0);
    for (int v = 0; v < 5; ++v) q[p + v * N] = out[v];
  }
}

__global__ void k_char_qs4(Box b, Grid g, const double *__restrict__ kv, SpongeDev sp, int shaped, double gamma,
                           double *qs, const double *q) {
  const long long tot = b.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const long long p = box_point(b, g, t, i, j, k);
    const long long N = g.N;
    double sv[5], qv[5], out[5];
    for (int v = 0; v < 5; ++v) {
      sv[v] = qs[p + v * N];
      qv[v] = q[p + v * N];
    }
    char_qs_point(sv, qv, kv[p], kv[p + N], kv[p + 2 * N], gamma, out, shaped ? sponge_at(sp, g, p) : 1.0);
    for (int v = 0; v < 5; ++v) qs[p + v * N] = out[v];
  }
}

__global__ void k_char_rhs4(Box b, Grid g, const double *__restrict__ kv, SpongeDev sp, int shaped, double gamma,
                            double dt, double *rhs, const double *q, const double *aim) {
  const long long tot = b.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const long long p = box_point(b, g, t, i, j, k);
    const long long N = g.N;
    double rv[5], qv[5], av[5], out[5];
    for (int v = 0; v < 5; ++v) {
      rv[v] = rhs[p + v * N];
      qv[v] = q[p + v * N];
      av[v] = aim[p + v * N];
    }
    char_rhs_point(rv, qv, av, kv[p], kv[p + N], kv[p + 2 * N], gamma, dt, out, shaped != 0,
                   shaped ? sponge_at(sp, g, p) : 0.0);
    for (int v = 0; v < 5; ++v) rhs[p + v * N] = out[v];
  }
}

// boundary normal vectors (init_orthogonal_and_diagonal_kvector, init_orthogonal_kvector,
// init_hedgehog_kvector, normalize_kvector: boundary_normal_vector.f90:37-261)
__global__ void k_kvector(Grid g, int kind, double x00, double x01, double x02, double L0, double L1, double L2,
                          double dx0, double dx1, double dx2, double *kv) {
  const long long N = g.N;
  const double half = 0.5 * fmin(fmin(dx0 / L0, dx1 / L1), dx2 / L2);
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    const long long i = p % g.n1, j = (p / g.n1) % g.n2, k = p / ((long long)g.n1 * g.n2);
    const double X[3] = {x00 + (g.n1 > 1 ? (double)i * dx0 : 0.0), x01 + (g.n2 > 1 ? (double)j * dx1 : 0.0),
                         x02 + (g.n3 > 1 ? (double)k * dx2 : 0.0)};
    const double Lv[3] = {L0, L1, L2};
    double kk[3];
    for (int d = 0; d < 3; ++d) kk[d] = X[d] - (x00 * (d == 0) + x01 * (d == 1) + x02 * (d == 2) + 0.5 * Lv[d]);
    bool normalize = true;
    if (kind != 2) {
      for (int d = 0; d < 3; ++d) kk[d] = kk[d] / Lv[d];
      const double a[3] = {fabs(kk[0]), fabs(kk[1]), fabs(kk[2])};
      const double m = fmax(fmax(a[0], a[1]), a[2]);
      const int dom = (m == a[0]) ? 0 : ((m == a[1]) ? 1 : 2);
      for (int d = 0; d < 3; ++d) {
        if (d == dom) kk[d] = copysign(1.0, kk[d]);
        else if (kind == 0 && m - a[d] < half) kk[d] = copysign(1.0, kk[d]);
        else kk[d] = 0.0;
      }
      normalize = (kind == 0);
    }
    if (normalize) {
      const double r = sqrt(kk[0] * kk[0] + kk[1] * kk[1] + kk[2] * kk[2]);
      for (int d = 0; d < 3; ++d) kk[d] = kk[d] / r;
    }
    for (int d = 0; d < 3; ++d) kv[p + d * N] = kk[d];
  }
}

void build_kvector(cruna_ctx *c) {
  const double L[3] = {c->cfg.x1[0] - c->cfg.x0[0], c->cfg.x1[1] - c->cfg.x0[1], c->cfg.x1[2] - c->cfg.x0[2]};
  k_kvector<<<(int)std::min<long long>(nblocks(c->g.N), 148LL * 32), kThreads, 0, c->stream>>>(
      c->g, c->cfg.kvector, c->cfg.x0[0], c->cfg.x0[1], c->cfg.x0[2], L[0], L[1], L[2], c->dx[0], c->dx[1],
      c->dx[2], c->kvec);
  CRUNA_LAUNCH_CHECK(c);
}

// wall_slip_no_thermodynamics (src/boundaries/wall_boundary_conditions.f90:13-23)
__global__ void k_wall(Box b, Grid g, int comp, double *rhs) {
  const long long tot = b.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const long long p = box_point(b, g, t, i, j, k);
    rhs[p + comp * g.N] = 0.0;
  }
}

// sponge_rhs / sponge_q / sponge_qs / sponge_rhss_correct (src/boundaries/sponge_layer_core.f90)
__global__ void k_sponge(int mode, Grid g, SpongeDev sp, double gamma, double *a, const double *b,
                         const double *qref) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.N;
       p += (long long)gridDim.x * blockDim.x) {
    const double sh = sponge_at(sp, g, p);
    // outside the sponge layers the shape is exactly 0 and every update below leaves a unchanged
    // (for finite values), so those points are not read or written
    if (sh == 0.0) continue;
    const long long N = g.N;
    if (mode == 0) {          // rhs -= shape*(q - qref): a = rhs, b = q
      for (int v = 0; v < 5; ++v) a[p + v * N] = a[p + v * N] - sh * (b[p + v * N] - qref[p + v * N]);
    } else if (mode == 1) {   // q -= shape*(q - qref): a = q
      for (int v = 0; v < 5; ++v) a[p + v * N] = a[p + v * N] - sh * (a[p + v * N] - qref[p + v * N]);
    } else if (mode == 2) {   // qs -= shape*qs
      for (int v = 0; v < 5; ++v) a[p + v * N] = a[p + v * N] - sh * a[p + v * N];
    } else {                  // rhss += shape*(-(A^T)^-1 C^T qs): a = rhss, b = qs, qref = q
      const double *q = qref;
      const double rho = q[p];
      const double u0 = q[p + N] / rho, u1 = q[p + 2 * N] / rho, u2 = q[p + 3 * N] / rho;
      const double s0 = 1.0 * b[p] - u0 / rho * b[p + N] - u1 / rho * b[p + 2 * N] - u2 / rho * b[p + 3 * N];
      const double s1 = 1.0 / rho * b[p + N];
      const double s2 = 1.0 / rho * b[p + 2 * N];
      const double s3 = 1.0 / rho * b[p + 3 * N];
      const double s4 = (gamma - 1.0) * b[p + 4 * N];
      a[p] += sh * s0;
      a[p + N] += sh * s1;
      a[p + 2 * N] += sh * s2;
      a[p + 3 * N] += sh * s3;
      a[p + 4 * N] += sh * s4;
    }
  }
}

void bc_q(cruna_ctx *c, double *q, int outside) {
  ProfScope ps(c, "boundary");
  for (const BCRow &r : c->bc) {
    Box b = box_of(r);
    const int blocks = nblocks(b.count());
    if (r.type == 200) {
      k_char_q<<<blocks, kThreads, 0, c->stream>>>(b, c->g, r.k[0], r.k[1], r.k[2], c->cfg.gamma, q, q,
                                                   offset_of(c, r.shift));
      CRUNA_LAUNCH_CHECK(c);
    } else if (r.type == 201) {
      k_char_q<<<blocks, kThreads, 0, c->stream>>>(b, c->g, r.k[0], r.k[1], r.k[2], c->cfg.gamma, q,
                                                   c->qref, 0);
      CRUNA_LAUNCH_CHECK(c);
    } else if (r.type == 401) {
      k_sponge<<<nblocks(c->g.N), kThreads, 0, c->stream>>>(1, c->g, c->sponge, c->cfg.gamma, q, nullptr,
                                                             c->qref);
      CRUNA_LAUNCH_CHECK(c);
    } else if (r.type == 202 || (r.type == 203 && (outside ? r.only != 1 : r.only != -1))) {
      k_char_q4<<<blocks, kThreads, 0, c->stream>>>(b, c->g, c->kvec, c->sponge, r.type == 203, c->cfg.gamma, q,
                                                    c->qref);
      CRUNA_LAUNCH_CHECK(c);
    }
  }
}

void bc_qs(cruna_ctx *c, double *qs, const double *q, int outside) {
  ProfScope ps(c, "boundary");
  for (const BCRow &r : c->bc) {
    Box b = box_of(r);
    const int blocks = nblocks(b.count());
    if (r.type == 200 || r.type == 201) {
      const long long off = r.type == 200 ? offset_of(c, r.shift) : 0;
      k_char_qs<<<blocks, kThreads, 0, c->stream>>>(b, c->g, r.k[0], r.k[1], r.k[2], c->cfg.gamma, qs, q,
                                                    off);
      CRUNA_LAUNCH_CHECK(c);
    } else if (r.type == 401) {
      k_sponge<<<nblocks(c->g.N), kThreads, 0, c->stream>>>(2, c->g, c->sponge, c->cfg.gamma, qs, nullptr,
                                                             nullptr);
      CRUNA_LAUNCH_CHECK(c);
    } else if (r.type == 202 || (r.type == 203 && (outside ? r.only != 1 : r.only != -1))) {
      k_char_qs4<<<blocks, kThreads, 0, c->stream>>>(b, c->g, c->kvec, c->sponge, r.type == 203, c->cfg.gamma, qs,
                                                     q);
      CRUNA_LAUNCH_CHECK(c);
    }
  }
}

void bc_rhs(cruna_ctx *c, double *rhs, const double *q) {
  ProfScope ps(c, "boundary");
  for (const BCRow &r : c->bc) {
    Box b = box_of(r);
    if (r.type == 100) {
      k_wall<<<nblocks(b.count()), kThreads, 0, c->stream>>>(b, c->g, r.comp, rhs);
      CRUNA_LAUNCH_CHECK(c);
    } else if (r.type == 204) {
      k_char_rhs<<<nblocks(b.count()), kThreads, 0, c->stream>>>(b, c->g, r.k[0], r.k[1], r.k[2],
                                                                c->cfg.gamma, c->cfg.dt, rhs, q, c->qref);
      CRUNA_LAUNCH_CHECK(c);
    } else if (r.type == 400) {
      k_sponge<<<nblocks(c->g.N), kThreads, 0, c->stream>>>(0, c->g, c->sponge, c->cfg.gamma, rhs, q,
                                                             c->qref);
      CRUNA_LAUNCH_CHECK(c);
    } else if (r.type == 205 || r.type == 206) {
      k_char_rhs4<<<nblocks(b.count()), kThreads, 0, c->stream>>>(b, c->g, c->kvec, c->sponge, r.type == 206,
                                                                 c->cfg.gamma, c->cfg.dt, rhs, q, c->qref);
      CRUNA_LAUNCH_CHECK(c);
    }
  }
}

void bc_rhss(cruna_ctx *c, double *rhss, const double *qs, const double *q) {
  ProfScope ps(c, "boundary");
  for (const BCRow &r : c->bc) {
    Box b = box_of(r);
    if (r.type == 100) {
      k_wall<<<nblocks(b.count()), kThreads, 0, c->stream>>>(b, c->g, r.comp, rhss);
      CRUNA_LAUNCH_CHECK(c);
    } else if (r.type == 400 && q != nullptr) {
      k_sponge<<<nblocks(c->g.N), kThreads, 0, c->stream>>>(3, c->g, c->sponge, c->cfg.gamma, rhss, qs, q);
      CRUNA_LAUNCH_CHECK(c);
    }
  }
}

// ------------------------------------------------------------------------------------------------
// RK4 stage update (src/time/rk_o4_e.f90:45-50 and :92-97): q_{s+1} = q0 + c*dt*k and the
// accumulation k1 + 2k2 + 2k3 + k4, finished by q1 = q0 + dt/6*acc
// ------------------------------------------------------------------------------------------------
__global__ void k_rk_stage(int stage, long long M, double dt, const double *__restrict__ k,
                           const double *__restrict__ q0, double *__restrict__ acc,
                           double *__restrict__ qn) {
  const double dth = dt * 0.5;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < M;
       p += (long long)gridDim.x * blockDim.x) {
    const double kv = k[p];
    if (stage == 1) {
      acc[p] = kv;
      qn[p] = q0[p] + dth * kv;
    } else if (stage == 2) {
      acc[p] = acc[p] + 2.0 * kv;
      qn[p] = q0[p] + dth * kv;
    } else if (stage == 3) {
      acc[p] = acc[p] + 2.0 * kv;
      qn[p] = q0[p] + dt * kv;
    } else {
      qn[p] = q0[p] + dt / 6.0 * (acc[p] + kv);
    }
  }
}

void rk_stage(cruna_ctx *c, int stage, double dt, const double *k, const double *q0, double *acc,
              double *qnext) {
  const long long M = c->g.N * 5;
  ProfScope ps(c, "rk_stage");
  k_rk_stage<<<(int)std::min<long long>(nblocks(M), 148LL * 32), kThreads, 0, c->stream>>>(stage, M, dt, k,
                                                                                           q0, acc, qnext);
  CRUNA_LAUNCH_CHECK(c);
}

void copy_state(cruna_ctx *c, double *dst, const double *src, int nfields) {
  if (dst == src) return;
  CRUNA_CUDA_CHECK(cudaMemcpyAsync(dst, src, sizeof(double) * c->g.N * nfields, cudaMemcpyDeviceToDevice,
                                   c->stream));
}

__global__ void k_add(long long M, double *dst, const double *src) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < M;
       p += (long long)gridDim.x * blockDim.x)
    dst[p] = dst[p] + src[p];
}

void add_fields(cruna_ctx *c, double *dst, const double *src, long long n) {
  k_add<<<(int)std::min<long long>(nblocks(n), 148LL * 32), kThreads, 0, c->stream>>>(n, dst, src);
  CRUNA_LAUNCH_CHECK(c);
}

// state check: flag bit 1 = non-finite, bit 2 = rho <= 0, bit 4 = p <= 0
__global__ void k_check(long long N, const double *q, int *flag) {
  int f = 0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    for (int v = 0; v < 5; ++v)
      if (!isfinite(q[p + v * N])) f |= 1;
    if (!(q[p] > 0.0)) f |= 2;
    if (!(q[p + 4 * N] > 0.0)) f |= 4;
  }
  if (f) atomicOr(flag, f);
}

int check_state(cruna_ctx *c, const double *q) {
  CRUNA_CUDA_CHECK(cudaMemsetAsync(c->flag, 0, sizeof(int), c->stream));
  k_check<<<(int)std::min<long long>(nblocks(c->g.N), 148LL * 16), kThreads, 0, c->stream>>>(c->g.N, q,
                                                                                             c->flag);
  CRUNA_LAUNCH_CHECK(c);
  int h = 0;
  CRUNA_CUDA_CHECK(cudaMemcpyAsync(&h, c->flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
  return h;
}

// ------------------------------------------------------------------------------------------------
// generic direct RHS: the call sequence of right_hand_side_direct_3d (ns_rho_rhou_p.f90:31-253)
// with the point-wise work fused into a few kernels
// ------------------------------------------------------------------------------------------------

__global__ void k_prim(long long N, const double *__restrict__ q, double *__restrict__ t, double WoR) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    const double r = q[p];
    t[p + F_U1 * N] = q[p + N] / r;          // ns_rho_rhou_p.f90:95-99
    t[p + F_U2 * N] = q[p + 2 * N] / r;
    t[p + F_U3 * N] = q[p + 3 * N] / r;
    t[p + F_T * N] = WoR * q[p + 4 * N] / r; // trafos.f90:57
  }
}

// mu, tau, lambda*grad T (ns_rho_rhou_p.f90:115-128, 193-197)
__global__ void k_visc(long long N, double *__restrict__ t, double mu0, double T0, double cp_over_pr) {
  const double S1 = 110.4;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    const double T = t[p + F_T * N];
    const double mu = mu0 * pow(T / T0, 1.5) * ((T0 + S1) / (T + S1));
    const double ux = t[p + F_UX * N], uy = t[p + F_UY * N], uz = t[p + F_UZ * N];
    const double vx = t[p + F_VX * N], vy = t[p + F_VY * N], vz = t[p + F_VZ * N];
    const double wx = t[p + F_WX * N], wy = t[p + F_WY * N], wz = t[p + F_WZ * N];
    const double mu_div = -(2.0 / 3.0 * mu * (ux + vy + wz));
    t[p + F_MU * N] = mu;
    t[p + F_T11 * N] = mu_div + 2 * mu * ux;
    t[p + F_T22 * N] = mu_div + 2 * mu * vy;
    t[p + F_T33 * N] = mu_div + 2 * mu * wz;
    t[p + F_T12 * N] = mu * (uy + vx);
    t[p + F_T13 * N] = mu * (uz + wx);
    t[p + F_T23 * N] = mu * (vz + wy);
    const double lam = mu * cp_over_pr;
    t[p + F_HX * N] = lam * t[p + F_TX * N];
    t[p + F_HY * N] = lam * t[p + F_TY * N];
    t[p + F_HZ * N] = lam * t[p + F_TZ * N];
  }
}

// assembly of the five equations in the reference's order (ns_rho_rhou_p.f90:131-209), + apply_force
__global__ void k_assemble(long long N, const double *__restrict__ t, double *__restrict__ rhs,
                           double gamma, const double *__restrict__ force) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
#define T_(f) t[p + (long long)(f) * N]
    double r1 = -T_(F_M1) - T_(F_M2) - T_(F_M3);
    double r2 = -T_(F_A1X) - T_(F_A1Y) - T_(F_A1Z) - T_(F_PX);
    r2 = r2 + T_(F_V1X) + T_(F_V1Y) + T_(F_V1Z);
    double r3 = -T_(F_A2X) - T_(F_A2Y) - T_(F_A2Z) - T_(F_PY);
    r3 = r3 + T_(F_V2X) + T_(F_V2Y) + T_(F_V2Z);
    double r4 = -T_(F_A3X) - T_(F_A3Y) - T_(F_A3Z) - T_(F_PZ);
    r4 = r4 + T_(F_V3X) + T_(F_V3Y) + T_(F_V3Z);
    const double gt = gamma / (gamma - 1.0);
    double r5 = gt * (-T_(F_EX) - T_(F_EY) - T_(F_EZ));
    r5 = r5 + T_(F_U1) * T_(F_PX) + T_(F_U2) * T_(F_PY) + T_(F_U3) * T_(F_PZ);
    r5 = r5 + T_(F_QX) + T_(F_QY) + T_(F_QZ);
    r5 = r5 + T_(F_T11) * T_(F_UX) + T_(F_T12) * T_(F_UY) + T_(F_T13) * T_(F_UZ) +
         T_(F_T12) * T_(F_VX) + T_(F_T22) * T_(F_VY) + T_(F_T23) * T_(F_VZ) +
         T_(F_T13) * T_(F_WX) + T_(F_T23) * T_(F_WY) + T_(F_T33) * T_(F_WZ);
    r5 = (gamma - 1.0) * r5;
#undef T_
    if (force) {
      r1 = r1 + force[p]; r2 = r2 + force[p + N]; r3 = r3 + force[p + 2 * N];
      r4 = r4 + force[p + 3 * N]; r5 = r5 + force[p + 4 * N];
    }
    rhs[p] = r1; rhs[p + N] = r2; rhs[p + 2 * N] = r3; rhs[p + 3 * N] = r4; rhs[p + 4 * N] = r5;
  }
}

void rhs_direct_generic(cruna_ctx *c, const double *q_in, double *rhs, double *qbc, int bc_mask) {
  const long long N = c->g.N;
  double *t = c->tmp;
  auto F = [&](int f) { return t + (long long)f * N; };
  const double *q = q_in;
  if (c->has_q_bc && (bc_mask & 1)) {                     // ns_rho_rhou_p.f90:89-92
    copy_state(c, qbc, q_in, 5);
    bc_q(c, qbc, 0);
    q = qbc;
  }
  const double *ru = q + N, *rv = q + 2 * N, *rw = q + 3 * N, *pp = q + 4 * N;
  const int blocks = (int)std::min<long long>(nblocks(N), 148LL * 32);
  k_prim<<<blocks, kThreads, 0, c->stream>>>(N, q, t, c->cfg.W / c->cfg.R);
  CRUNA_LAUNCH_CHECK(c);
  const double *dx = c->dx;
  // velocity gradients (:102-112), the three components of one direction in one launch
  for (int d = 0; d < 3; ++d) {
    FieldSet fs;
    for (int v = 0; v < 3; ++v) fs.add(F(F_U1 + v), nullptr, F(F_UX + 3 * v + d));
    apply_diff_set(c, d, fs, dx[d]);
  }
  // temperature gradient for the heat flux (:189-191), h absent unless heat_flux_dx
  for (int d = 0; d < 3; ++d)
    apply_diff(c, d, F(F_T), nullptr, F(F_TX + d), c->cfg.heat_flux_dx ? dx[d] : 1.0, 1);
  k_visc<<<blocks, kThreads, 0, c->stream>>>(N, t, c->cfg.mu0, c->cfg.T0,
                                             c->cfg.gamma * (c->cfg.R / c->cfg.W) / (c->cfg.gamma - 1.0) /
                                                 c->cfg.Pr);
  CRUNA_LAUNCH_CHECK(c);
  // mass (:131-133)
  apply_diff(c, 0, ru, nullptr, F(F_M1), dx[0], 1);
  apply_diff(c, 1, rv, nullptr, F(F_M2), dx[1], 1);
  apply_diff(c, 2, rw, nullptr, F(F_M3), dx[2], 1);
  // momentum (:138-177): fluxes q(:,:,:,1+d)*u_v and the stress divergence
  const int taus[3][3] = {{F_T11, F_T12, F_T13}, {F_T12, F_T22, F_T23}, {F_T13, F_T23, F_T33}};
  const int afl[3][3] = {{F_A1X, F_A1Y, F_A1Z}, {F_A2X, F_A2Y, F_A2Z}, {F_A3X, F_A3Y, F_A3Z}};
  const int vfl[3][3] = {{F_V1X, F_V1Y, F_V1Z}, {F_V2X, F_V2Y, F_V2Z}, {F_V3X, F_V3Y, F_V3Z}};
  const double *rq[3] = {ru, rv, rw};
  for (int d = 0; d < 3; ++d) {  // per direction: the three fluxes rho u_d u_v, then the stresses tau_vd
    FieldSet fl, st;
    for (int v = 0; v < 3; ++v) {
      fl.add(rq[d], F(F_U1 + v), F(afl[v][d]));
      st.add(F(taus[v][d]), nullptr, F(vfl[v][d]));
    }
    apply_diff_set(c, d, fl, dx[d]);
    apply_diff_set(c, d, st, dx[d]);
  }
  for (int v = 0; v < 3; ++v) apply_diff(c, v, pp, nullptr, F(F_PX + 7 * v), dx[v], 1);
  // pressure flux (:180-182) and heat flux divergence (:195-197)
  for (int d = 0; d < 3; ++d) apply_diff(c, d, pp, F(F_U1 + d), F(F_EX + d), dx[d], 1);
  for (int d = 0; d < 3; ++d)
    apply_diff(c, d, F(F_HX + d), nullptr, F(F_QX + d), c->cfg.heat_flux_dx ? dx[d] : 1.0, 1);
  k_assemble<<<blocks, kThreads, 0, c->stream>>>(N, t, rhs, c->cfg.gamma, c->force);
  CRUNA_LAUNCH_CHECK(c);
  if (c->has_rhs_bc && (bc_mask & 2)) bc_rhs(c, rhs, q);  // :218
}

// the forward part the discrete adjoint re-uses: u, T (:95-116), grad u, grad T, mu, tau, lambda grad T
// (:102-128, :189-191) and grad p (:145, :159, :173) into the generic workspace
void generic_forward_gradients(cruna_ctx *c, const double *q) {
  const long long N = c->g.N;
  double *t = c->tmp;
  auto F = [&](int f) { return t + (long long)f * N; };
  const int blocks = (int)std::min<long long>(nblocks(N), 148LL * 32);
  k_prim<<<blocks, kThreads, 0, c->stream>>>(N, q, t, c->cfg.W / c->cfg.R);
  CRUNA_LAUNCH_CHECK(c);
  const double *dx = c->dx;
  for (int d = 0; d < 3; ++d) {
    FieldSet fs;
    for (int v = 0; v < 3; ++v) fs.add(F(F_U1 + v), nullptr, F(F_UX + 3 * v + d));
    apply_diff_set(c, d, fs, dx[d]);
  }
  for (int d = 0; d < 3; ++d)
    apply_diff(c, d, F(F_T), nullptr, F(F_TX + d), c->cfg.heat_flux_dx ? dx[d] : 1.0, 1);
  k_visc<<<blocks, kThreads, 0, c->stream>>>(N, t, c->cfg.mu0, c->cfg.T0,
                                             c->cfg.gamma * (c->cfg.R / c->cfg.W) / (c->cfg.gamma - 1.0) /
                                                 c->cfg.Pr);
  CRUNA_LAUNCH_CHECK(c);
  for (int v = 0; v < 3; ++v) apply_diff(c, v, q + 4 * N, nullptr, F(F_PX + 7 * v), dx[v], 1);
}

// ------------------------------------------------------------------------------------------------
// generic adjoint RHS: right_hand_side_adjoint_3d (ns_rho_rhou_p.f90:257-536)
// ------------------------------------------------------------------------------------------------
enum AdjField {
  A_U1, A_U2, A_U3, A_GPR, A_IR,
  A_D0, // 5 fields: D_d qs(v) for v = 0..4
  A_S = A_D0 + 5,  // D_d(u_d * qs5)
  A_P,             // D_d p
  kAdjFields
};

__global__ void k_adj_prim(long long N, const double *__restrict__ q, double *__restrict__ t, double gamma) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    const double gm1 = gamma - 1.0;
    t[p + A_GPR * N] = gamma * q[p + 4 * N] / (q[p] * gm1);   // :292-294
    t[p + A_IR * N] = 1.0 / q[p];
    t[p + A_U1 * N] = q[p + N] / q[p];                          // :299-301
    t[p + A_U2 * N] = q[p + 2 * N] / q[p];
    t[p + A_U3 * N] = q[p + 3 * N] / q[p];
  }
}

// one direction's contribution (:317-370 for d=0, :386-440 for d=1, :456-509 for d=2)
__global__ void k_adj_dir(long long N, int d, int first, const double *__restrict__ t,
                          const double *__restrict__ qs, double *__restrict__ rhs, double gamma) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    const double gm1 = gamma - 1.0;
    const double u1 = t[p + A_U1 * N], u2 = t[p + A_U2 * N], u3 = t[p + A_U3 * N];
    const double gpr = t[p + A_GPR * N], ir = t[p + A_IR * N];
    const double a = t[p + (A_D0 + 0) * N], b = t[p + (A_D0 + 1) * N], c = t[p + (A_D0 + 2) * N],
                 dd = t[p + (A_D0 + 3) * N], e = t[p + (A_D0 + 4) * N];
    const double sx = t[p + A_S * N], px = t[p + A_P * N];
    const double qs5 = qs[p + 4 * N];
    double r1 = first ? 0.0 : rhs[p], r2 = first ? 0.0 : rhs[p + N], r3 = first ? 0.0 : rhs[p + 2 * N],
           r4 = first ? 0.0 : rhs[p + 3 * N], r5 = first ? 0.0 : rhs[p + 4 * N];
    const double ud = d == 0 ? u1 : (d == 1 ? u2 : u3);
    if (d == 0) {
      r1 = r1 + (u1 * u1) * b + (u1 * u2) * c + (u1 * u3) * dd + gpr * u1 * e;
      r2 = r2 - a - 2.0 * u1 * b - u2 * c - u3 * dd - gpr * e;
      r3 = r3 - u1 * c;
      r4 = r4 - u1 * dd;
      r5 = r5 - gm1 * b - gamma * u1 * e;
    } else if (d == 1) {
      r1 = r1 + (u2 * u1) * b + (u2 * u2) * c + (u2 * u3) * dd + gpr * u2 * e;
      r2 = r2 - u2 * b;
      r3 = r3 - a - u1 * b - 2 * u2 * c - u3 * dd - gpr * e;
      r4 = r4 - u2 * dd;
      r5 = r5 - gm1 * c - gamma * u2 * e;
    } else {
      r1 = r1 + (u3 * u1) * b + (u3 * u2) * c + (u3 * u3) * dd + gpr * u3 * e;
      r2 = r2 - u3 * b;
      r3 = r3 - u3 * c;
      r4 = r4 - a - u1 * b - u2 * c - 2 * u3 * dd - gpr * e;
      r5 = r5 - gm1 * dd - gamma * u3 * e;
    }
    // -(A^T)^-1 (C^T qs)_d: D_d(-u_d*qs5) = -D_d(u_d*qs5)
    r5 = r5 - gm1 * (-sx);
    // +(A^T)^-1 C~_d p_d
    r1 = r1 + qs5 * ud * ir * px;
    if (d == 0) r2 = r2 - qs5 * ir * px;
    else if (d == 1) r3 = r3 - qs5 * ir * px;
    else r4 = r4 - qs5 * ir * px;
    rhs[p] = r1; rhs[p + N] = r2; rhs[p + 2 * N] = r3; rhs[p + 3 * N] = r4; rhs[p + 4 * N] = r5;
  }
}

void rhs_adjoint_generic(cruna_ctx *c, const double *qs_in, const double *q, const double *g, double *rhs,
                         double *qsbc) {
  const long long N = c->g.N;
  double *t = c->tmp;
  auto F = [&](int f) { return t + (long long)f * N; };
  const double *qs = qs_in;
  if (c->has_q_bc) {                                      // :287-290
    copy_state(c, qsbc, qs_in, 5);
    bc_qs(c, qsbc, q, 0);
    qs = qsbc;
  }
  const int blocks = (int)std::min<long long>(nblocks(N), 148LL * 32);
  k_adj_prim<<<blocks, kThreads, 0, c->stream>>>(N, q, t, c->cfg.gamma);
  CRUNA_LAUNCH_CHECK(c);
  for (int d = 0; d < 3; ++d) {
    apply_diff(c, d, qs, nullptr, F(A_D0), c->dx[d], 5);                       // 5 fields at once
    apply_diff(c, d, qs + 4 * N, F(A_U1 + d), F(A_S), c->dx[d], 1);            // D_d(u_d*qs5)
    apply_diff(c, d, q + 4 * N, nullptr, F(A_P), c->dx[d], 1);                 // D_d p
    k_adj_dir<<<blocks, kThreads, 0, c->stream>>>(N, d, d == 0, t, qs, rhs, c->cfg.gamma);
    CRUNA_LAUNCH_CHECK(c);
  }
  if (g) add_fields(c, rhs, g, 5 * N);                                         // :512
  if (c->has_rhs_bc) bc_rhss(c, rhs, qs, nullptr);                             // :518 (without q)
}

}  // namespace cruna
