// Helpers shared by the generic kernels (ops.cu) and the discrete adjoint (discrete_adjoint.cu):
// launch sizing, line geometry, the explicit part of a line operator (host and device, so the
// library can read its own operators' matrices), boundary boxes, the sponge shape and the field
// layout of the generic RHS workspace.
#pragma once

#include "cruna_internal.cuh"

namespace cruna {

constexpr int kThreads = 256;

inline int nblocks(long long work, int threads = kThreads) {
  long long b = (work + threads - 1) / threads;
  return (int)(b < 1 ? 1 : b);
}

// ------------------------------------------------------------------------------------------------
// line operators
// ------------------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ void line_geom(const Grid &g, int dir, long long p, long long &base,
                                          long long &stride, int &i) {
  // p is a point index inside one field; returns the line base offset, stride and position
  const long long n1 = g.n1, n12 = (long long)g.n1 * g.n2;
  const long long ii = p % n1, jj = (p / n1) % g.n2, kk = p / n12;
  if (dir == 0) { i = (int)ii; stride = 1; base = p - ii; }
  else if (dir == 1) { i = (int)jj; stride = n1; base = p - jj * n1; }
  else { i = (int)kk; stride = n12; base = p - kk * n12; }
}

__host__ __device__ __forceinline__ double ldv(const double *f1, const double *f2, long long idx) {
  return f2 ? f1[idx] * f2[idx] : f1[idx];
}

// explicit part of the operator at position i of the line starting at f + base
__host__ __device__ inline double explicit_part(const LineOp &op, const double *f1, const double *f2, long long base,
                                long long s, int i) {
  const int n = op.n;
  if (op.kind == OP_ZERO) return 0.0;
  if (op.kind == OP_COPY) return ldv(f1, f2, base + i * s);
  if (op.periodic) {
    if (op.antisym) {
      double t = 0.0;
      for (int m = 1; m <= op.r; ++m) {
        int ip = (i + m) % n, im = ((i - m) % n + n) % n;
        double d = ldv(f1, f2, base + ip * s) - ldv(f1, f2, base + im * s);
        t = (m == 1) ? op.c[1] * d : t + op.c[m] * d;
      }
      return t;
    }
    double t = op.c[0] * ldv(f1, f2, base + i * s);
    for (int m = 1; m <= op.r; ++m) {
      int ip = (i + m) % n, im = ((i - m) % n + n) % n;
      t = t + op.c[m] * (ldv(f1, f2, base + ip * s) + ldv(f1, f2, base + im * s));
    }
    return t;
  }
  if (i >= op.nb && i < n - op.nb) {
    if (op.antisym) {
      double t = 0.0;
      for (int m = 1; m <= op.r; ++m) {
        double d = ldv(f1, f2, base + (i + m) * s) - ldv(f1, f2, base + (i - m) * s);
        t = (m == 1) ? op.c[1] * d : t + op.c[m] * d;
      }
      return t;
    }
    double t = op.c[0] * ldv(f1, f2, base + i * s);
    for (int m = 1; m <= op.r; ++m)
      t = t + op.c[m] * (ldv(f1, f2, base + (i + m) * s) + ldv(f1, f2, base + (i - m) * s));
    return t;
  }
  const bool start = i < op.nb;
  const int row = start ? i : n - 1 - i;
  if (op.keep_ends && row == 0) return ldv(f1, f2, base + i * s);
  double t = 0.0;
  for (int m = 0; m < op.bw; ++m) {
    const int j = start ? m : n - 1 - m;
    t = (m == 0) ? op.brow[row][0] * ldv(f1, f2, base + j * s)
                 : t + op.brow[row][m] * ldv(f1, f2, base + j * s);
  }
  return (op.antisym && !start) ? -t : t;
}

// one output point of the explicit part: stencil or closure row, derivative scale, filter blend
__host__ __device__ inline double line_point(const LineOp &op, const double *a, const double *b, long long base,
                                      long long s, int i, double scale) {
  double v = explicit_part(op, a, b, base, s, i);
  if (op.kind == OP_STENCIL && op.antisym) v = v * scale;
  if (op.blend > 0.0) {
    const double q = ldv(a, b, base + i * s);
    v = q - op.blend * (q - v);
  }
  return v;
}

// ------------------------------------------------------------------------------------------------
// sponge shape on the fly: phi = (((sx*sym)*syp)*szm)*szp, shape = amp*(1 - phi)
// (src/boundaries/shape_functions.f90:104-145)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ double sponge_at(const SpongeDev &sp, const Grid &g, long long p) {
  const long long i = p % g.n1, j = (p / g.n1) % g.n2, k = p / ((long long)g.n1 * g.n2);
  double phi = sp.sx[i] * sp.sym[j];
  phi = phi * sp.syp[j];
  phi = phi * sp.szm[k];
  phi = phi * sp.szp[k];
  return sp.amp * (1.0 - phi);
}

struct Box {
  int is, ie, js, je, ks, ke;
  __host__ __device__ long long count() const { return (long long)(ie - is + 1) * (je - js + 1) * (ke - ks + 1); }
};

__device__ __forceinline__ long long box_point(const Box &b, const Grid &g, long long t, int &i, int &j,
                                               int &k) {
  const int ni = b.ie - b.is + 1, nj = b.je - b.js + 1;
  i = b.is + (int)(t % ni);
  j = b.js + (int)((t / ni) % nj);
  k = b.ks + (int)(t / ((long long)ni * nj));
  return i + (long long)g.n1 * (j + (long long)g.n2 * k);
}

inline Box box_of(const BCRow &r) { return Box{r.is, r.ie, r.js, r.je, r.ks, r.ke}; }

inline long long offset_of(const cruna_ctx *c, const int sh[3]) {
  return sh[0] + (long long)c->g.n1 * (sh[1] + (long long)c->g.n2 * sh[2]);
}

// up to kMax fields of one line operator in one launch: out[f] = op(f1[f]) or op(f1[f] * f2[f])
struct FieldSet {
  static constexpr int kMax = 8;
  const double *f1[kMax] = {};
  const double *f2[kMax] = {};
  double *out[kMax] = {};
  int n = 0;
  void add(const double *a, const double *b, double *o) {
    f1[n] = a;
    f2[n] = b;
    out[n] = o;
    ++n;
  }
};

// Dx_d of every field of a set with spacing h (ops.cu): one launch where the fast line kernels apply
void apply_diff_set(cruna_ctx *c, int dir, const FieldSet &fs, double h);

// field slots of the generic RHS workspace (cruna_ctx::tmp)
enum GenericField {
  F_U1, F_U2, F_U3, F_T,
  F_UX, F_UY, F_UZ, F_VX, F_VY, F_VZ, F_WX, F_WY, F_WZ, F_TX, F_TY, F_TZ,
  F_MU, F_T11, F_T22, F_T33, F_T12, F_T13, F_T23, F_HX, F_HY, F_HZ,
  // divergence terms
  F_M1, F_M2, F_M3,                         // mass: d1(ru) d2(rv) d3(rw)
  F_A1X, F_A1Y, F_A1Z, F_PX, F_V1X, F_V1Y, F_V1Z,
  F_A2X, F_A2Y, F_A2Z, F_PY, F_V2X, F_V2Y, F_V2Z,
  F_A3X, F_A3Y, F_A3Z, F_PZ, F_V3X, F_V3Y, F_V3Z,
  F_EX, F_EY, F_EZ, F_QX, F_QY, F_QZ,
  kGenericFields
};

}  // namespace cruna
