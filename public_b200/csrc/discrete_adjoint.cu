// Exact discrete adjoint of the direct time step: the transpose of what the direct path computes.
//
// The reference's adjoint (src/equations/ns_rho_rhou_p.f90:257-536) is the continuous inviscid
// adjoint, which is not the transpose of the discrete operator, so its gradients differ from finite
// differences of the discrete objective by several per cent.  This file transposes, in reverse mode:
//   * right_hand_side_direct_3d (ns_rho_rhou_p.f90:31-253): BC on q (:92), primitives (:95-116),
//     the 42 derivatives (each line operator B^-1 A transposed to A^T B^-T), Sutherland viscosity,
//     stresses, heat flux and friction work (:118-209), forcing (:212), BC on the RHS (:218);
//   * one loop step of calc_direct (computation_direct.f90:64-107): classical RK4 (rk_o4_e.f90:17-58),
//     BC on q outside the RHS, filters i1, i2, i3 (their transposes in reverse order).
// Point-wise characteristic treatments (nonreflecting.f90:46-137, :237-341) are differentiated in
// forward mode with dual numbers, which gives their Jacobians exactly.
//
// Transposed line operators: the explicit part A of every derivative / filter is read back from the
// operator itself (line_point on unit vectors, host side), transposed into a band, and the compact
// part's B^T is factored with the same dgttrf restatement (cyclic B is symmetric and reused).
#include <algorithm>
#include <cmath>
#include <vector>

#include "bc_point.cuh"
#include "cruna_internal.cuh"
#include "dual.cuh"
#include "ops_common.cuh"

namespace cruna {

namespace {

constexpr double kS1 = 110.4;  // Sutherland constant (ns_rho_rhou_p_trafos.f90:124)

// backward workspace layout (fields of N points)
enum VjpField {
  V_L = 0,        // 5: D_d^T of the five RHS cotangents
  V_MB = 5,       // 3: cotangent of rho u_d
  V_UB = 8,       // 3: cotangent of u_v
  V_PB = 11,      // 1: cotangent of p
  V_TAUB = 12,    // 6: cotangents of tau_11, tau_22, tau_33, tau_12, tau_13, tau_23
  V_MUB = 18,     // 1: cotangent of mu
  V_TGB = 19,     // 3: cotangent of d_d T
  V_GB = 22,      // 9: cotangent of d_d u_v, stored [d][v]
  V_B = 31,       // 3: cotangent of d_v p
  V_TB = 34,      // 1: cotangent of T
  V_SCR = 35,     // 5: solve scratch of the transposed operators
  kVjpFields = 40
};

// state-sized buffers (cruna_ctx::vjp_st)
enum VjpState { S_QREP, S_LPRE, S_LQ, S_Q2, S_Q3, S_Q4, S_Q1, S_K, S_ACC, S_LQ1, S_LK, S_MU };

__host__ __device__ __forceinline__ int tau_slot(int v, int d) {
  // symmetric stress component (v, d) -> 0..5 in the order 11, 22, 33, 12, 13, 23
  if (v == d) return v;
  const int a = v < d ? v : d, b = v < d ? d : v;
  return a == 0 ? (b == 1 ? 3 : 4) : 5;
}

// ------------------------------------------------------------------------------------------------
// transposed line operators
// ------------------------------------------------------------------------------------------------
template <class T>
T *upload_vec(cruna_ctx *c, const std::vector<T> &v) {
  if (v.empty()) return nullptr;
  double *p = dalloc(c, (v.size() * sizeof(T) + sizeof(double) - 1) / sizeof(double));
  CRUNA_CUDA_CHECK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return reinterpret_cast<T *>(p);
}

void build_transpose(cruna_ctx *c, const LineOp &op, const HostFactors &hf, LineOpT &t) {
  t = LineOpT();
  t.n = op.n;
  t.kind = op.kind;
  if (op.kind != OP_STENCIL) return;
  const int n = op.n;
  const int W = std::max(op.r, op.bw);
  int lo = -W, hi = W;
  if (op.periodic && n < 2 * W + 1) {
    lo = -((n - 1) / 2);
    hi = lo + n - 1;
  }
  t.periodic = op.periodic;
  t.lo = lo;
  t.hi = hi;
  const int w = hi - lo + 1;
  std::vector<double> band((size_t)n * w, 0.0);
  // unit vector with W zeros of padding on both sides (closure rows never read outside the line)
  std::vector<double> e((size_t)n + 2 * W, 0.0);
  double *line = e.data() + W;
  for (int i = 0; i < n; ++i) {
    for (int o = lo; o <= hi; ++o) {
      int j = i + o;
      if (op.periodic) j = ((j % n) + n) % n;
      else if (j < 0 || j >= n) continue;
      line[j] = 1.0;
      const double a = line_point(op, line, nullptr, 0, 1, i, 1.0);  // A_ij
      line[j] = 0.0;
      if (a == 0.0) continue;
      int ot = i - j;  // (A^T)_{j,i}: row j, offset i - j
      if (op.periodic) ot = ((ot - lo) % n + n) % n + lo;
      if (ot < lo || ot > hi) throw ApiError{CRUNA_ERR_UNSUPPORTED, "line operator wider than its band"};
      band[(size_t)j * w + (ot - lo)] += a;
    }
  }
  t.band = upload_vec(c, band);
  if (!op.solve) return;
  t.solve = 1;
  if (op.cyclic) {  // the cyclic matrix (alpha off-diagonals and corners) is symmetric: B^T = B
    t.sop = op;
    return;
  }
  HostFactors ht;  // B^T of the open tridiagonal matrix
  ht.dl = hf.raw_du;
  ht.d = hf.raw_d;
  ht.du = hf.raw_dl;
  ht.du2.assign(n > 2 ? n - 2 : 1, 0.0);
  ht.ipiv.assign(n, 0);
  if (lapack_dgttrf(n, ht.dl.data(), ht.d.data(), ht.du.data(), ht.du2.data(), ht.ipiv.data()) != 0)
    throw ApiError{CRUNA_ERR_UNSUPPORTED, "dgttrf of a transposed compact operator failed"};
  std::vector<double> inv(ht.d.size());
  for (size_t i = 0; i < ht.d.size(); ++i) inv[i] = 1.0 / ht.d[i];
  t.sop = op;
  t.sop.cyclic = 0;
  t.sop.dl = upload_vec(c, ht.dl);
  t.sop.inv_d = upload_vec(c, inv);
  t.sop.du = upload_vec(c, ht.du);
  t.sop.du2 = upload_vec(c, ht.du2);
  t.sop.ipiv = upload_vec(c, ht.ipiv);
  t.sop.nopiv = 1;
  for (size_t i = 0; i + 1 < ht.ipiv.size(); ++i)
    if (ht.ipiv[i] != (int)i + 1) t.sop.nopiv = 0;
}

__global__ void k_band_T(LineOpT op, Grid g, int dir, const double *__restrict__ in, double *__restrict__ out,
                         double scale, int nfields, int accumulate) {
  const long long total = g.N * nfields;
  const int n = op.n, w = op.hi - op.lo + 1;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long fld = t / g.N, p = t - fld * g.N;
    long long base, s;
    int i;
    line_geom(g, dir, p, base, s, i);
    const double *a = in + fld * g.N + base;
    const double *row = op.band + (long long)i * w;
    double v = 0.0;
    for (int o = op.lo; o <= op.hi; ++o) {
      int j = i + o;
      if (op.periodic) {
        if (j < 0) j += n;
        else if (j >= n) j -= n;
      } else if (j < 0 || j >= n) {
        continue;
      }
      v += row[o - op.lo] * a[j * s];
    }
    v *= scale;
    out[t] = accumulate ? out[t] + v : v;
  }
}

// the same banded product with the line position from the launch grid (x = block x range, y = j,
// (k, field) = z, strided) instead of a division per point; DIR is compile-time
template <int DIR>
__global__ void __launch_bounds__(128) k_band_T_grid(LineOpT op, Grid g, const double *__restrict__ in,
                                                     double *__restrict__ out, double scale, int nfields,
                                                     int accumulate) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= g.n1) return;
  const int j = blockIdx.y;
  const int n = op.n, w = op.hi - op.lo + 1;
  const long long n12 = (long long)g.n1 * g.n2;
  const long long s = DIR == 0 ? 1 : (DIR == 1 ? (long long)g.n1 : n12);
  for (int kf = blockIdx.z; kf < g.n3 * nfields; kf += gridDim.z) {
    const int fld = kf / g.n3, k = kf - fld * g.n3;
    const long long p = x + (long long)g.n1 * j + n12 * k;
    const int i = DIR == 0 ? x : (DIR == 1 ? j : k);
    const double *a = in + (long long)fld * g.N + p - (long long)i * s;  // the line's first point
    const double *__restrict__ row = op.band + (long long)i * w;
    double v = 0.0;
    for (int o = op.lo; o <= op.hi; ++o) {
      int jj = i + o;
      if (op.periodic) {
        if (jj < 0) jj += n;
        else if (jj >= n) jj -= n;
      } else if (jj < 0 || jj >= n) {
        continue;
      }
      v += row[o - op.lo] * a[jj * s];
    }
    v *= scale;
    double *o_ = out + (long long)fld * g.N + p;
    *o_ = accumulate ? *o_ + v : v;
  }
}

// out (+)= scale * A^T B^-T in, on nfields fields along dir
void apply_T(cruna_ctx *c, const LineOpT &t, int dir, const double *in, double *out, double scale, int nfields,
             int accumulate, double *scratch) {
  const long long M = c->g.N * nfields;
  if (t.kind == OP_ZERO) {
    if (!accumulate) CRUNA_CUDA_CHECK(cudaMemsetAsync(out, 0, sizeof(double) * M, c->stream));
    return;
  }
  if (t.kind == OP_COPY) {
    if (accumulate) add_fields(c, out, in, M);
    else copy_state(c, out, in, nfields);
    return;
  }
  const double *src = in;
  if (t.solve) {
    copy_state(c, scratch, in, nfields);
    launch_line_solve(c, t.sop, dir, scratch, nfields);
    src = scratch;
  }
  ProfScope ps(c, "band_T");
  if (c->g.n2 <= 65535) {
    const int bx = c->g.n1 >= 128 ? 128 : (c->g.n1 >= 64 ? 64 : 32);
    const dim3 grid((c->g.n1 + bx - 1) / bx, c->g.n2, std::min(c->g.n3 * nfields, 65535));
    if (dir == 0) k_band_T_grid<0><<<grid, bx, 0, c->stream>>>(t, c->g, src, out, scale, nfields, accumulate);
    else if (dir == 1) k_band_T_grid<1><<<grid, bx, 0, c->stream>>>(t, c->g, src, out, scale, nfields, accumulate);
    else k_band_T_grid<2><<<grid, bx, 0, c->stream>>>(t, c->g, src, out, scale, nfields, accumulate);
  } else {
    k_band_T<<<(int)std::min<long long>(nblocks(M), 148LL * 64), kThreads, 0, c->stream>>>(
        t, c->g, dir, src, out, scale, nfields, accumulate);
  }
  CRUNA_LAUNCH_CHECK(c);
}

double diff_scale(const cruna_ctx *c, int d, double h) {
  const LineOp &op = c->dop[d];
  return (op.kind == OP_STENCIL && op.antisym) ? 1.0 / (h * op.div) : 1.0;
}

// D_d^T with the grid spacing h (the direct path's apply_diff scale 1/(h*div))
void diff_T(cruna_ctx *c, int d, const double *in, double *out, double h, int nfields, int accumulate) {
  apply_T(c, c->dopT[d], d, in, out, diff_scale(c, d, h), nfields, accumulate, c->vjp_ws + V_SCR * c->g.N);
}

// filter_i_d^T of a state in place (scratch: 5 fields)
void filter_T(cruna_ctx *c, int d, double *lam, double *scratch) {
  const LineOpT &t = c->fopT[d];
  if (t.kind == OP_COPY) return;
  apply_T(c, t, d, lam, scratch, 1.0, 5, 0, c->vjp_ws + V_SCR * c->g.N);
  copy_state(c, lam, scratch, 5);
}

// ------------------------------------------------------------------------------------------------
// boundary conditions: forward replay with saved box values, transposes in reverse row order
// ------------------------------------------------------------------------------------------------
__global__ void k_pack(Box b, Grid g, const double *a, const double *aux, long long aux_off, double *save) {
  const long long tot = b.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const long long p = box_point(b, g, t, i, j, k);
    for (int v = 0; v < 5; ++v) {
      save[t * 10 + v] = a[p + v * g.N];
      save[t * 10 + 5 + v] = aux ? aux[p + aux_off + v * g.N] : 0.0;
    }
  }
}

// type 201 (aim = qref, K = 5) and 200 (aim = q at p + off, differentiated too, K = 10)
template <int K>
__global__ void k_char_q_T(Box b, Grid g, double k1, double k2, double k3, double gamma, const double *save,
                           const double *qref, long long aim_off, double *lam) {
  const long long tot = b.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const long long p = box_point(b, g, t, i, j, k);
    const long long N = g.N;
    Dual<K> qd[5], out[5];
    for (int v = 0; v < 5; ++v) qd[v] = Dual<K>::seed(save[t * 10 + v], v);
    double l[5];
    for (int v = 0; v < 5; ++v) l[v] = lam[p + v * N];
    if (K == 10) {
      Dual<K> ad[5];
      for (int v = 0; v < 5; ++v) ad[v] = Dual<K>::seed(save[t * 10 + 5 + v], (5 + v) % K);
      char_q_point(qd, ad, k1, k2, k3, gamma, out);
    } else {
      double av[5];
      for (int v = 0; v < 5; ++v) av[v] = qref[p + v * N];
      char_q_point(qd, av, k1, k2, k3, gamma, out);
    }
    for (int jj = 0; jj < 5; ++jj) {
      double s = 0.0;
      for (int v = 0; v < 5; ++v) s += l[v] * out[v].d[jj];
      lam[p + jj * N] = s;
    }
    if (K == 10) {  // the aim point p + off lies outside the box (one plane inwards)
      for (int jj = 0; jj < 5; ++jj) {
        double s = 0.0;
        for (int v = 0; v < 5; ++v) s += l[v] * out[v].d[(5 + jj) % K];
        lam[p + aim_off + jj * N] += s;
      }
    }
  }
}

// type 204: rhs and q both differentiated (slots 0..4 rhs, 5..9 q)
__global__ void k_char_rhs_T(Box b, Grid g, double k1, double k2, double k3, double gamma, double dt,
                             const double *save, const double *qb, const double *qref, double *lam, double *lam_q) {
  const long long tot = b.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const long long p = box_point(b, g, t, i, j, k);
    const long long N = g.N;
    Dual<10> rd[5], qd[5], out[5];
    double av[5], l[5];
    for (int v = 0; v < 5; ++v) {
      rd[v] = Dual<10>::seed(save[t * 10 + v], v);
      qd[v] = Dual<10>::seed(qb[p + v * N], 5 + v);
      av[v] = qref[p + v * N];
      l[v] = lam[p + v * N];
    }
    char_rhs_point(rd, qd, av, k1, k2, k3, gamma, dt, out);
    for (int jj = 0; jj < 5; ++jj) {
      double sr = 0.0, sq = 0.0;
      for (int v = 0; v < 5; ++v) {
        sr += l[v] * out[v].d[jj];
        sq += l[v] * out[v].d[5 + jj];
      }
      lam[p + jj * N] = sr;
      lam_q[p + jj * N] += sq;
    }
  }
}

// zonal types 202 (shape 1) and 203 (shape-weighted): aim = qref, the boundary normal from the
// k-vector field (nonreflecting.f90:141-233)
__global__ void k_char_q4_T(Box b, Grid g, const double *__restrict__ kv, SpongeDev sp, int shaped, double gamma,
                            const double *save, const double *qref, double *lam) {
  const long long tot = b.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const long long p = box_point(b, g, t, i, j, k);
    const long long N = g.N;
    Dual<5> qd[5], out[5];
    double av[5], l[5];
    for (int v = 0; v < 5; ++v) {
      qd[v] = Dual<5>::seed(save[t * 10 + v], v);
      av[v] = qref[p + v * N];
      l[v] = lam[p + v * N];
    }
    char_q_point(qd, av, kv[p], kv[p + N], kv[p + 2 * N], gamma, out, shaped ? sponge_at(sp, g, p) : 1.0);
    for (int jj = 0; jj < 5; ++jj) {
      double sum = 0.0;
      for (int v = 0; v < 5; ++v) sum += l[v] * out[v].d[jj];
      lam[p + jj * N] = sum;
    }
  }
}

// zonal types 205 and 206 on the RHS (nonreflecting.f90:345-449): rhs and q differentiated
__global__ void k_char_rhs4_T(Box b, Grid g, const double *__restrict__ kv, SpongeDev sp, int shaped,
                              double gamma, double dt, const double *save, const double *qb, const double *qref,
                              double *lam, double *lam_q) {
  const long long tot = b.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const long long p = box_point(b, g, t, i, j, k);
    const long long N = g.N;
    Dual<10> rd[5], qd[5], out[5];
    double av[5], l[5];
    for (int v = 0; v < 5; ++v) {
      rd[v] = Dual<10>::seed(save[t * 10 + v], v);
      qd[v] = Dual<10>::seed(qb[p + v * N], 5 + v);
      av[v] = qref[p + v * N];
      l[v] = lam[p + v * N];
    }
    char_rhs_point(rd, qd, av, kv[p], kv[p + N], kv[p + 2 * N], gamma, dt, out, shaped != 0,
                   shaped ? sponge_at(sp, g, p) : 0.0);
    for (int jj = 0; jj < 5; ++jj) {
      double sr = 0.0, sq = 0.0;
      for (int v = 0; v < 5; ++v) {
        sr += l[v] * out[v].d[jj];
        sq += l[v] * out[v].d[5 + jj];
      }
      lam[p + jj * N] = sr;
      lam_q[p + jj * N] += sq;
    }
  }
}

// the q-BC rows that act in this call: type 203 only inside or only outside the RHS (r.only)
bool q_row_active(const BCRow &r, int outside) {
  return r.type != 203 || (outside ? r.only != 1 : r.only != -1);
}

// mode 0: lam *= (1 - shape) (transpose of the type 401 sponge on q); mode 1: lam_q -= shape * lam
// (type 400 sponge on the RHS, sponge_layer_core.f90:45-48 and :80-84)
__global__ void k_sponge_T(int mode, Grid g, SpongeDev sp, double *a, const double *b) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < g.N;
       p += (long long)gridDim.x * blockDim.x) {
    const double sh = sponge_at(sp, g, p);
    for (int v = 0; v < 5; ++v) {
      const long long x = p + v * g.N;
      if (mode == 0) a[x] = a[x] - sh * a[x];
      else a[x] = a[x] - sh * b[x];
    }
  }
}

__global__ void k_wall_T(Box b, Grid g, int comp, double *lam) {
  const long long tot = b.count();
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    const long long p = box_point(b, g, t, i, j, k);
    lam[p + comp * g.N] = 0.0;
  }
}

// runs one row of the boundary table through the direct path's dispatcher
template <class F>
void with_single_row(cruna_ctx *c, const BCRow &row, F &&f) {
  std::vector<BCRow> one(1, row);
  std::swap(c->bc, one);
  try {
    f();
  } catch (...) {
    std::swap(c->bc, one);
    throw;
  }
  std::swap(c->bc, one);
}

// replays set_boundary_condition_q(q, outside) (boundary_conditions.f90:52-136) on a copy of q, row
// by row as the direct path applies them, saving each characteristic row's box input; returns the
// post-BC state
double *bc_q_replay(cruna_ctx *c, const double *q, int outside) {
  double *qr = c->vjp_st[S_QREP];
  copy_state(c, qr, q, 5);
  for (size_t r = 0; r < c->bc.size(); ++r) {
    const BCRow &row = c->bc[r];
    Box b = box_of(row);
    if (row.type == 200 || row.type == 201 || row.type == 202 || (row.type == 203 && q_row_active(row, outside))) {
      const long long off = row.type == 200 ? offset_of(c, row.shift) : 0;
      k_pack<<<nblocks(b.count()), kThreads, 0, c->stream>>>(b, c->g, qr, row.type == 200 ? qr : nullptr, off,
                                                              c->vjp_save[r]);
      CRUNA_LAUNCH_CHECK(c);
    }
    const BCRow copy = row;
    with_single_row(c, copy, [&]() { bc_q(c, qr, outside); });
  }
  return qr;
}

// transpose of set_boundary_condition_q(., outside), in place on lam, using the saves of the last replay
void bc_q_T(cruna_ctx *c, double *lam, int outside) {
  for (size_t rr = c->bc.size(); rr-- > 0;) {
    const BCRow &row = c->bc[rr];
    Box b = box_of(row);
    const int blocks = nblocks(b.count());
    if (row.type == 202 || (row.type == 203 && q_row_active(row, outside))) {
      k_char_q4_T<<<blocks, kThreads, 0, c->stream>>>(b, c->g, c->kvec, c->sponge, row.type == 203, c->cfg.gamma,
                                                      c->vjp_save[rr], c->qref, lam);
      CRUNA_LAUNCH_CHECK(c);
    } else if (row.type == 401) {
      k_sponge_T<<<nblocks(c->g.N), kThreads, 0, c->stream>>>(0, c->g, c->sponge, lam, nullptr);
      CRUNA_LAUNCH_CHECK(c);
    } else if (row.type == 201) {
      k_char_q_T<5><<<blocks, kThreads, 0, c->stream>>>(b, c->g, row.k[0], row.k[1], row.k[2], c->cfg.gamma,
                                                          c->vjp_save[rr], c->qref, 0, lam);
      CRUNA_LAUNCH_CHECK(c);
    } else if (row.type == 200) {
      k_char_q_T<10><<<blocks, kThreads, 0, c->stream>>>(b, c->g, row.k[0], row.k[1], row.k[2], c->cfg.gamma,
                                                           c->vjp_save[rr], nullptr, offset_of(c, row.shift), lam);
      CRUNA_LAUNCH_CHECK(c);
    }
  }
}

// transpose of set_boundary_condition_rhs(rhs, qb) (boundary_conditions.f90:228-298): lam is the
// RHS cotangent (in place: becomes the cotangent before the BC), lam_q receives the qb cotangent
void bc_rhs_T(cruna_ctx *c, const double *qb, double *lam, double *lam_q) {
  auto characteristic = [](int type) { return type == 204 || type == 205 || type == 206; };
  bool any = false;
  for (const BCRow &r : c->bc) any = any || characteristic(r.type);
  if (any) {  // replay on the RHS before the BC, saving each characteristic row's box input
    double *R = c->vjp_st[S_K];
    rhs_direct_generic(c, qb, R, c->st[4], 0);
    for (size_t r = 0; r < c->bc.size(); ++r) {
      const BCRow &row = c->bc[r];
      Box b = box_of(row);
      if (characteristic(row.type)) {
        k_pack<<<nblocks(b.count()), kThreads, 0, c->stream>>>(b, c->g, R, nullptr, 0, c->vjp_save[r]);
        CRUNA_LAUNCH_CHECK(c);
      }
      const BCRow copy = row;
      with_single_row(c, copy, [&]() { bc_rhs(c, R, qb); });
    }
  }
  for (size_t rr = c->bc.size(); rr-- > 0;) {
    const BCRow &row = c->bc[rr];
    Box b = box_of(row);
    const int blocks = nblocks(b.count());
    if (row.type == 100) {
      k_wall_T<<<blocks, kThreads, 0, c->stream>>>(b, c->g, row.comp, lam);
      CRUNA_LAUNCH_CHECK(c);
    } else if (row.type == 400) {
      k_sponge_T<<<nblocks(c->g.N), kThreads, 0, c->stream>>>(1, c->g, c->sponge, lam_q, lam);
      CRUNA_LAUNCH_CHECK(c);
    } else if (row.type == 204) {
      k_char_rhs_T<<<blocks, kThreads, 0, c->stream>>>(b, c->g, row.k[0], row.k[1], row.k[2], c->cfg.gamma,
                                                        c->cfg.dt, c->vjp_save[rr], qb, c->qref, lam, lam_q);
      CRUNA_LAUNCH_CHECK(c);
    } else if (row.type == 205 || row.type == 206) {
      k_char_rhs4_T<<<blocks, kThreads, 0, c->stream>>>(b, c->g, c->kvec, c->sponge, row.type == 206, c->cfg.gamma,
                                                        c->cfg.dt, c->vjp_save[rr], qb, c->qref, lam, lam_q);
      CRUNA_LAUNCH_CHECK(c);
    }
  }
}

// ------------------------------------------------------------------------------------------------
// transpose of the interior RHS (ns_rho_rhou_p.f90:95-209)
// ------------------------------------------------------------------------------------------------
// one direction's transposed derivatives of the five RHS components: mass (:131-135), momentum fluxes
// and stress divergence (:138-177), pressure flux (:180-186), heat-flux divergence (:195-200)
__global__ void k_vjp_dir(long long N, int d, double ratio, double gamma, double cp_pr, const double *__restrict__ q,
                          const double *__restrict__ t, double *__restrict__ w) {
  const double gm1 = gamma - 1.0, gt = gamma / gm1;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
#define W_(f) w[p + (long long)(f) * N]
#define T_(f) t[p + (long long)(f) * N]
    const double L0 = W_(V_L), L1 = W_(V_L + 1), L2 = W_(V_L + 2), L3 = W_(V_L + 3), L4 = W_(V_L + 4);
    const double u0 = T_(F_U1), u1 = T_(F_U2), u2 = T_(F_U3);
    const double md = q[p + (1 + d) * N], pr = q[p + 4 * N];
    const double Lv[3] = {L1, L2, L3};
    W_(V_MB + d) = W_(V_MB + d) - L0 - (u0 * L1 + u1 * L2 + u2 * L3);
    for (int v = 0; v < 3; ++v) {
      W_(V_UB + v) = W_(V_UB + v) - md * Lv[v];
      W_(V_TAUB + tau_slot(v, d)) = W_(V_TAUB + tau_slot(v, d)) + Lv[v];
    }
    const double e = -gt * gm1 * L4;
    const double ud = d == 0 ? u0 : (d == 1 ? u1 : u2);
    W_(V_UB + d) = W_(V_UB + d) + pr * e;
    W_(V_PB) = W_(V_PB) + ud * e;
    const double hb = gm1 * ratio * L4;
    const double mu = T_(F_MU);
    W_(V_TGB + d) = mu * cp_pr * hb;
    W_(V_MUB) = W_(V_MUB) + cp_pr * T_(F_TX + d) * hb;
#undef W_
#undef T_
  }
}

// friction work and u . grad p (:187, :204-206), stresses (:118-128), Sutherland (trafos.f90:140)
__global__ void k_vjp_mid(long long N, double gamma, const double *__restrict__ lam, const double *__restrict__ t,
                          double *__restrict__ w) {
  const double gm1 = gamma - 1.0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
#define W_(f) w[p + (long long)(f) * N]
#define T_(f) t[p + (long long)(f) * N]
    const double L5 = gm1 * lam[p + 4 * N];
    double G[3][3];
    for (int v = 0; v < 3; ++v)
      for (int d = 0; d < 3; ++d) G[v][d] = T_(F_UX + 3 * v + d);
    const double tau[6] = {T_(F_T11), T_(F_T22), T_(F_T33), T_(F_T12), T_(F_T13), T_(F_T23)};
    const double mu = T_(F_MU), T = T_(F_T);
    const double u[3] = {T_(F_U1), T_(F_U2), T_(F_U3)};
    const double P[3] = {T_(F_PX), T_(F_PY), T_(F_PZ)};
    double tb[6];
    for (int s = 0; s < 6; ++s) tb[s] = W_(V_TAUB + s);
    double Gb[3][3];
    for (int v = 0; v < 3; ++v)
      for (int d = 0; d < 3; ++d) {
        tb[tau_slot(v, d)] += L5 * G[v][d];
        Gb[v][d] = L5 * tau[tau_slot(v, d)];
      }
    const double div = G[0][0] + G[1][1] + G[2][2];
    double mub = W_(V_MUB);
    for (int v = 0; v < 3; ++v) mub += tb[v] * (-(2.0 / 3.0) * div + 2.0 * G[v][v]);
    mub += tb[3] * (G[0][1] + G[1][0]) + tb[4] * (G[0][2] + G[2][0]) + tb[5] * (G[1][2] + G[2][1]);
    const double st = tb[0] + tb[1] + tb[2];
    for (int v = 0; v < 3; ++v)
      for (int d = 0; d < 3; ++d)
        Gb[v][d] += (v == d) ? 2.0 * mu * tb[v] - (2.0 / 3.0) * mu * st : mu * tb[tau_slot(v, d)];
    for (int v = 0; v < 3; ++v)
      for (int d = 0; d < 3; ++d) W_(V_GB + 3 * d + v) = Gb[v][d];
    W_(V_TB) = mub * mu * (1.5 / T - 1.0 / (T + kS1));
    for (int v = 0; v < 3; ++v) {
      W_(V_UB + v) = W_(V_UB + v) + L5 * P[v];
      W_(V_B + v) = -lam[p + (1 + v) * N] + L5 * u[v];
    }
#undef W_
#undef T_
  }
}

// primitives u = rho u / rho, T = (W/R) p / rho (:95-99, trafos.f90:57) transposed
__global__ void k_vjp_final(long long N, double WoR, const double *__restrict__ q, const double *__restrict__ t,
                            const double *__restrict__ w, double *__restrict__ out, const double *__restrict__ add) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
#define W_(f) w[p + (long long)(f) * N]
#define T_(f) t[p + (long long)(f) * N]
    const double rho = q[p];
    const double u0 = T_(F_U1), u1 = T_(F_U2), u2 = T_(F_U3), T = T_(F_T);
    const double ub0 = W_(V_UB), ub1 = W_(V_UB + 1), ub2 = W_(V_UB + 2), tb = W_(V_TB);
    double o[5];
    o[0] = -(ub0 * u0 + ub1 * u1 + ub2 * u2) / rho - tb * T / rho;
    o[1] = W_(V_MB) + ub0 / rho;
    o[2] = W_(V_MB + 1) + ub1 / rho;
    o[3] = W_(V_MB + 2) + ub2 / rho;
    o[4] = W_(V_PB) + WoR * tb / rho;
    for (int v = 0; v < 5; ++v) out[p + v * N] = add ? o[v] + add[p + v * N] : o[v];
#undef W_
#undef T_
  }
}

void interior_vjp(cruna_ctx *c, const double *qb, const double *lam, double *mu, const double *lam_q) {
  const long long N = c->g.N;
  ensure_generic(c);
  generic_forward_gradients(c, qb);
  double *w = c->vjp_ws;
  auto Wf = [&](int f) { return w + (long long)f * N; };
  CRUNA_CUDA_CHECK(cudaMemsetAsync(Wf(V_MB), 0, sizeof(double) * N * (V_MUB + 1 - V_MB), c->stream));
  CRUNA_CUDA_CHECK(cudaMemsetAsync(Wf(V_TGB), 0, sizeof(double) * N * 3, c->stream));
  const int blocks = (int)std::min<long long>(nblocks(N), 148LL * 32);
  const double gamma = c->cfg.gamma;
  const double cp_pr = gamma * (c->cfg.R / c->cfg.W) / (gamma - 1.0) / c->cfg.Pr;
  bool live[3];
  double hT[3];
  for (int d = 0; d < 3; ++d) {
    live[d] = c->dop[d].kind != OP_ZERO;  // an empty direction contributes nothing (and has dx = inf)
    hT[d] = c->cfg.heat_flux_dx ? c->dx[d] : 1.0;
  }
  for (int d = 0; d < 3; ++d) {
    if (!live[d]) continue;
    diff_T(c, d, lam, Wf(V_L), c->dx[d], 5, 0);
    const double ratio = diff_scale(c, d, hT[d]) / diff_scale(c, d, c->dx[d]);
    k_vjp_dir<<<blocks, kThreads, 0, c->stream>>>(N, d, ratio, gamma, cp_pr, qb, c->tmp, w);
    CRUNA_LAUNCH_CHECK(c);
  }
  k_vjp_mid<<<blocks, kThreads, 0, c->stream>>>(N, gamma, lam, c->tmp, w);
  CRUNA_LAUNCH_CHECK(c);
  for (int d = 0; d < 3; ++d) {
    if (!live[d]) continue;
    diff_T(c, d, Wf(V_B + d), Wf(V_PB), c->dx[d], 1, 1);      // grad p
    diff_T(c, d, Wf(V_GB + 3 * d), Wf(V_UB), c->dx[d], 3, 1);  // grad u, v, w along d
    diff_T(c, d, Wf(V_TGB + d), Wf(V_TB), hT[d], 1, 1);        // grad T
  }
  k_vjp_final<<<blocks, kThreads, 0, c->stream>>>(N, c->cfg.W / c->cfg.R, qb, c->tmp, w, mu, lam_q);
  CRUNA_LAUNCH_CHECK(c);
}

__global__ void k_lin2(long long M, double a, const double *__restrict__ x, double b, const double *__restrict__ y,
                       double *__restrict__ out) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < M;
       p += (long long)gridDim.x * blockDim.x)
    out[p] = y ? a * x[p] + b * y[p] : a * x[p];
}

void lin2(cruna_ctx *c, double a, const double *x, double b, const double *y, double *out) {
  const long long M = c->g.N * 5;
  k_lin2<<<(int)std::min<long long>(nblocks(M), 148LL * 32), kThreads, 0, c->stream>>>(M, a, x, b, y, out);
  CRUNA_LAUNCH_CHECK(c);
}

void ensure_vjp(cruna_ctx *c) {
  if (c->vjp_ready) return;
  if (c->cfg.precision != CRUNA_FP64)
    throw ApiError{CRUNA_ERR_UNSUPPORTED, "the discrete adjoint transposes the FP64 operator: precision must be FP64"};
  if (c->closure_mlp) throw ApiError{CRUNA_ERR_UNSUPPORTED, "the discrete adjoint does not transpose the closure"};
  if (c->halo_fn) throw ApiError{CRUNA_ERR_UNSUPPORTED, "the discrete adjoint runs on one block (no z slabs)"};
  for (int d = 0; d < 3; ++d) {
    if (!c->dopT_built[d]) build_transpose(c, c->dop[d], c->dhf[d], c->dopT[d]);
    c->dopT_built[d] = true;
    build_transpose(c, c->fop[d], c->fhf[d], c->fopT[d]);
  }
  c->vjp_ws = dalloc(c, (size_t)c->g.N * kVjpFields);
  for (double *&s : c->vjp_st) s = dalloc(c, (size_t)c->g.N * 5);
  c->vjp_save.assign(c->bc.size(), nullptr);
  for (size_t r = 0; r < c->bc.size(); ++r) {
    const BCRow &row = c->bc[r];
    if (row.type >= 200 && row.type <= 206)
      c->vjp_save[r] = dalloc(c, (size_t)box_of(row).count() * 10);
  }
  ensure_generic(c);
  if (!c->st[4]) c->st[4] = dalloc(c, (size_t)c->g.N * 5);
  c->vjp_ready = true;
}

bool due_at(int freq, int nt) { return freq > 0 && nt % freq == 0; }

}  // namespace

// (d rhs_direct / d q)^T lam at q; gf_acc (optional) += (d rhs / d f)^T lam
void rhs_direct_vjp(cruna_ctx *c, const double *q, const double *lam, double *mu, double *gf_acc) {
  ensure_vjp(c);
  const double *qb = c->has_q_bc ? bc_q_replay(c, q, 0) : q;
  double *lpre = c->vjp_st[S_LPRE], *lq = c->vjp_st[S_LQ];
  copy_state(c, lpre, lam, 5);
  if (c->has_rhs_bc) {
    CRUNA_CUDA_CHECK(cudaMemsetAsync(lq, 0, sizeof(double) * c->g.N * 5, c->stream));
    bc_rhs_T(c, qb, lpre, lq);
  }
  if (gf_acc) add_fields(c, gf_acc, lpre, c->g.N * 5);
  interior_vjp(c, qb, lpre, mu, c->has_rhs_bc ? lq : nullptr);
  if (c->has_q_bc) bc_q_T(c, mu, 0);
}

// transpose of one calc_direct loop step nt at q0: lam0 = (d q1 / d q0)^T lam1, gf_acc += (d q1/d f)^T lam1
void step_direct_vjp(cruna_ctx *c, const double *q0, const double *lam1, double *lam0, double *gf_acc, int nt) {
  ensure_vjp(c);
  double **S = c->vjp_st;
  const double dt = c->cfg.dt, dth = 0.5 * dt;
  double *k = S[S_K], *acc = S[S_ACC];
  // forward: the stage states of time_stepper_direct (rk_o4_e.f90:17-58), on the direct path's kernels
  const bool need_q1 = c->has_q_bc;
  if (use_fused(c)) {
    rhs_direct_fused(c, q0, k, 1, q0, acc, S[S_Q2], dt);
    rhs_direct_fused(c, S[S_Q2], k, 2, q0, acc, S[S_Q3], dt);
    rhs_direct_fused(c, S[S_Q3], k, 3, q0, acc, S[S_Q4], dt);
    if (need_q1) rhs_direct_fused(c, S[S_Q4], k, 4, q0, acc, S[S_Q1], dt);
  } else {
    rhs_direct_generic(c, q0, k, c->st[4]);
    rk_stage(c, 1, dt, k, q0, acc, S[S_Q2]);
    rhs_direct_generic(c, S[S_Q2], k, c->st[4]);
    rk_stage(c, 2, dt, k, q0, acc, S[S_Q3]);
    rhs_direct_generic(c, S[S_Q3], k, c->st[4]);
    rk_stage(c, 3, dt, k, q0, acc, S[S_Q4]);
    if (need_q1) {
      rhs_direct_generic(c, S[S_Q4], k, c->st[4]);
      rk_stage(c, 4, dt, k, q0, acc, S[S_Q1]);
    }
  }
  // reverse: filters i3, i2, i1, then the BC on q outside the RHS (computation_direct.f90:76-100)
  double *l1 = S[S_LQ1], *lk = S[S_LK], *mu = S[S_MU];
  copy_state(c, l1, lam1, 5);
  for (int d = 2; d >= 0; --d)
    if (due_at(c->cfg.di_freq[d], nt)) filter_T(c, d, l1, k);
  if (c->has_q_bc) {
    bc_q_replay(c, S[S_Q1], 1);
    bc_q_T(c, l1, 1);
  }
  // RK4 transposed: lam0 = l1 + sum_s J_s^T lk_s, stages in reverse order
  copy_state(c, lam0, l1, 5);
  lin2(c, dt / 6.0, l1, 0.0, nullptr, lk);
  rhs_direct_vjp(c, S[S_Q4], lk, mu, gf_acc);
  add_fields(c, lam0, mu, c->g.N * 5);
  lin2(c, dt / 3.0, l1, dt, mu, lk);
  rhs_direct_vjp(c, S[S_Q3], lk, mu, gf_acc);
  add_fields(c, lam0, mu, c->g.N * 5);
  lin2(c, dt / 3.0, l1, dth, mu, lk);
  rhs_direct_vjp(c, S[S_Q2], lk, mu, gf_acc);
  add_fields(c, lam0, mu, c->g.N * 5);
  lin2(c, dt / 6.0, l1, dth, mu, lk);
  rhs_direct_vjp(c, q0, lk, mu, gf_acc);
  add_fields(c, lam0, mu, c->g.N * 5);
}

void diff_transpose(cruna_ctx *c, int d, const double *in, double *out, double h, double *scratch) {
  if (!c->dopT_built[d]) {
    build_transpose(c, c->dop[d], c->dhf[d], c->dopT[d]);
    c->dopT_built[d] = true;
  }
  apply_T(c, c->dopT[d], d, in, out, diff_scale(c, d, h), 1, 0, scratch);
}

}  // namespace cruna
