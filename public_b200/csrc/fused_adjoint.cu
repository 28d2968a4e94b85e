// Fused explicit-stencil adjoint RHS of right_hand_side_adjoint_3d (src/equations/ns_rho_rhou_p.f90:
// 257-536, the continuous inviscid adjoint) with the RK4 stage update of time_stepper_adjoint
// (src/time/rk_o4_e.f90:92-97) in the epilogue.
//
// One z-marching pass per RK stage evaluates the reference's 21 derivative calls -- D_d qs(1..5),
// D_d(u_d*qs5) and D_d p for d = 1, 2, 3 -- from one shared-memory x-y plane (8 fields with R-wide
// halos) and per-thread z columns (7 fields), then assembles the five adjoint equations in the
// reference's order, adds the source g and updates the stage.
#include <cmath>
#include <stdexcept>

#include "cruna_internal.cuh"
#include "fused_common.cuh"

namespace cruna {

using namespace fz;

namespace {

struct AdjArgs {
  Grid g;
  DirOpF op[3];
  int kc;
  double gamma;
  const double *qs;    // stage input (5 fields)
  const double *q;     // frozen direct state (5 fields)
  const double *src;   // adjoint source g (5 fields) or null
  double *rhs;
  int stage;
  double dt;
  const double *q0;
  double *acc;
  double *qnext;
};

// per-direction contribution in the reference's order (ns_rho_rhou_p.f90:317-370 / 386-440 / 456-509)
__device__ __forceinline__ void adj_dir(int d, double u1, double u2, double u3, double gpr, double ir,
                                        double qs5, double gamma, double a, double b, double c, double dd,
                                        double e, double s, double pd, double &r1, double &r2, double &r3,
                                        double &r4, double &r5) {
  const double gm1 = gamma - 1.0;
  if (d == 0) {
    r1 = r1 + (u1 * u1) * b + (u1 * u2) * c + (u1 * u3) * dd + gpr * u1 * e;
    r2 = r2 - a - 2.0 * u1 * b - u2 * c - u3 * dd - gpr * e;
    r3 = r3 - u1 * c;
    r4 = r4 - u1 * dd;
    r5 = r5 - gm1 * b - gamma * u1 * e;
    r5 = r5 - gm1 * (-s);
    r1 = r1 + qs5 * u1 * ir * pd;
    r2 = r2 - qs5 * ir * pd;
  } else if (d == 1) {
    r1 = r1 + (u2 * u1) * b + (u2 * u2) * c + (u2 * u3) * dd + gpr * u2 * e;
    r2 = r2 - u2 * b;
    r3 = r3 - a - u1 * b - 2 * u2 * c - u3 * dd - gpr * e;
    r4 = r4 - u2 * dd;
    r5 = r5 - gm1 * c - gamma * u2 * e;
    r5 = r5 - gm1 * (-s);
    r1 = r1 + qs5 * u2 * ir * pd;
    r3 = r3 - qs5 * ir * pd;
  } else {
    r1 = r1 + (u3 * u1) * b + (u3 * u2) * c + (u3 * u3) * dd + gpr * u3 * e;
    r2 = r2 - u3 * b;
    r3 = r3 - u3 * c;
    r4 = r4 - a - u1 * b - u2 * c - 2 * u3 * dd - gpr * e;
    r5 = r5 - gm1 * dd - gamma * u3 * e;
    r5 = r5 - gm1 * (-s);
    r1 = r1 + qs5 * u3 * ir * pd;
    r4 = r4 - qs5 * ir * pd;
  }
}

// plane fields: 0..4 qs1..qs5, 5 p, 6 u, 7 v ; column fields: 0..4 qs1..qs5, 5 p, 6 w
template <int R>
__global__ void __launch_bounds__(TX *TY, 2) k_adj_pass(const __grid_constant__ AdjArgs a) {
  using T = double;
  constexpr int PW = TX + 2 * R, PH = TY + 2 * R, PS = PW * PH;
  constexpr int NS = ring_slots(R);
  constexpr int NPF = 8, NRF = 7;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *plane = reinterpret_cast<T *>(smem_raw);          // [NPF][PH][PW]
  T *ring = plane + NPF * PS;                          // [NS][NRF][TY*TX]
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int k0 = blockIdx.z * a.kc;
  const int k1 = min(k0 + a.kc, a.g.n3);
  const DirOpF &ox = a.op[0], &oy = a.op[1], &oz = a.op[2];
  const int gi = gidx(ox, i0 + tx), gj = gidx(oy, j0 + ty);
  const long long N = a.g.N, n1 = a.g.n1, n12 = (long long)a.g.n1 * a.g.n2;
  const bool inside = (i0 + tx) < a.g.n1 && (j0 + ty) < a.g.n2;
  const bool col = gi >= 0 && gj >= 0;
  const long long colpt = gi + n1 * gj;

  auto ring_at = [&](int slot, int f) -> T * { return ring + (slot * NRF + f) * (TX * TY) + tid; };
  auto put_ring = [&](int kk, const double *qsv, double rho, double rw, double p) {
    const int sl = ((kk % NS) + NS) % NS;
#pragma unroll
    for (int v = 0; v < 5; ++v) *ring_at(sl, v) = qsv[v];
    *ring_at(sl, 5) = p;
    *ring_at(sl, 6) = rw * (1.0 / rho);
  };
  for (int kk = k0 - R; kk < k0 + R; ++kk) {
    const int gk = gidx(oz, kk);
    if (gk < 0 || !col) continue;
    const long long pt = colpt + n12 * gk;
    double qsv[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) qsv[v] = a.qs[pt + v * N];
    put_ring(kk, qsv, a.q[pt], a.q[pt + 3 * N], a.q[pt + 4 * N]);
  }
  // register prefetch: ring plane k+R (qs 5 + rho, rho*w, p) and centre rho, rho*u, rho*v of plane k
  double pf[8];
  double pc[3] = {1.0, 0.0, 0.0};
  int pf_k = -1;
  auto prefetch = [&](int kk, int kc) {
    const int gk = gidx(oz, kk);
    pf_k = (gk >= 0 && col) ? gk : -1;
    if (pf_k >= 0) {
      const long long pt = colpt + n12 * gk;
#pragma unroll
      for (int v = 0; v < 5; ++v) pf[v] = a.qs[pt + v * N];
      pf[5] = a.q[pt];
      pf[6] = a.q[pt + 3 * N];
      pf[7] = a.q[pt + 4 * N];
    }
    if (col && kc < k1) {
      const long long pt = colpt + n12 * kc;
      pc[0] = a.q[pt];
      pc[1] = a.q[pt + N];
      pc[2] = a.q[pt + 2 * N];
    }
  };
  prefetch(k0 + R, k0);
  constexpr int nhalo = 2 * R * (TX + TY);
  for (int k = k0; k < k1; ++k) {
    if (pf_k >= 0) put_ring(k + R, pf, pf[5], pf[6], pf[7]);
    const int slot = k % NS;
    const double rho_c = pc[0], ir_c = 1.0 / pc[0];
    {
      T *c = plane + (ty + R) * PW + (tx + R);
#pragma unroll
      for (int v = 0; v < 6; ++v) c[v * PS] = *ring_at(slot, v);
      c[6 * PS] = pc[1] * ir_c;
      c[7 * PS] = pc[2] * ir_c;
    }
    prefetch(k + R + 1, k + 1);
    for (int h = tid; h < nhalo; h += TX * TY) {
      int lx, ly;
      if (h < 2 * R * TY) {
        const int side = h / (R * TY), e = h % (R * TY);
        ly = e / R;
        lx = side == 0 ? -R + e % R : TX + e % R;
      } else {
        const int e2 = h - 2 * R * TY;
        const int side = e2 / (R * TX), e = e2 % (R * TX);
        lx = e % TX;
        ly = side == 0 ? -R + e / TX : TY + e / TX;
      }
      const int hi = gidx(ox, i0 + lx), hj = gidx(oy, j0 + ly);
      if (hi < 0 || hj < 0) continue;
      const long long pt = hi + n1 * hj + n12 * k;
      T *c = plane + (ly + R) * PW + (lx + R);
#pragma unroll
      for (int v = 0; v < 5; ++v) c[v * PS] = a.qs[pt + v * N];
      const double ir = 1.0 / a.q[pt];
      c[5 * PS] = a.q[pt + 4 * N];
      c[6 * PS] = a.q[pt + N] * ir;
      c[7 * PS] = a.q[pt + 2 * N] * ir;
    }
    __syncthreads();
    if (inside) {
      const int i = i0 + tx, j = j0 + ty;
      const T *c = plane + (ty + R) * PW + (tx + R);
      T zq[5][NS], zp[NS], zw[NS];
#pragma unroll
      for (int m = -R; m <= R; ++m) {
        const int sl = (slot + m + NS) % NS;
#pragma unroll
        for (int v = 0; v < 5; ++v) zq[v][m + R] = *ring_at(sl, v);
        zp[m + R] = *ring_at(sl, 5);
        zw[m + R] = *ring_at(sl, 6);
      }
      const double u1 = c[6 * PS], u2 = c[7 * PS], u3 = zw[R];
      const double qs5 = zq[4][R];
      const double gm1 = a.gamma - 1.0;
      const double gpr = a.gamma * zp[R] / (rho_c * gm1);       // :293
      const double ir = 1.0 / rho_c;                            // :294
      double r1 = 0.0, r2 = 0.0, r3 = 0.0, r4 = 0.0, r5 = 0.0;  // :296
      {
        const double s = ox.scale;
        const double A = dsm<T, R>(ox, c, 1, i) * s, B = dsm<T, R>(ox, c + PS, 1, i) * s,
                     Cc = dsm<T, R>(ox, c + 2 * PS, 1, i) * s, D = dsm<T, R>(ox, c + 3 * PS, 1, i) * s,
                     E = dsm<T, R>(ox, c + 4 * PS, 1, i) * s;
        const double S = dsm2<T, R>(ox, c + 6 * PS, c + 4 * PS, 1, i) * s;
        const double P = dsm<T, R>(ox, c + 5 * PS, 1, i) * s;
        adj_dir(0, u1, u2, u3, gpr, ir, qs5, a.gamma, A, B, Cc, D, E, S, P, r1, r2, r3, r4, r5);
      }
      {
        const double s = oy.scale;
        const double A = dsm<T, R>(oy, c, PW, j) * s, B = dsm<T, R>(oy, c + PS, PW, j) * s,
                     Cc = dsm<T, R>(oy, c + 2 * PS, PW, j) * s, D = dsm<T, R>(oy, c + 3 * PS, PW, j) * s,
                     E = dsm<T, R>(oy, c + 4 * PS, PW, j) * s;
        const double S = dsm2<T, R>(oy, c + 7 * PS, c + 4 * PS, PW, j) * s;
        const double P = dsm<T, R>(oy, c + 5 * PS, PW, j) * s;
        adj_dir(1, u1, u2, u3, gpr, ir, qs5, a.gamma, A, B, Cc, D, E, S, P, r1, r2, r3, r4, r5);
      }
      {
        const double s = oz.scale;
        const double A = dsz<T, R>(oz, zq[0], k) * s, B = dsz<T, R>(oz, zq[1], k) * s,
                     Cc = dsz<T, R>(oz, zq[2], k) * s, D = dsz<T, R>(oz, zq[3], k) * s,
                     E = dsz<T, R>(oz, zq[4], k) * s;
        const double S = dsz2<T, R>(oz, zw, zq[4], k) * s;
        const double P = dsz<T, R>(oz, zp, k) * s;
        adj_dir(2, u1, u2, u3, gpr, ir, qs5, a.gamma, A, B, Cc, D, E, S, P, r1, r2, r3, r4, r5);
      }
      const long long pt = i + n1 * j + n12 * k;
      if (a.src) {                                              // :512
        r1 = r1 + a.src[pt]; r2 = r2 + a.src[pt + N]; r3 = r3 + a.src[pt + 2 * N];
        r4 = r4 + a.src[pt + 3 * N]; r5 = r5 + a.src[pt + 4 * N];
      }
      const double kv[5] = {r1, r2, r3, r4, r5};
      if (a.stage == 0) {
#pragma unroll
        for (int v = 0; v < 5; ++v) a.rhs[pt + v * N] = kv[v];
      } else {
        const double dt = a.dt, dth = a.dt * 0.5;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const long long o = pt + v * N;
          const double q0 = a.q0[o];
          if (a.stage == 1) {
            a.acc[o] = kv[v];
            a.qnext[o] = q0 + dth * kv[v];
          } else if (a.stage == 2) {
            a.acc[o] = a.acc[o] + 2.0 * kv[v];
            a.qnext[o] = q0 + dth * kv[v];
          } else if (a.stage == 3) {
            a.acc[o] = a.acc[o] + 2.0 * kv[v];
            a.qnext[o] = q0 + dt * kv[v];
          } else {
            a.qnext[o] = q0 + dt / 6.0 * (a.acc[o] + kv[v]);
          }
        }
      }
    }
    __syncthreads();
  }
}

template <int R>
size_t smem_adj() {
  return sizeof(double) * (8 * (TX + 2 * R) * (TY + 2 * R) + ring_slots(R) * 7 * TX * TY);
}

template <int R>
void launch_adj(cruna_ctx *c, AdjArgs &a) {
  static bool configured = false;
  if (!configured) {
    CRUNA_CUDA_CHECK(cudaFuncSetAttribute(k_adj_pass<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem_adj<R>()));
    configured = true;
  }
  const int bx = (c->g.n1 + TX - 1) / TX, by = (c->g.n2 + TY - 1) / TY;
  const int n3 = c->g.n3;
  int nz = std::max(1, std::min(n3, (4 * 148 + bx * by - 1) / (bx * by)));
  int kc = (n3 + nz - 1) / nz;
  kc = std::max(kc, std::min(n3, 4 * R));
  nz = (n3 + kc - 1) / kc;
  a.kc = kc;
  ProfScope ps(c, "adj_pass");
  k_adj_pass<R><<<dim3(bx, by, nz), dim3(TX, TY), smem_adj<R>(), c->stream>>>(a);
  CRUNA_LAUNCH_CHECK(c);
}

}  // namespace

// one adjoint RHS evaluation (stage 0) or RK stage (1..4) through the fused pass
void rhs_adjoint_fused(cruna_ctx *c, const double *qs_in, const double *q, const double *g, double *rhs,
                       int stage, const double *qs0, double *acc, double *qnext, double dt) {
  const double *qs = qs_in;
  if (c->has_q_bc) {                                               // ns_rho_rhou_p.f90:287-290
    copy_state(c, c->st[4], qs_in, 5);
    bc_qs(c, c->st[4], q, 0);
    qs = c->st[4];
  }
  AdjArgs a;
  a.g = c->g;
  for (int d = 0; d < 3; ++d) a.op[d] = to_dir(c->dop[d], c->dx[d], true);
  a.gamma = c->cfg.gamma;
  a.qs = qs;
  a.q = q;
  a.src = g;
  a.dt = dt;
  a.q0 = qs0;
  a.acc = acc;
  a.qnext = qnext;
  const bool split = stage != 0 && c->has_rhs_bc;
  a.stage = split ? 0 : stage;
  a.rhs = (stage == 0 || split) ? rhs : nullptr;
  int R = 0;
  for (int d = 0; d < 3; ++d) R = std::max(R, halo_of(c->dop[d]));
  if (R <= 2) launch_adj<2>(c, a);
  else launch_adj<4>(c, a);
  if (stage == 0 || split) {
    if (c->has_rhs_bc) bc_rhss(c, rhs, qs, nullptr);                // :518 (without q)
    if (split) rk_stage(c, stage, dt, rhs, qs0, acc, qnext);
  }
}

}  // namespace cruna
