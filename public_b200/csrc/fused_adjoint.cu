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
  double p_ref;        // FP32 stencils: pressure offset differenced instead of p (0 in FP64)
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

// plane fields: 0..4 qs1..qs5, 5 p - p_ref, 6 u, 7 v ; column fields: 0..4 qs1..qs5, 5 p - p_ref, 6 w.
// T is the type of the shared-memory fields and of the derivatives (double, or float for the
// FP32-stencil precision); the assembly and the RK update stay in double.
template <typename T, int R, bool PER>
__global__ void __launch_bounds__(TX *TY, sizeof(T) == 4 ? 3 : 2) k_adj_pass(const __grid_constant__ AdjArgs a) {
  constexpr int PW = TX + 2 * R, PH = TY + 2 * R, PS = PW * PH;
  constexpr int NS = ring_slots(R);
  constexpr int NPF = 8, NRF = 7, RS = TX * TY;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *plane = reinterpret_cast<T *>(smem_raw);          // [NPF][PH][PW]
  T *ring = plane + NPF * PS;                          // [NS][NRF][TY*TX]
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int k0 = blockIdx.z * a.kc;
  const int k1 = min(k0 + a.kc, a.g.n3);
  const DirOpF &ox = a.op[0], &oy = a.op[1], &oz = a.op[2];
  const int n1 = a.g.n1, n12 = a.g.n1 * a.g.n2;
  const int gi = gidx(ox, i0 + tx), gj = gidx(oy, j0 + ty);
  const long long N = a.g.N;
  const bool inside = (i0 + tx) < a.g.n1 && (j0 + ty) < a.g.n2;
  const bool col = gi >= 0 && gj >= 0;
  const int colpt = gi + n1 * gj;
  const double *S0 = a.qs, *S1 = a.qs + N, *S2 = a.qs + 2 * N, *S3 = a.qs + 3 * N, *S4 = a.qs + 4 * N;
  const double *Q0 = a.q, *Q1 = a.q + N, *Q2 = a.q + 2 * N, *Q3 = a.q + 3 * N, *Q4 = a.q + 4 * N;
  HaloSet<R> hs;
  hs.init(ox, oy, i0, j0, tid, n1);

  auto put_ring = [&](int kk, const double *v8) {
    // v8: qs1..qs5, rho, rho*w, p
    T *rp = ring + (((kk % NS) + NS) % NS) * NRF * RS + tid;
#pragma unroll
    for (int f = 0; f < 5; ++f) rp[f * RS] = T(v8[f]);
    rp[5 * RS] = T(v8[7] - a.p_ref);
    rp[6 * RS] = T(v8[6] * (1.0 / v8[5]));
  };
  auto load8 = [&](long long pt, double *v8) {
    v8[0] = S0[pt]; v8[1] = S1[pt]; v8[2] = S2[pt]; v8[3] = S3[pt]; v8[4] = S4[pt];
    v8[5] = Q0[pt]; v8[6] = Q3[pt]; v8[7] = Q4[pt];
  };
  for (int kk = k0 - R; kk < k0 + R; ++kk) {
    const int gk = gidx(oz, kk);
    if (gk < 0 || !col) continue;
    double v8[8];
    load8(colpt + (long long)n12 * gk, v8);
    put_ring(kk, v8);
  }
  // register prefetch of the ring plane k+R+1 and the centre (rho, rho*u, rho*v) of plane k+1
  double pf[8];
  double pc[4] = {1.0, 0.0, 0.0, 1.0};
  int pf_ok = 0;
  auto prefetch = [&](int kk, int kc) {
    const int gk = gidx(oz, kk);
    pf_ok = (gk >= 0 && col);
    if (pf_ok) load8(colpt + (long long)n12 * gk, pf);
    if (col && kc < k1) {
      const long long pt = colpt + (long long)n12 * kc;
      pc[0] = Q0[pt];
      pc[1] = Q1[pt];
      pc[2] = Q2[pt];
      pc[3] = Q4[pt];
    }
  };
  prefetch(k0 + R, k0);
  constexpr int NHT = HaloSet<R>::PER_THREAD;
  double hv[NHT][9];      // qs1..qs5, rho, rho*u, rho*v, p of the halo cells, one plane ahead
  auto halo_fetch = [&](int kk) {
    const long long kofs = (long long)n12 * kk;
#pragma unroll
    for (int h = 0; h < NHT; ++h) {
      if (hs.goff[h] < 0) continue;
      const long long pt = hs.goff[h] + kofs;
      hv[h][0] = S0[pt]; hv[h][1] = S1[pt]; hv[h][2] = S2[pt]; hv[h][3] = S3[pt]; hv[h][4] = S4[pt];
      hv[h][5] = Q0[pt]; hv[h][6] = Q1[pt]; hv[h][7] = Q2[pt]; hv[h][8] = Q4[pt];
    }
  };
  halo_fetch(k0);
  for (int k = k0; k < k1; ++k) {
    if (pf_ok) put_ring(k + R, pf);
    const int slot = k % NS;
    const double rho_c = pc[0], p_c = pc[3];
    const double ir = 1.0 / rho_c;                            // ns_rho_rhou_p.f90:294
    const double u1 = pc[1] * ir, u2 = pc[2] * ir;
    {
      T *c = plane + (ty + R) * PW + (tx + R);
      const T *rp = ring + slot * NRF * RS + tid;
#pragma unroll
      for (int f = 0; f < 6; ++f) c[f * PS] = rp[f * RS];
      c[6 * PS] = T(u1);
      c[7 * PS] = T(u2);
    }
    const long long kofs = (long long)n12 * k;
    // epilogue inputs of this plane, issued before the barrier so their latency overlaps the stencils
    const long long opt = (i0 + tx) + (long long)n1 * (j0 + ty) + kofs;
    double e_src[5] = {0, 0, 0, 0, 0}, e_q0[5] = {0, 0, 0, 0, 0}, e_acc[5] = {0, 0, 0, 0, 0};
    if (inside) {
      if (a.src) {
#pragma unroll
        for (int v = 0; v < 5; ++v) e_src[v] = a.src[opt + v * N];
      }
      if (a.stage != 0) {
#pragma unroll
        for (int v = 0; v < 5; ++v) e_q0[v] = a.q0[opt + v * N];
      }
      if (a.stage >= 2) {
#pragma unroll
        for (int v = 0; v < 5; ++v) e_acc[v] = a.acc[opt + v * N];
      }
    }
#pragma unroll
    for (int h = 0; h < NHT; ++h) {
      if (hs.goff[h] < 0) continue;
      T *c = plane + hs.cell[h];
      c[0 * PS] = T(hv[h][0]); c[1 * PS] = T(hv[h][1]); c[2 * PS] = T(hv[h][2]); c[3 * PS] = T(hv[h][3]);
      c[4 * PS] = T(hv[h][4]);
      const double hir = 1.0 / hv[h][5];
      c[5 * PS] = T(hv[h][8] - a.p_ref);
      c[6 * PS] = T(hv[h][6] * hir);
      c[7 * PS] = T(hv[h][7] * hir);
    }
    prefetch(k + R + 1, k + 1);
    if (k + 1 < k1) halo_fetch(k + 1);
    __syncthreads();
    if (inside) {
      const int i = i0 + tx, j = j0 + ty;
      const T *c = plane + (ty + R) * PW + (tx + R);
      int so[NS];
#pragma unroll
      for (int m = -R; m <= R; ++m) so[m + R] = ((slot + m + NS) % NS) * NRF * RS + tid;
      const double qs5 = c[4 * PS];
      const double gm1 = a.gamma - 1.0;
      const double u3 = ring[so[R] + 6 * RS];
      const double gpr = a.gamma * p_c / (rho_c * gm1);         // :293
      double r1 = 0.0, r2 = 0.0, r3 = 0.0, r4 = 0.0, r5 = 0.0;  // :296
      {
        const double s = ox.scale;
        const double A = D1<T, R, PER>(ox, c, 1, i) * s, B = D1<T, R, PER>(ox, c + PS, 1, i) * s,
                     Cc = D1<T, R, PER>(ox, c + 2 * PS, 1, i) * s, D = D1<T, R, PER>(ox, c + 3 * PS, 1, i) * s,
                     E = D1<T, R, PER>(ox, c + 4 * PS, 1, i) * s;
        const double Sx = D2<T, R, PER>(ox, c + 6 * PS, c + 4 * PS, 1, i) * s;
        const double P = D1<T, R, PER>(ox, c + 5 * PS, 1, i) * s;
        adj_dir(0, u1, u2, u3, gpr, ir, qs5, a.gamma, A, B, Cc, D, E, Sx, P, r1, r2, r3, r4, r5);
      }
      {
        const double s = oy.scale;
        const double A = D1<T, R, PER>(oy, c, PW, j) * s, B = D1<T, R, PER>(oy, c + PS, PW, j) * s,
                     Cc = D1<T, R, PER>(oy, c + 2 * PS, PW, j) * s, D = D1<T, R, PER>(oy, c + 3 * PS, PW, j) * s,
                     E = D1<T, R, PER>(oy, c + 4 * PS, PW, j) * s;
        const double Sy = D2<T, R, PER>(oy, c + 7 * PS, c + 4 * PS, PW, j) * s;
        const double P = D1<T, R, PER>(oy, c + 5 * PS, PW, j) * s;
        adj_dir(1, u1, u2, u3, gpr, ir, qs5, a.gamma, A, B, Cc, D, E, Sy, P, r1, r2, r3, r4, r5);
      }
      {
        const double s = oz.scale;
        T zc[NS], zq5[NS];
        double Z[5];
#pragma unroll
        for (int m = 0; m < NS; ++m) zq5[m] = ring[so[m] + 4 * RS];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
#pragma unroll
          for (int m = 0; m < NS; ++m) zc[m] = ring[so[m] + f * RS];
          Z[f] = Dz1<T, R, PER>(oz, zc, k) * s;
        }
        Z[4] = Dz1<T, R, PER>(oz, zq5, k) * s;
#pragma unroll
        for (int m = 0; m < NS; ++m) zc[m] = ring[so[m] + 6 * RS];
        const double Sz = Dz2<T, R, PER>(oz, zc, zq5, k) * s;
#pragma unroll
        for (int m = 0; m < NS; ++m) zc[m] = ring[so[m] + 5 * RS];
        const double P = Dz1<T, R, PER>(oz, zc, k) * s;
        adj_dir(2, u1, u2, u3, gpr, ir, qs5, a.gamma, Z[0], Z[1], Z[2], Z[3], Z[4], Sz, P, r1, r2, r3, r4, r5);
      }
      if (a.src) {                                              // :512
        r1 = r1 + e_src[0]; r2 = r2 + e_src[1]; r3 = r3 + e_src[2]; r4 = r4 + e_src[3]; r5 = r5 + e_src[4];
      }
      const double kv[5] = {r1, r2, r3, r4, r5};
      if (a.stage == 0) {
#pragma unroll
        for (int v = 0; v < 5; ++v) a.rhs[opt + v * N] = kv[v];
      } else {
        const double dt = a.dt, dth = a.dt * 0.5;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const long long o = opt + v * N;
          if (a.stage == 1) {
            a.acc[o] = kv[v];
            a.qnext[o] = e_q0[v] + dth * kv[v];
          } else if (a.stage == 2) {
            a.acc[o] = e_acc[v] + 2.0 * kv[v];
            a.qnext[o] = e_q0[v] + dth * kv[v];
          } else if (a.stage == 3) {
            a.acc[o] = e_acc[v] + 2.0 * kv[v];
            a.qnext[o] = e_q0[v] + dt * kv[v];
          } else {
            a.qnext[o] = e_q0[v] + dt / 6.0 * (e_acc[v] + kv[v]);
          }
        }
      }
    }
    __syncthreads();
  }
}

template <typename T, int R>
size_t smem_adj() {
  return sizeof(T) * (8 * (TX + 2 * R) * (TY + 2 * R) + ring_slots(R) * 7 * TX * TY);
}

template <typename T, int R, bool PER>
void launch_adj(cruna_ctx *c, AdjArgs &a) {
  static bool configured = false;
  if (!configured) {
    CRUNA_CUDA_CHECK(cudaFuncSetAttribute(k_adj_pass<T, R, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem_adj<T, R>()));
    configured = true;
  }
  const int bx = (c->g.n1 + TX - 1) / TX, by = (c->g.n2 + TY - 1) / TY;
  int nz = 1;
  a.kc = z_chunk(c->g.n3, bx, by, R, nz);
  ProfScope ps(c, "adj_pass");
  k_adj_pass<T, R, PER><<<dim3(bx, by, nz), dim3(TX, TY), smem_adj<T, R>(), c->stream>>>(a);
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
  const bool fp32 = c->cfg.precision == CRUNA_FP32_STENCIL;
  if (fp32 && !c->refs_set) {  // the pressure offset of the FP32 stencils (as the direct passes)
    double h[2] = {0.0, 1.0};
    CRUNA_CUDA_CHECK(cudaMemcpyAsync(&h[0], q + 4 * c->g.N, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CRUNA_CUDA_CHECK(cudaMemcpyAsync(&h[1], q, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    c->p_ref = h[0];
    c->T_ref = c->cfg.W / c->cfg.R * h[0] / h[1];
    c->refs_set = true;
  }
  AdjArgs a;
  a.g = c->g;
  a.p_ref = fp32 ? c->p_ref : 0.0;
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
  const int Rl = R <= 2 ? 2 : 4;
  bool per = true;
  for (int d = 0; d < 3; ++d) per = per && c->dop[d].kind == OP_STENCIL && c->dop[d].periodic && c->dop[d].r == Rl;
  if (fp32) {
    if (Rl == 2) {
      if (per) launch_adj<float, 2, true>(c, a);
      else launch_adj<float, 2, false>(c, a);
    } else {
      if (per) launch_adj<float, 4, true>(c, a);
      else launch_adj<float, 4, false>(c, a);
    }
  } else if (Rl == 2) {
    if (per) launch_adj<double, 2, true>(c, a);
    else launch_adj<double, 2, false>(c, a);
  } else {
    if (per) launch_adj<double, 4, true>(c, a);
    else launch_adj<double, 4, false>(c, a);
  }
  if (stage == 0 || split) {
    if (c->has_rhs_bc) bc_rhss(c, rhs, qs, nullptr);                // :518 (without q)
    if (split) rk_stage(c, stage, dt, rhs, qs0, acc, qnext);
  }
}

}  // namespace cruna
