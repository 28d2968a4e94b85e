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
#include <type_traits>

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
  static const int res = resident_blocks(k_adj_pass<T, R, PER>, TX * TY, smem_adj<T, R>());
  int nz = 1;
  a.kc = z_chunk_balanced(c->g.n3, bx * by, res, device_sms(), R, nz);
  ProfScope ps(c, "adj_pass");
  k_adj_pass<T, R, PER><<<dim3(bx, by, nz), dim3(TX, TY), smem_adj<T, R>(), c->stream>>>(a);
  CRUNA_LAUNCH_CHECK(c);
}

// ------------------------------------------------------------------------------------------------
// TMA-fed variant (FP64).  One thread streams every input of the pass into shared memory with
// cp.async.bulk.tensor, so no registers hold loads in flight:
//   * the (TX+2R) x (TY+2R) tile of all five fields of qs and of q, one plane ahead, into a two-stage
//     ring (x/y stencils);
//   * the TX x TY column box of qs and q R planes ahead (the new entry of the z columns), issued as
//     soon as the previous one has been read;
//   * the column boxes of q0 and acc of the RK stage update, issued one plane ahead.
// The z columns (qs1..qs5, p, w over 2R+1 planes) live in registers and shift by one plane per step.
// TMA fills cells outside the grid with zeros.  At a periodic x edge whose wrapped cells form one
// R-wide strip, a side box brings that strip (TMA, one plane ahead) and the threads copy it into the
// tile; any other wrapped cell (y edges, grids narrower than a tile) is patched with plain loads.  The
// products u*qs5 (x rows) and v*qs5 (y columns) are formed once per cell in shared memory, the centre
// cells with the owning thread's 1/rho.  Every mbarrier wait is bounded; a block whose wait runs out
// sets the error flag, waits (bounded) for its copies in flight and returns.
// ------------------------------------------------------------------------------------------------
struct AdjTmaMaps {
  CUtensorMap qs_tile, q_tile;   // box (TX+2R, TY+2R, 1, 5)
  CUtensorMap qs_col, q_col;     // box (TX, TY, 1, 5)
  CUtensorMap qs_side, q_side;   // box (R, TY, 1, 5)
  CUtensorMap q0_col, acc_col;   // box (TX, TY, 1, 5) of the RK stage inputs (unused at stage 0)
};

template <int R>
struct AdjTmaLayout {
  static constexpr int PW = TX + 2 * R, PH = TY + 2 * R, PS = PW * PH;
  static constexpr int TILE = 5 * PS;             // doubles of one tensor's tile (5 fields)
  static constexpr int COL = 5 * TX * TY;         // doubles of one tensor's column box
  static constexpr int SIDE = 5 * TY * R;         // doubles of one tensor's side strip
  static constexpr int SIDEP = ((SIDE + 15) / 16) * 16;   // its slot (128-byte multiple)
  // offsets in doubles (every TMA destination a multiple of 128 bytes)
  static constexpr int o_tile = 0;                       // [stage][tensor 0 qs / 1 q][field][PH][PW]
  static constexpr int o_col = o_tile + 2 * 2 * TILE;    // [tensor][field][TY][TX]  (plane k + R)
  static constexpr int o_epi = o_col + 2 * COL;          // [0 q0 / 1 acc][field][TY][TX]  (plane k)
  static constexpr int o_side = o_epi + 2 * COL;         // [stage][tensor][field][TY][R]
  static constexpr int o_px = o_side + 2 * 2 * SIDEP;     // [TY][PW]   u*qs5
  static constexpr int o_py = o_px + TY * PW;            // [PH][TX]   v*qs5
  static constexpr int o_bar = o_py + PH * TX;           // mbarriers: tile[2], col, epi
  static constexpr size_t bytes = sizeof(double) * o_bar + 4 * sizeof(uint64_t);
  static constexpr uint32_t tile_tx = 2u * TILE * 8u, col_tx = 2u * COL * 8u, side_tx = 2u * SIDE * 8u;
  static constexpr int NPT = (PS + TX * TY - 1) / (TX * TY);   // tile cells per thread (plain patches)
  static constexpr int NHALO = 2 * R * TY + 2 * R * TX;       // non-centre product cells
};

template <int R, bool PER>
__global__ void __launch_bounds__(TX *TY, 2) k_adj_tma(const __grid_constant__ AdjArgs a,
                                                      const __grid_constant__ AdjTmaMaps m, int *err) {
  using L = AdjTmaLayout<R>;
  constexpr int PW = L::PW, PS = L::PS;
  constexpr int NS = ring_slots(R);
  constexpr int NQ = 7;                          // column fields: qs1..qs5, p, w
  extern __shared__ __align__(128) double sm[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + L::o_bar);   // [0..1] tile stages, [2] column, [3] epilogue
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int k0 = blockIdx.z * a.kc;
  const int k1 = min(k0 + a.kc, a.g.n3);
  const DirOpF &ox = a.op[0], &oy = a.op[1], &oz = a.op[2];
  const int n1 = a.g.n1, n2 = a.g.n2, n12 = a.g.n1 * a.g.n2;
  const long long N = a.g.N;
  const bool inside = (i0 + tx) < n1 && (j0 + ty) < n2;
  const bool epi = a.stage != 0;

  // periodic x edge: 1 = wrapped strip on the left (columns 0..R-1), 2 = on the right (TX+R..TX+2R-1),
  // both brought by a side box; 3 = wrapped cells otherwise (plain patches)
  int xmode = 0;
  if (ox.kind != 0 && ox.periodic) {
    const bool lo = i0 - R < 0, hi = i0 + TX + R > n1;
    if (lo && !hi && n1 >= R) xmode = 1;
    else if (hi && !lo && i0 + TX == n1) xmode = 2;
    else if (lo || hi) xmode = 3;
  }
  // tile cells this thread patches with plain loads: in-plane source offset and shared-memory cell
  int pcell[L::NPT], poff[L::NPT];
  int mine = 0;
#pragma unroll
  for (int c = 0; c < L::NPT; ++c) {
    const int cell = tid + c * TX * TY;
    pcell[c] = -1;
    poff[c] = 0;
    if (cell < PS) {
      const int lx = cell % PW - R, ly = cell / PW - R;
      const bool hx = lx < 0 || lx >= TX, hy = ly < 0 || ly >= TY;
      const int gi = i0 + lx, gj = j0 + ly;
      const bool outx = gi < 0 || gi >= n1, outy = gj < 0 || gj >= n2;
      const bool side_covers = (xmode == 1 || xmode == 2) && outx && !hy && !outy;
      if (!(hx && hy) && (outx || outy) && !side_covers) {    // corners are never read
        const int wi = gidx(ox, gi), wj = gidx(oy, gj);
        if (wi >= 0 && wj >= 0) {
          pcell[c] = cell;
          poff[c] = wi + n1 * wj;
          mine = 1;
        }
      }
    }
  }
  const bool patch_block = __syncthreads_or(mine) != 0;

  auto issue_tile = [&](int k, int st) {
    double *tq = sm + L::o_tile + st * 2 * L::TILE;
    const bool side = xmode == 1 || xmode == 2;
    tma_expect(&bar[st], L::tile_tx + (side ? L::side_tx : 0u));
    tma_load4(&m.qs_tile, tq, &bar[st], i0 - R, j0 - R, k, 0);
    tma_load4(&m.q_tile, tq + L::TILE, &bar[st], i0 - R, j0 - R, k, 0);
    if (side) {
      double *sd = sm + L::o_side + st * 2 * L::SIDEP;
      const int xs = xmode == 1 ? n1 - R : 0;
      tma_load4(&m.qs_side, sd, &bar[st], xs, j0, k, 0);
      tma_load4(&m.q_side, sd + L::SIDEP, &bar[st], xs, j0, k, 0);
    }
  };
  auto issue_col = [&](int k) {                   // column box of plane k + R
    const int gk = gidx(oz, k + R);
    if (gk >= 0) {
      tma_expect(&bar[2], L::col_tx);
      tma_load4(&m.qs_col, sm + L::o_col, &bar[2], i0, j0, gk, 0);
      tma_load4(&m.q_col, sm + L::o_col + L::COL, &bar[2], i0, j0, gk, 0);
    } else {
      mbar_arrive(&bar[2]);
    }
  };
  auto issue_epi = [&](int k) {                   // q0 (and acc from stage 2 on) of plane k
    tma_expect(&bar[3], (a.stage >= 2 ? 2u : 1u) * L::COL * 8u);
    tma_load4(&m.q0_col, sm + L::o_epi, &bar[3], i0, j0, k, 0);
    if (a.stage >= 2) tma_load4(&m.acc_col, sm + L::o_epi + L::COL, &bar[3], i0, j0, k, 0);
  };
  int n_tile0 = 0, n_tile1 = 0, n_col = 0, n_epi = 0;   // copies issued per barrier (thread 0's view)
  if (tid == 0) {
    for (int b = 0; b < 4; ++b) tc::mbar_init(&bar[b], 1);
    issue_tile(k0, 0);
    n_tile0 = 1;
    issue_col(k0);
    n_col = 1;
    if (epi) {
      issue_epi(k0);
      n_epi = 1;
    }
  }

  // z columns over NS + 1 slots, two planes per loop trip: at the top of a trip starting at plane k,
  // zq[f][0 .. NS-2] hold planes k-R .. k+R-1; plane k pushes k+R into slot NS-1 and reads slots
  // 0 .. NS-1, plane k+1 pushes k+1+R into slot NS and reads 1 .. NS; the trip ends by a shift of two
  // (half the register moves of a shift per plane)
  double zq[NQ][NS + 1];
  {
    const int gi = gidx(ox, i0 + tx), gj = gidx(oy, j0 + ty);
    const bool col = inside && gi >= 0 && gj >= 0;
    const long long cp = gi + (long long)n1 * gj;
#pragma unroll
    for (int mm = 0; mm < NS - 1; ++mm) {
      const int gk = gidx(oz, k0 - R + mm);
#pragma unroll
      for (int f = 0; f < NQ; ++f) zq[f][mm] = 0.0;
      if (col && gk >= 0) {
        const long long pt = cp + (long long)n12 * gk;
#pragma unroll
        for (int f = 0; f < 5; ++f) zq[f][mm] = a.qs[pt + f * N];
        zq[5][mm] = a.q[pt + 4 * N] - a.p_ref;
        zq[6][mm] = a.q[pt + 3 * N] * (1.0 / a.q[pt]);
      }
    }
  }
  __syncthreads();                                  // barriers initialised before anyone waits

  // non-centre product cells: c < 2R*TY on the x rows, the rest on the y columns
  auto halo_product_cell = [&](int c, int &dst, int &cell, bool &isx) {
    if (c < 2 * R * TY) {
      const int row = c / (2 * R), col = c % (2 * R);
      const int lx = col < R ? col : col + TX;
      dst = row * PW + lx;
      cell = (row + R) * PW + lx;
      isx = true;
    } else {
      const int c2 = c - 2 * R * TY;
      const int row = c2 / TX, col = c2 % TX;
      const int ly = row < R ? row : row + TY;
      dst = ly * TX + col;
      cell = ly * PW + col + R;
      isx = false;
    }
  };

  int ok = 1;
  auto step = [&](auto offc, int k) {
    constexpr int OFF = decltype(offc)::value;
    const int idx = k - k0, st = idx & 1;
    if (tid == 0 && k + 1 < k1) {
      tc::fence_async_smem();                       // generic reads of that stage (step k-1) before TMA writes
      issue_tile(k + 1, st ^ 1);
      if (st) n_tile0++;
      else n_tile1++;
    }
    const long long kofs = (long long)n12 * k;
    ok = ok && tc::mbar_wait(&bar[st], (uint32_t)((idx >> 1) & 1), kTmaSpinLimit) &&
         tc::mbar_wait(&bar[2], (uint32_t)(idx & 1), kTmaSpinLimit);
    double *tqs = sm + L::o_tile + st * 2 * L::TILE, *tq = tqs + L::TILE;
    if (xmode == 1 || xmode == 2) {                 // side strip into the tile's wrapped columns
      const double *sd = sm + L::o_side + st * 2 * L::SIDEP;
      const int c0 = xmode == 1 ? 0 : TX + R;
      for (int e = tid; e < 2 * L::SIDE; e += TX * TY) {
        const int t = e / L::SIDE, r = e % L::SIDE;
        const int f = r / (TY * R), row = (r / R) % TY, col = r % R;
        (t ? tq : tqs)[f * PS + (row + R) * PW + c0 + col] = sd[t * L::SIDEP + r];
      }
    }
    if (patch_block && ok) {
#pragma unroll
      for (int c = 0; c < L::NPT; ++c) {
        if (pcell[c] < 0) continue;
        const long long pt = poff[c] + kofs;
#pragma unroll
        for (int f = 0; f < 5; ++f) {
          tqs[f * PS + pcell[c]] = a.qs[pt + f * N];
          tq[f * PS + pcell[c]] = a.q[pt + f * N];
        }
      }
    }
    if (xmode != 0 || patch_block) __syncthreads();
    // new column entry (plane k + R) and the shift
    {
      const double *cq = sm + L::o_col;
      double nv[NQ];
#pragma unroll
      for (int f = 0; f < 5; ++f) nv[f] = cq[f * TX * TY + tid];
      nv[5] = cq[L::COL + 4 * TX * TY + tid] - a.p_ref;
      nv[6] = cq[L::COL + 3 * TX * TY + tid] * (1.0 / cq[L::COL + tid]);
      const bool have = gidx(oz, k + R) >= 0;
#pragma unroll
      for (int f = 0; f < NQ; ++f) zq[f][NS - 1 + OFF] = have ? nv[f] : 0.0;
    }
    // centre values and the products u*qs5 / v*qs5: centre cells by their owner, the rest shared out
    const int cc = (ty + R) * PW + (tx + R);
    const double rho_c = tq[cc], p_c = tq[4 * PS + cc];
    const double ir = 1.0 / rho_c;                                 // ns_rho_rhou_p.f90:294
    const double u1 = tq[PS + cc] * ir, u2 = tq[2 * PS + cc] * ir;
    const double qs5 = tqs[4 * PS + cc];
    {
      double *px = sm + L::o_px, *py = sm + L::o_py;
      px[ty * PW + tx + R] = u1 * qs5;
      py[(ty + R) * TX + tx] = u2 * qs5;
      for (int c = tid; c < L::NHALO; c += TX * TY) {
        int dst, cell;
        bool isx;
        halo_product_cell(c, dst, cell, isx);
        const double vel = tq[(isx ? PS : 2 * PS) + cell] * (1.0 / tq[cell]);
        (isx ? px : py)[dst] = vel * tqs[4 * PS + cell];
      }
    }
    tc::fence_async_smem();                         // this thread's shared-memory accesses before the next TMA writes
    ok = __syncthreads_and(ok);
    if (!ok) return;
    if (tid == 0 && k + 1 < k1) {                   // every thread has taken its column entry
      tc::fence_async_smem();
      issue_col(k + 1);
      n_col++;
    }
    double kv[5];
    {
      const int i = i0 + tx, j = j0 + ty;
      const double *cqs = tqs + cc, *cqp = tq + 4 * PS + cc;
      const double gm1 = a.gamma - 1.0;
      const double u3 = zq[6][R + OFF];
      const double gpr = a.gamma * p_c / (rho_c * gm1);            // :293
      double r1 = 0.0, r2 = 0.0, r3 = 0.0, r4 = 0.0, r5 = 0.0;     // :296
      {
        const double s = ox.scale;
        const double A = D1<double, R, PER>(ox, cqs, 1, i) * s, B = D1<double, R, PER>(ox, cqs + PS, 1, i) * s,
                     Cc = D1<double, R, PER>(ox, cqs + 2 * PS, 1, i) * s,
                     D = D1<double, R, PER>(ox, cqs + 3 * PS, 1, i) * s,
                     E = D1<double, R, PER>(ox, cqs + 4 * PS, 1, i) * s;
        const double Sx = D1<double, R, PER>(ox, sm + L::o_px + ty * PW + tx + R, 1, i) * s;
        const double P = D1<double, R, PER>(ox, cqp, 1, i) * s;
        adj_dir(0, u1, u2, u3, gpr, ir, qs5, a.gamma, A, B, Cc, D, E, Sx, P, r1, r2, r3, r4, r5);
      }
      {
        const double s = oy.scale;
        const double A = D1<double, R, PER>(oy, cqs, PW, j) * s, B = D1<double, R, PER>(oy, cqs + PS, PW, j) * s,
                     Cc = D1<double, R, PER>(oy, cqs + 2 * PS, PW, j) * s,
                     D = D1<double, R, PER>(oy, cqs + 3 * PS, PW, j) * s,
                     E = D1<double, R, PER>(oy, cqs + 4 * PS, PW, j) * s;
        const double Sy = D1<double, R, PER>(oy, sm + L::o_py + (ty + R) * TX + tx, TX, j) * s;
        const double P = D1<double, R, PER>(oy, cqp, PW, j) * s;
        adj_dir(1, u1, u2, u3, gpr, ir, qs5, a.gamma, A, B, Cc, D, E, Sy, P, r1, r2, r3, r4, r5);
      }
      {
        const double s = oz.scale;
        const double Z0 = Dz1<double, R, PER>(oz, zq[0] + OFF, k) * s, Z1 = Dz1<double, R, PER>(oz, zq[1] + OFF, k) * s,
                     Z2 = Dz1<double, R, PER>(oz, zq[2] + OFF, k) * s, Z3 = Dz1<double, R, PER>(oz, zq[3] + OFF, k) * s,
                     Z4 = Dz1<double, R, PER>(oz, zq[4] + OFF, k) * s;
        const double Sz = Dz2<double, R, PER>(oz, zq[6] + OFF, zq[4] + OFF, k) * s;
        const double P = Dz1<double, R, PER>(oz, zq[5] + OFF, k) * s;
        adj_dir(2, u1, u2, u3, gpr, ir, qs5, a.gamma, Z0, Z1, Z2, Z3, Z4, Sz, P, r1, r2, r3, r4, r5);
      }
      kv[0] = r1; kv[1] = r2; kv[2] = r3; kv[3] = r4; kv[4] = r5;
    }
    const long long opt = (i0 + tx) + (long long)n1 * (j0 + ty) + kofs;
    if (a.src && inside) {                                         // :512
#pragma unroll
      for (int v = 0; v < 5; ++v) kv[v] = kv[v] + a.src[opt + v * N];
    }
    if (epi) ok = ok && tc::mbar_wait(&bar[3], (uint32_t)(idx & 1), kTmaSpinLimit);
    if (inside) {
      if (a.stage == 0) {
#pragma unroll
        for (int v = 0; v < 5; ++v) a.rhs[opt + v * N] = kv[v];
      } else {
        const double *eq0 = sm + L::o_epi + tid, *eacc = sm + L::o_epi + L::COL + tid;
        const double dt = a.dt, dth = a.dt * 0.5;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const long long o = opt + v * N;
          const double q0v = eq0[v * TX * TY];
          if (a.stage == 1) {
            a.acc[o] = kv[v];
            a.qnext[o] = q0v + dth * kv[v];
          } else if (a.stage == 2) {
            a.acc[o] = eacc[v * TX * TY] + 2.0 * kv[v];
            a.qnext[o] = q0v + dth * kv[v];
          } else if (a.stage == 3) {
            a.acc[o] = eacc[v * TX * TY] + 2.0 * kv[v];
            a.qnext[o] = q0v + dt * kv[v];
          } else {
            a.qnext[o] = q0v + dt / 6.0 * (eacc[v * TX * TY] + kv[v]);
          }
        }
      }
    }
    tc::fence_async_smem();
    ok = __syncthreads_and(ok);                     // every read of stage st and of the epilogue box done
    if (!ok) return;
    if (tid == 0 && epi && k + 1 < k1) {
      tc::fence_async_smem();
      issue_epi(k + 1);
      n_epi++;
    }
  };
  for (int k = k0; k < k1; k += 2) {
    step(std::integral_constant<int, 0>{}, k);
    if (!ok) break;
    if (k + 1 < k1) {
      step(std::integral_constant<int, 1>{}, k + 1);
      if (!ok) break;
    }
#pragma unroll
    for (int f = 0; f < NQ; ++f) {
#pragma unroll
      for (int mm = 0; mm < NS - 1; ++mm) zq[f][mm] = zq[f][mm + 2];
    }
  }
  if (!ok) {
    if (tid == 0) {
      atomicExch(err, 1);
      // the copies possibly still in flight: the latest phase of every barrier that was armed
      if (n_tile0 > 0) tc::mbar_wait(&bar[0], (uint32_t)((n_tile0 - 1) & 1), kTmaSpinLimit);
      if (n_tile1 > 0) tc::mbar_wait(&bar[1], (uint32_t)((n_tile1 - 1) & 1), kTmaSpinLimit);
      if (n_col > 0) tc::mbar_wait(&bar[2], (uint32_t)((n_col - 1) & 1), kTmaSpinLimit);
      if (n_epi > 0) tc::mbar_wait(&bar[3], (uint32_t)((n_epi - 1) & 1), kTmaSpinLimit);
    }
    __syncthreads();
  }
}

template <int R, bool PER>
bool launch_adj_tma(cruna_ctx *c, AdjArgs &a) {
  using L = AdjTmaLayout<R>;
  AdjTmaMaps m;
  const int n1 = c->g.n1, n2 = c->g.n2, n3 = c->g.n3;
  const long long N = c->g.N;
  const double *q0 = a.stage != 0 ? a.q0 : a.qs, *acc = a.stage >= 2 ? a.acc : a.qs;
  if (!tma_field_map(a.qs, n1, n2, n3, 5, N, L::PW, L::PH, 5, &m.qs_tile) ||
      !tma_field_map(a.q, n1, n2, n3, 5, N, L::PW, L::PH, 5, &m.q_tile) ||
      !tma_field_map(a.qs, n1, n2, n3, 5, N, TX, TY, 5, &m.qs_col) ||
      !tma_field_map(a.q, n1, n2, n3, 5, N, TX, TY, 5, &m.q_col) ||
      !tma_field_map(a.qs, n1, n2, n3, 5, N, R, TY, 5, &m.qs_side) ||
      !tma_field_map(a.q, n1, n2, n3, 5, N, R, TY, 5, &m.q_side) ||
      !tma_field_map(q0, n1, n2, n3, 5, N, TX, TY, 5, &m.q0_col) ||
      !tma_field_map(acc, n1, n2, n3, 5, N, TX, TY, 5, &m.acc_col))
    return false;
  static bool configured = false;
  if (!configured) {
    CRUNA_CUDA_CHECK(cudaFuncSetAttribute(k_adj_tma<R, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)L::bytes));
    configured = true;
  }
  const int bx = (n1 + TX - 1) / TX, by = (n2 + TY - 1) / TY;
  static const int res = resident_blocks(k_adj_tma<R, PER>, TX * TY, L::bytes);
  int nz = 1;
  a.kc = z_chunk_balanced(n3, bx * by, res, device_sms(), R, nz);
  ProfScope ps(c, "adj_pass");
  k_adj_tma<R, PER><<<dim3(bx, by, nz), dim3(TX, TY), L::bytes, c->stream>>>(a, m, c->flag + 1);
  CRUNA_LAUNCH_CHECK(c);
  return true;
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
  } else if (c->tma_fused && (Rl == 2 ? (per ? launch_adj_tma<2, true>(c, a) : launch_adj_tma<2, false>(c, a))
                                        : (per ? launch_adj_tma<4, true>(c, a) : launch_adj_tma<4, false>(c, a)))) {
    // TMA-fed pass launched
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
