// Fused explicit-stencil RHS of right_hand_side_direct_3d (src/equations/ns_rho_rhou_p.f90:31-253)
// for the explicit derivative cores (o2_e_c_o, o4_e_c_p, o4_e_c_o, o8_e_c_p, empty).
//
// Two z-marching kernels per RHS evaluation replace the reference's 42 transpose+line-core calls:
//   pass G reads q once and produces, per point, the six viscous stresses, the three heat fluxes
//   lambda*dT/dx_d, the friction work tau:grad(u), and the convective part of all five equations
//   (30 first derivatives);
//   pass D differentiates the stresses and heat fluxes (12 derivatives), assembles the five
//   equations in the reference's order, adds the forcing and, inside a time step, performs the RK4
//   stage update (rk_o4_e.f90:45-50) in its epilogue.
// A block owns a TX x TY column of the x-y plane and marches along z: the current plane (with R-wide
// x/y halos) lives in shared memory, and each thread keeps the 2R+1 z-neighbours of its own column
// in a private shared-memory ring, so every input value is read from HBM about once per pass.
//
// Precision: T = double is the plain FP64 path.  T = float is the FP32-stencil path: shared-memory
// fields, derivatives, fluxes and the pass-G outputs are FP32, the pressure and temperature are
// differenced as offsets p - p_ref and T - T_ref formed in FP64 (so the large mean does not eat the
// FP32 mantissa; d(p*u) is evaluated as p_ref*du + d((p-p_ref)*u)), and the assembled RHS, the RK4
// accumulation and the state stay FP64.
#include <cmath>
#include <stdexcept>
#include <string>

#include "cruna_internal.cuh"
#include "fused_common.cuh"

namespace cruna {

using namespace fz;

namespace {

// ------------------------------------------------------------------------------------------------
// pass G
// plane fields: 0 u, 1 v, 2 w, 3 T', 4 p', 5 rho*u, 6 rho*v ; ring fields: 0 u, 1 v, 2 w, 3 T', 4 p', 5 rho*w
// ------------------------------------------------------------------------------------------------
// Shared memory of the closure part of pass G: BF16 weights in the tcgen05 K-major layout, biases,
// the MMA mbarrier and the TMEM address; the activation tiles X [128][16] and H [128][64] reuse the
// plane when it is large enough (FP64), else follow this block.
struct ClSmem {
  __nv_bfloat16 W1[mlp::HID * 16];
  __nv_bfloat16 W2[mlp::HID * mlp::HID];
  __nv_bfloat16 W3[16 * mlp::HID];
  float b1[mlp::HID], b2[mlp::HID], b3[16];
  uint64_t mbar;
  uint32_t tmem;
};
constexpr size_t kClActBytes = (128 * 16 + 128 * mlp::HID) * sizeof(__nv_bfloat16);

template <typename T, int R>
constexpr size_t plane_bytes_g() { return sizeof(T) * 7 * (TX + 2 * R) * (TY + 2 * R); }
template <typename T, int R>
constexpr size_t ring_bytes_g() { return sizeof(T) * ring_slots(R) * 6 * TX * TY; }
template <typename T, int R>
constexpr size_t cl_offset_g() { return ((plane_bytes_g<T, R>() + ring_bytes_g<T, R>() + 1023) / 1024) * 1024; }
template <typename T, int R>
constexpr bool cl_alias_plane() { return plane_bytes_g<T, R>() >= kClActBytes; }

template <typename T, int R, bool PER, bool CL = false>
__global__ void __launch_bounds__(TX *TY, sizeof(T) == 4 ? 3 : 2) k_pass_g(const __grid_constant__ FusedArgs a) {
  constexpr int PW = TX + 2 * R, PH = TY + 2 * R, PS = PW * PH;
  constexpr int NS = ring_slots(R);
  constexpr int NRF = 6, RS = TX * TY;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  T *plane = reinterpret_cast<T *>(smem_raw);          // [7][PH][PW]
  T *ring = plane + 7 * PS;                            // [NS][NRF][TY*TX]
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int k0 = blockIdx.z * a.kc;
  const int k1 = min(k0 + a.kc, a.g.n3);
  const DirOpF &ox = a.op[0], &oy = a.op[1], &oz = a.op[2];
  const int n1 = a.g.n1, n12 = a.g.n1 * a.g.n2;
  const int gi = gidx(ox, i0 + tx), gj = gidx(oy, j0 + ty);
  const bool inside = (i0 + tx) < a.g.n1 && (j0 + ty) < a.g.n2;
  const bool col = gi >= 0 && gj >= 0;
  const int colpt = gi + n1 * gj;
  const long long N = a.g.N;
  const double *Q0 = a.q, *Q1 = a.q + N, *Q2 = a.q + 2 * N, *Q3 = a.q + 3 * N, *Q4 = a.q + 4 * N;
  HaloSet<R> hs;
  hs.init(ox, oy, i0, j0, tid, n1);
  // closure: weights staged once per block, TMEM for the three products (128 lanes x 128 columns)
  ClSmem *cs = nullptr;
  __nv_bfloat16 *clX = nullptr, *clH = nullptr;
  uint32_t cl_phase = 0;
  int cl_ok = 1;
  if constexpr (CL) {
    cs = reinterpret_cast<ClSmem *>(smem_raw + cl_offset_g<T, R>());
    unsigned char *act = cl_alias_plane<T, R>() ? smem_raw : smem_raw + cl_offset_g<T, R>() + ((sizeof(ClSmem) + 1023) / 1024) * 1024;
    clX = reinterpret_cast<__nv_bfloat16 *>(act);
    clH = clX + 128 * 16;
    mlp::stage_weights(a.cl_P, cs->W1, cs->W2, cs->W3, nullptr, nullptr);
    if (tid < mlp::HID) {
      cs->b1[tid] = a.cl_P[mlp::OB1 + tid];
      cs->b2[tid] = a.cl_P[mlp::OB2 + tid];
    }
    if (tid < 16) cs->b3[tid] = tid < mlp::OUT ? a.cl_P[mlp::OB3 + tid] : 0.0f;
    if (tid == 0) tc::mbar_init(&cs->mbar, 1);
    if (ty == 0) tc::tmem_alloc(&cs->tmem, 128);
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
  }

  auto put_ring = [&](int kk, double r, double ru, double rv, double rw, double p) {
    const int sl = ((kk % NS) + NS) % NS;
    T *rp = ring + sl * NRF * RS + tid;
    const double ir = 1.0 / r;
    rp[0 * RS] = T(ru * ir);
    rp[1 * RS] = T(rv * ir);
    rp[2 * RS] = T(rw * ir);
    rp[3 * RS] = T(a.WoR * p * ir - a.T_ref);
    rp[4 * RS] = T(p - a.p_ref);
    rp[5 * RS] = T(rw);
  };
  for (int kk = k0 - R; kk < k0 + R; ++kk) {
    const int gk = gidx(oz, kk);
    if (gk < 0 || !col) continue;
    const long long pt = colpt + (long long)n12 * gk;
    put_ring(kk, Q0[pt], Q1[pt], Q2[pt], Q3[pt], Q4[pt]);
  }
  double pf[5] = {1, 0, 0, 0, 0};
  double pruv[2] = {0, 0};
  int pf_ok = 0;
  auto prefetch = [&](int kk, int kc) {
    const int gk = gidx(oz, kk);
    pf_ok = (gk >= 0 && col);
    if (pf_ok) {
      const long long pt = colpt + (long long)n12 * gk;
      pf[0] = Q0[pt]; pf[1] = Q1[pt]; pf[2] = Q2[pt]; pf[3] = Q3[pt]; pf[4] = Q4[pt];
    }
    if (col && kc < k1) {
      const long long pt = colpt + (long long)n12 * kc;
      pruv[0] = Q1[pt];
      pruv[1] = Q2[pt];
    }
  };
  prefetch(k0 + R, k0);
  // raw state of this thread's halo cells, loaded one plane ahead
  constexpr int NHT = HaloSet<R>::PER_THREAD;
  double hv[NHT][5];
  auto halo_fetch = [&](int kk) {
    const long long kofs = (long long)n12 * kk;
#pragma unroll
    for (int h = 0; h < NHT; ++h) {
      if (hs.goff[h] < 0) continue;
      const long long pt = hs.goff[h] + kofs;
      hv[h][0] = Q0[pt]; hv[h][1] = Q1[pt]; hv[h][2] = Q2[pt]; hv[h][3] = Q3[pt]; hv[h][4] = Q4[pt];
    }
  };
  halo_fetch(k0);

  for (int k = k0; k < k1; ++k) {
    T outv[CL ? NG : 1];                               // closure: pass-G outputs held across the network
    float feat[CL ? mlp::IN : 1];
    if (pf_ok) put_ring(k + R, pf[0], pf[1], pf[2], pf[3], pf[4]);
    const int slot = k % NS;
    {
      T *c = plane + (ty + R) * PW + (tx + R);
      const T *rp = ring + slot * NRF * RS + tid;
#pragma unroll
      for (int f = 0; f < 5; ++f) c[f * PS] = rp[f * RS];
      c[5 * PS] = T(pruv[0]);
      c[6 * PS] = T(pruv[1]);
    }
    const long long kofs = (long long)n12 * k;
#pragma unroll
    for (int h = 0; h < NHT; ++h) {
      if (hs.goff[h] < 0) continue;
      const double r = hv[h][0], ru = hv[h][1], rv = hv[h][2], rw = hv[h][3], p = hv[h][4];
      const double ir = 1.0 / r;
      T *c = plane + hs.cell[h];
      c[0 * PS] = T(ru * ir); c[1 * PS] = T(rv * ir); c[2 * PS] = T(rw * ir);
      c[3 * PS] = T(a.WoR * p * ir - a.T_ref);
      c[4 * PS] = T(p - a.p_ref); c[5 * PS] = T(ru); c[6 * PS] = T(rv);
    }
    prefetch(k + R + 1, k + 1);
    if (k + 1 < k1) halo_fetch(k + 1);
    __syncthreads();
    if (inside) {
      const int i = i0 + tx, j = j0 + ty;
      const T *c = plane + (ty + R) * PW + (tx + R);
      const T *U = c, *V = c + PS, *W = c + 2 * PS, *TT = c + 3 * PS, *P = c + 4 * PS, *RU = c + 5 * PS,
              *RV = c + 6 * PS;
      int so[NS];
#pragma unroll
      for (int m = -R; m <= R; ++m) so[m + R] = ((slot + m + NS) % NS) * NRF * RS + tid;
      auto column = [&](int f, T *v) {
#pragma unroll
        for (int m = 0; m < NS; ++m) v[m] = ring[so[m] + f * RS];
      };
      const T sx = T(ox.scale), sy = T(oy.scale), sz = T(oz.scale);
      // z derivatives one column at a time (rho*w and w stay for the products)
      T zrw[NS], zw[NS], zt[NS];
      column(5, zrw);
      column(2, zw);
      const T m3 = Dz1<T, R, PER>(oz, zrw, k) * sz;
      const T wz = Dz1<T, R, PER>(oz, zw, k) * sz;
      const T a3z = Dz2<T, R, PER>(oz, zrw, zw, k) * sz;
      column(0, zt);
      const T uz = Dz1<T, R, PER>(oz, zt, k) * sz;
      const T a1z = Dz2<T, R, PER>(oz, zrw, zt, k) * sz;
      const T uc = zt[R];
      column(1, zt);
      const T vz = Dz1<T, R, PER>(oz, zt, k) * sz;
      const T a2z = Dz2<T, R, PER>(oz, zrw, zt, k) * sz;
      const T vc = zt[R];
      column(3, zt);
      const T tgz = Dz1<T, R, PER>(oz, zt, k) * T(oz.scale_h);
      const T Tc = zt[R];
      column(4, zt);
      const T pz = Dz1<T, R, PER>(oz, zt, k) * sz;
      const T ezp = Dz2<T, R, PER>(oz, zt, zw, k) * sz;
      const T wc = zw[R];
      // velocity gradients (ns_rho_rhou_p.f90:102-112) and temperature gradient (:189-191)
      const T ux = D1<T, R, PER>(ox, U, 1, i) * sx, uy = D1<T, R, PER>(oy, U, PW, j) * sy;
      const T vx = D1<T, R, PER>(ox, V, 1, i) * sx, vy = D1<T, R, PER>(oy, V, PW, j) * sy;
      const T wx = D1<T, R, PER>(ox, W, 1, i) * sx, wy = D1<T, R, PER>(oy, W, PW, j) * sy;
      const T tgx = D1<T, R, PER>(ox, TT, 1, i) * T(ox.scale_h);
      const T tgy = D1<T, R, PER>(oy, TT, PW, j) * T(oy.scale_h);
      // viscosity mu0 (T/T0)^1.5 (T0+S1)/(T+S1) and stresses (:115-128); x^1.5 as x*sqrt(x)
      const double Tabs = double(Tc) + a.T_ref;
      const double tr = Tabs / a.T0;
      const T mu = T(a.mu0 * (tr * sqrt(tr)) * ((a.T0 + 110.4) / (Tabs + 110.4)));
      const T mu_div = -(T(2.0 / 3.0) * mu * (ux + vy + wz));
      const T t11 = mu_div + T(2) * mu * ux;
      const T t22 = mu_div + T(2) * mu * vy;
      const T t33 = mu_div + T(2) * mu * wz;
      const T t12 = mu * (uy + vx);
      const T t13 = mu * (uz + wx);
      const T t23 = mu * (vz + wy);
      const T lam = mu * T(a.cp_over_pr);
      const T phi = t11 * ux + t12 * uy + t13 * uz + t12 * vx + t22 * vy + t23 * vz + t13 * wx + t23 * wy +
                    t33 * wz;                                     // :204-206
      // convective terms (:131-186)
      const T m1 = D1<T, R, PER>(ox, RU, 1, i) * sx, m2 = D1<T, R, PER>(oy, RV, PW, j) * sy;
      const T px = D1<T, R, PER>(ox, P, 1, i) * sx, py = D1<T, R, PER>(oy, P, PW, j) * sy;
      const T a1x = D2<T, R, PER>(ox, RU, U, 1, i) * sx, a1y = D2<T, R, PER>(oy, RV, U, PW, j) * sy;
      const T a2x = D2<T, R, PER>(ox, RU, V, 1, i) * sx, a2y = D2<T, R, PER>(oy, RV, V, PW, j) * sy;
      const T a3x = D2<T, R, PER>(ox, RU, W, 1, i) * sx, a3y = D2<T, R, PER>(oy, RV, W, PW, j) * sy;
      const T pref = T(a.p_ref);
      const T ex = pref * ux + D2<T, R, PER>(ox, P, U, 1, i) * sx;
      const T ey = pref * vy + D2<T, R, PER>(oy, P, V, PW, j) * sy;
      const T ez = pref * wz + ezp;
      const double gt = a.gamma / (a.gamma - 1.0);
      const T c1 = -m1 - m2 - m3;
      const T c2 = -a1x - a1y - a1z - px;
      const T c3 = -a2x - a2y - a2z - py;
      const T c4 = -a3x - a3y - a3z - pz;
      T c5 = T(gt) * (-ex - ey - ez);
      c5 = c5 + uc * px + vc * py + wc * pz;
      const T o[NG] = {c1, c2, c3, c4, c5, t11, t12, t13, t22, t23, t33, lam * tgx, lam * tgy, lam * tgz, phi};
      if constexpr (CL) {
#pragma unroll
        for (int f = 0; f < NG; ++f) outv[f] = o[f];
        // features of the closure (the unfused path's order): grad u, rho, T, filter width; or the
        // scale-free form grad u / g, rho, T, g delta with g = |grad u|
        const double gr[9] = {double(ux), double(uy), double(uz), double(vx), double(vy), double(vz),
                              double(wx), double(wy), double(wz)};
        double g2 = 0.0;
#pragma unroll
        for (int f = 0; f < 9; ++f) g2 += gr[f] * gr[f];
        const double gm = sqrt(g2), ginv = gm > 0.0 ? 1.0 / gm : 0.0;
#pragma unroll
        for (int f = 0; f < 9; ++f) feat[f] = (float)(a.cl_norm ? gr[f] * ginv : gr[f]);
        feat[9] = (float)a.q[i + (long long)n1 * j + kofs];
        feat[10] = (float)Tabs;
        feat[11] = (float)(a.cl_norm ? gm * a.cl_delta : a.cl_delta);
      } else {
        T *go = static_cast<T *>(a.gbuf);
        const long long pt = i + (long long)n1 * j + kofs;
#pragma unroll
        for (int f = 0; f < NG; ++f) go[pt + f * N] = o[f];
      }
    }
    if constexpr (CL) {
      // the network on the block's 128 points: thread = point = TMEM lane (tcgen05, BF16 operands)
      __syncthreads();                             // every plane read done: X / H may reuse the plane
      float v[16];
#pragma unroll
      for (int f = 0; f < 16; ++f) v[f] = 0.0f;
      if (inside) {
#pragma unroll
        for (int f = 0; f < mlp::IN; ++f) v[f] = (feat[f] - a.cl_sc.in_mean[f]) * a.cl_sc.in_inv[f];
      }
      mlp::put8(clX, tid, 0, 16, v);
      mlp::put8(clX, tid, 8, 16, v + 8);
      const uint32_t tb = cs->tmem, lane = (uint32_t)(ty * 32) << 16;
      auto mma = [&](uint32_t col, const __nv_bfloat16 *A, const __nv_bfloat16 *B, int K, int Nn) {
        tc::fence_before();
        tc::fence_async_smem();
        __syncthreads();
        if (tid == 0) {
          tc::fence_after();
          tc::gemm_bf16(tb + col, tc::smem_addr(A), tc::smem_addr(B), K, Nn, false);
          tc::commit(&cs->mbar);
        }
        cl_ok = __syncthreads_and(cl_ok && tc::mbar_wait(&cs->mbar, cl_phase, mlp::kWaitLimit));
        cl_phase ^= 1;
        tc::fence_after();
      };
      mma(0, clX, cs->W1, 16, 64);
      for (int c = 0; c < 4 && cl_ok; ++c) {
        tc::tmem_ld16(tb + lane + c * 16, v);
#pragma unroll
        for (int e = 0; e < 16; ++e) v[e] = mlp::gelu(v[e] + cs->b1[c * 16 + e]);
        mlp::put8(clH, tid, c * 16, 64, v);
        mlp::put8(clH, tid, c * 16 + 8, 64, v + 8);
      }
      if (cl_ok) mma(64, clH, cs->W2, 64, 64);
      if (cl_ok) {
        // H1 has been consumed by the finished product: H2 takes its place
        for (int c = 0; c < 4; ++c) {
          tc::tmem_ld16(tb + lane + 64 + c * 16, v);
#pragma unroll
          for (int e = 0; e < 16; ++e) v[e] = mlp::gelu(v[e] + cs->b2[c * 16 + e]);
          mlp::put8(clH, tid, c * 16, 64, v);
          mlp::put8(clH, tid, c * 16 + 8, 64, v + 8);
        }
        mma(0, clH, cs->W3, 64, 16);
      }
      if (cl_ok) tc::tmem_ld16(tb + lane + 0, v);
      if (inside && cl_ok) {
        // model stresses (order 11, 22, 33, 12, 13, 23) in the momentum fluxes: tau_ij - tau_ij(model)
        const double gd = (double)feat[11];
        const double scl = a.cl_norm ? (double)feat[9] * gd * gd : 1.0;
        double tm[mlp::OUT];
#pragma unroll
        for (int o2 = 0; o2 < mlp::OUT; ++o2) tm[o2] = (double)((v[o2] + cs->b3[o2]) * a.cl_sc.out_scale[o2]) * scl;
        outv[5] = T(double(outv[5]) - tm[0]);    // t11
        outv[6] = T(double(outv[6]) - tm[3]);    // t12
        outv[7] = T(double(outv[7]) - tm[4]);    // t13
        outv[8] = T(double(outv[8]) - tm[1]);    // t22
        outv[9] = T(double(outv[9]) - tm[5]);    // t23
        outv[10] = T(double(outv[10]) - tm[2]);  // t33
        T *go = static_cast<T *>(a.gbuf);
        const long long pt = (i0 + tx) + (long long)n1 * (j0 + ty) + kofs;
#pragma unroll
        for (int f = 0; f < NG; ++f) go[pt + f * N] = outv[f];
      }
      if (!cl_ok) break;
    }
    __syncthreads();
  }
  if constexpr (CL) {
    if (!cl_ok) {
      if (tid == 0) atomicExch(a.cl_err, 1);
      tc::mbar_wait(&cs->mbar, cl_phase, mlp::kWaitLimit);   // a product still in flight ends first
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (ty == 0) tc::tmem_free(cs->tmem, 128);
  }
}

// ------------------------------------------------------------------------------------------------
// pass D
// plane fields: 0 t11, 1 t12, 2 t13, 3 t22, 4 t23, 5 hx, 6 hy ; ring fields: 0 t13, 1 t23, 2 t33, 3 hz
// ------------------------------------------------------------------------------------------------
template <typename T, int R, bool PER>
__global__ void __launch_bounds__(TX *TY, 3) k_pass_d(const __grid_constant__ FusedArgs a) {
  constexpr int PW = TX + 2 * R, PH = TY + 2 * R, PS = PW * PH;
  constexpr int NS = ring_slots(R);
  constexpr int NRF = 4, RS = TX * TY;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  T *plane = reinterpret_cast<T *>(smem_raw);          // [7][PH][PW]
  T *ring = plane + 7 * PS;                            // [NS][NRF][TY*TX]
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
  const T *G = static_cast<const T *>(a.gbuf);
  constexpr int pfld[7] = {5, 6, 7, 8, 9, 11, 12};   // G fields of the plane
  constexpr int rfld[4] = {7, 9, 10, 13};            // G fields of the ring
  HaloSet<R> hs;
  hs.init(ox, oy, i0, j0, tid, n1);

  for (int kk = k0 - R; kk < k0 + R; ++kk) {
    const int gk = gidx(oz, kk);
    if (gk < 0 || !col) continue;
    const long long pt = colpt + (long long)n12 * gk;
    T *rp = ring + (((kk % NS) + NS) % NS) * NRF * RS + tid;
#pragma unroll
    for (int f = 0; f < NRF; ++f) rp[f * RS] = G[pt + rfld[f] * N];
  }
  T pf[NRF];
  T pc[7];
  int pf_ok = 0;
  auto prefetch = [&](int kk, int kc) {
    const int gk = gidx(oz, kk);
    pf_ok = (gk >= 0 && col);
    if (pf_ok) {
      const long long pt = colpt + (long long)n12 * gk;
#pragma unroll
      for (int f = 0; f < NRF; ++f) pf[f] = G[pt + rfld[f] * N];
    }
    if (col && kc < k1) {
      const long long pt = colpt + (long long)n12 * kc;
#pragma unroll
      for (int f = 0; f < 7; ++f) pc[f] = G[pt + pfld[f] * N];
    }
  };
  prefetch(k0 + R, k0);
  constexpr int NHT = HaloSet<R>::PER_THREAD;
  T hv[NHT][7];
  auto halo_fetch = [&](int kk) {
    const long long kofs = (long long)n12 * kk;
#pragma unroll
    for (int h = 0; h < NHT; ++h) {
      if (hs.goff[h] < 0) continue;
      const long long pt = hs.goff[h] + kofs;
#pragma unroll
      for (int f = 0; f < 7; ++f) hv[h][f] = G[pt + pfld[f] * N];
    }
  };
  halo_fetch(k0);
  for (int k = k0; k < k1; ++k) {
    if (pf_ok) {
      T *rp = ring + (((k + R) % NS + NS) % NS) * NRF * RS + tid;
#pragma unroll
      for (int f = 0; f < NRF; ++f) rp[f * RS] = pf[f];
    }
    const int slot = k % NS;
    {
      T *c = plane + (ty + R) * PW + (tx + R);
#pragma unroll
      for (int f = 0; f < 7; ++f) c[f * PS] = pc[f];
    }
    const long long kofs = (long long)n12 * k;
    // epilogue inputs of this plane, issued before the barrier so their latency overlaps the stencils
    const long long opt = (i0 + tx) + (long long)n1 * (j0 + ty) + kofs;
    T e_g[6];
    double e_f[5] = {0, 0, 0, 0, 0}, e_q0[5] = {0, 0, 0, 0, 0}, e_acc[5] = {0, 0, 0, 0, 0};
    if (inside) {
#pragma unroll
      for (int f = 0; f < 5; ++f) e_g[f] = G[opt + f * N];
      e_g[5] = G[opt + 14 * N];
      if (a.force) {
#pragma unroll
        for (int v = 0; v < 5; ++v) e_f[v] = a.force[opt + v * N];
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
#pragma unroll
      for (int f = 0; f < 7; ++f) c[f * PS] = hv[h][f];
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
      T zc[NS];
      const T sx = T(ox.scale), sy = T(oy.scale), sz = T(oz.scale);
#pragma unroll
      for (int m = 0; m < NS; ++m) zc[m] = ring[so[m] + 0 * RS];
      const T v1z = Dz1<T, R, PER>(oz, zc, k) * sz;               // d_z tau_13
#pragma unroll
      for (int m = 0; m < NS; ++m) zc[m] = ring[so[m] + 1 * RS];
      const T v2z = Dz1<T, R, PER>(oz, zc, k) * sz;               // d_z tau_23
#pragma unroll
      for (int m = 0; m < NS; ++m) zc[m] = ring[so[m] + 2 * RS];
      const T v3z = Dz1<T, R, PER>(oz, zc, k) * sz;               // d_z tau_33
#pragma unroll
      for (int m = 0; m < NS; ++m) zc[m] = ring[so[m] + 3 * RS];
      const T qz = Dz1<T, R, PER>(oz, zc, k) * T(oz.scale_h);     // d_z (lambda d_z T)
      const T v1x = D1<T, R, PER>(ox, c + 0 * PS, 1, i) * sx;     // d_x tau_11
      const T v1y = D1<T, R, PER>(oy, c + 1 * PS, PW, j) * sy;    // d_y tau_12
      const T v2x = D1<T, R, PER>(ox, c + 1 * PS, 1, i) * sx;     // d_x tau_21
      const T v2y = D1<T, R, PER>(oy, c + 3 * PS, PW, j) * sy;    // d_y tau_22
      const T v3x = D1<T, R, PER>(ox, c + 2 * PS, 1, i) * sx;     // d_x tau_31
      const T v3y = D1<T, R, PER>(oy, c + 4 * PS, PW, j) * sy;    // d_y tau_32
      const T qx = D1<T, R, PER>(ox, c + 5 * PS, 1, i) * T(ox.scale_h);
      const T qy = D1<T, R, PER>(oy, c + 6 * PS, PW, j) * T(oy.scale_h);
      const long long pt = opt;
      (void)i; (void)j;
      // assembly in the reference's order (:135, 143-149, 157-163, 171-177, 185-209)
      double r1 = double(e_g[0]);
      double r2 = double(e_g[1]);
      r2 = r2 + double(v1x); r2 = r2 + double(v1y); r2 = r2 + double(v1z);
      double r3 = double(e_g[2]);
      r3 = r3 + double(v2x); r3 = r3 + double(v2y); r3 = r3 + double(v2z);
      double r4 = double(e_g[3]);
      r4 = r4 + double(v3x); r4 = r4 + double(v3y); r4 = r4 + double(v3z);
      double r5 = double(e_g[4]);
      r5 = r5 + double(qx); r5 = r5 + double(qy); r5 = r5 + double(qz);
      r5 = r5 + double(e_g[5]);
      r5 = (a.gamma - 1.0) * r5;
      if (a.force) {                                              // :212
        r1 = r1 + e_f[0]; r2 = r2 + e_f[1]; r3 = r3 + e_f[2]; r4 = r4 + e_f[3]; r5 = r5 + e_f[4];
      }
      const double kv[5] = {r1, r2, r3, r4, r5};
      if (a.stage == 0) {
#pragma unroll
        for (int v = 0; v < 5; ++v) a.rhs[pt + v * N] = kv[v];
      } else {
        // RK4 stage update (rk_o4_e.f90:45-50)
        const double dt = a.dt, dth = a.dt * 0.5;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const long long o = pt + v * N;
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
size_t smem_g() {
  return sizeof(T) * (7 * (TX + 2 * R) * (TY + 2 * R) + ring_slots(R) * 6 * TX * TY);
}
template <typename T, int R>
size_t smem_g_cl() {
  return cl_offset_g<T, R>() + ((sizeof(ClSmem) + 1023) / 1024) * 1024 + (cl_alias_plane<T, R>() ? 0 : kClActBytes);
}
template <typename T, int R>
size_t smem_d() {
  return sizeof(T) * (7 * (TX + 2 * R) * (TY + 2 * R) + ring_slots(R) * 4 * TX * TY);
}

template <typename T, int R, bool PER>
void launch_passes(cruna_ctx *c, FusedArgs &a) {
  static bool configured = false;
  if (!configured) {
    CRUNA_CUDA_CHECK(cudaFuncSetAttribute(k_pass_g<T, R, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem_g<T, R>()));
    CRUNA_CUDA_CHECK(cudaFuncSetAttribute(k_pass_d<T, R, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem_d<T, R>()));
    configured = true;
  }
  const int bx = (c->g.n1 + TX - 1) / TX, by = (c->g.n2 + TY - 1) / TY;
  static const int res_g = resident_blocks(k_pass_g<T, R, PER>, TX * TY, smem_g<T, R>());
  static const int res_d = resident_blocks(k_pass_d<T, R, PER>, TX * TY, smem_d<T, R>());
  const int sms = device_sms();
  int nz = 1;
  if (a.cl_P) {                                    // pass G with the closure network in place
    static bool cl_configured = false;
    if (!cl_configured) {
      CRUNA_CUDA_CHECK(cudaFuncSetAttribute(k_pass_g<T, R, PER, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem_g_cl<T, R>()));
      cl_configured = true;
    }
    static const int res_cl = resident_blocks(k_pass_g<T, R, PER, true>, TX * TY, smem_g_cl<T, R>());
    a.kc = z_chunk_balanced(c->g.n3, bx * by, res_cl, sms, R, nz);
    ProfScope ps(c, "pass_g_closure");
    k_pass_g<T, R, PER, true><<<dim3(bx, by, nz), dim3(TX, TY), smem_g_cl<T, R>(), c->stream>>>(a);
    CRUNA_LAUNCH_CHECK(c);
  } else {
    a.kc = z_chunk_balanced(c->g.n3, bx * by, res_g, sms, R, nz);
    ProfScope ps(c, "pass_g");
    k_pass_g<T, R, PER><<<dim3(bx, by, nz), dim3(TX, TY), smem_g<T, R>(), c->stream>>>(a);
    CRUNA_LAUNCH_CHECK(c);
  }
  {
    a.kc = z_chunk_balanced(c->g.n3, bx * by, res_d, sms, R, nz);
    ProfScope ps(c, "pass_d");
    k_pass_d<T, R, PER><<<dim3(bx, by, nz), dim3(TX, TY), smem_d<T, R>(), c->stream>>>(a);
    CRUNA_LAUNCH_CHECK(c);
  }
}

template <typename T>
void launch_for(cruna_ctx *c, FusedArgs &a, int R, bool per) {
  if (R <= 2) {
    if (per) launch_passes<T, 2, true>(c, a);
    else launch_passes<T, 2, false>(c, a);
  } else {
    if (per) launch_passes<T, 4, true>(c, a);
    else launch_passes<T, 4, false>(c, a);
  }
}

}  // namespace

namespace fz {
DirOpF to_dir(const LineOp &op, double dx, bool heat_dx) {
  DirOpF d;
  d.n = op.n;
  d.kind = op.kind == OP_ZERO ? 0 : 1;
  d.periodic = op.periodic;
  d.r = op.r;
  for (int m = 0; m <= op.r && m < 5; ++m) d.c[m] = op.c[m];
  d.nb = op.nb;
  d.bw = op.bw;
  for (int r = 0; r < 2; ++r)
    for (int m = 0; m < 5; ++m) d.brow[r][m] = op.brow[r][m];
  d.scale = 1.0 / (dx * op.div);
  d.scale_h = heat_dx ? d.scale : 1.0 / (1.0 * op.div);
  return d;
}

int halo_of(const LineOp &op) {
  if (op.kind == OP_ZERO) return 0;
  return op.periodic ? op.r : std::max(op.r, op.bw - 1);
}

}  // namespace fz

// the closure network runs inside pass G (fused RHS path, closure attached and not switched off)
bool closure_in_pass(const cruna_ctx *c) { return c->closure_mlp && c->closure_fused && use_fused(c); }

bool fused_supported(const cruna_ctx *c) {
  for (int d = 0; d < 3; ++d) {
    const LineOp &op = c->dop[d];
    if (op.kind == OP_STENCIL && op.solve) return false;           // compact cores: generic path
    if (op.kind == OP_STENCIL && (op.r > 4 || op.nb > 2 || op.bw > 5)) return false;
  }
  int R = 0;
  for (int d = 0; d < 3; ++d) R = std::max(R, halo_of(c->dop[d]));
  if (R > 4) return false;
  if (c->has_nonlocal_bc) return false;                            // 200 / 204: generic path
  return true;
}

void rhs_direct_fused(cruna_ctx *c, const double *q_in, double *rhs, int stage, const double *q0, double *acc,
                      double *qnext, double dt) {
  const bool fp32 = c->cfg.precision == CRUNA_FP32_STENCIL;
  const long long N = c->g.N;
  if (!c->fz) {
    void *p = nullptr;
    CRUNA_CUDA_CHECK(cudaMalloc(&p, (size_t)NG * N * (fp32 ? sizeof(float) : sizeof(double))));
    c->allocations.push_back(p);
    c->fz = static_cast<double *>(p);
  }
  const double *q = q_in;
  if (c->has_q_bc) {                                               // ns_rho_rhou_p.f90:89-92
    copy_state(c, c->st[4], q_in, 5);
    bc_q(c, c->st[4], 0);
    q = c->st[4];
  }
  if (fp32 && !c->refs_set) {
    // offsets for the FP32 differencing: the pressure and temperature of the first point of the first
    // state this path sees (deterministic; any value near the mean keeps p - p_ref small)
    double h[2] = {0.0, 1.0};
    CRUNA_CUDA_CHECK(cudaMemcpyAsync(&h[0], q + 4 * N, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CRUNA_CUDA_CHECK(cudaMemcpyAsync(&h[1], q, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    c->p_ref = h[0];
    c->T_ref = c->cfg.W / c->cfg.R * h[0] / h[1];
    c->refs_set = true;
  }
  FusedArgs a;
  a.g = c->g;
  for (int d = 0; d < 3; ++d) a.op[d] = to_dir(c->dop[d], c->dx[d], c->cfg.heat_flux_dx != 0);
  a.WoR = c->cfg.W / c->cfg.R;
  a.mu0 = c->cfg.mu0;
  a.T0 = c->cfg.T0;
  a.gamma = c->cfg.gamma;
  a.cp_over_pr = c->cfg.gamma * (c->cfg.R / c->cfg.W) / (c->cfg.gamma - 1.0) / c->cfg.Pr;
  a.p_ref = fp32 ? c->p_ref : 0.0;
  a.T_ref = fp32 ? c->T_ref : 0.0;
  a.q = q;
  a.gbuf = c->fz;
  a.force = c->force;
  if (closure_in_pass(c)) {                        // the closure's stresses enter through pass G
    int *flag = nullptr;
    mlp_device_view(c->closure_mlp, &a.cl_P, &a.cl_sc, &flag);
    a.cl_err = flag;
    a.cl_delta = c->closure_delta;
    a.cl_norm = c->closure_norm ? 1 : 0;
    a.force = c->user_force;
  }
  a.dt = dt;
  a.q0 = q0;
  a.acc = acc;
  a.qnext = qnext;
  // rhs boundary conditions act on the finished rhs: then the RK update runs after them
  const bool split = stage != 0 && c->has_rhs_bc;
  a.stage = split ? 0 : stage;
  a.rhs = (stage == 0 || split) ? rhs : nullptr;
  int R = 0;
  for (int d = 0; d < 3; ++d) R = std::max(R, halo_of(c->dop[d]));
  const int Rl = R <= 2 ? 2 : 4;
  bool per = true;
  for (int d = 0; d < 3; ++d) per = per && c->dop[d].kind == OP_STENCIL && c->dop[d].periodic && c->dop[d].r == Rl;
  if (fp32) launch_for<float>(c, a, R, per);
  else launch_for<double>(c, a, R, per);
  if (stage == 0 || split) {
    if (c->has_rhs_bc) bc_rhs(c, rhs, q);                          // :218
    if (split) rk_stage(c, stage, dt, rhs, q0, acc, qnext);
  }
}

}  // namespace cruna

// ------------------------------------------------------------------------------------------------
// Allocation-free variant of the fused direct RHS.
//
// Some callers cannot allocate device memory at the point where they need an RHS evaluation: a
// host code whose device memory is owned by another allocator (a framework's caching pool, a
// Fortran code that sizes every array once at start-up and forbids allocation in its time loop), or
// an embedded solver that must run with a fixed, pre-planned footprint.  cruna_init allocates the
// context's buffers and therefore does not serve them.  cruna_rhs_direct_noalloc evaluates the same
// two fused passes with no context: the 15-field intermediate of pass G lives in the file-scope
// device array below (kNoAllocMaxPoints points, 15.7 MB, held by every GPU that loads the library
// until the process exits), and the caller passes the input state and the output RHS.
// ------------------------------------------------------------------------------------------------
namespace cruna {
namespace {

constexpr long long kNoAllocMaxPoints = 131072;          // e.g. 64 x 64 x 32 grid points
static __device__ __align__(256) double g_noalloc_scratch[NG * kNoAllocMaxPoints];

void noalloc_msg(char *buf, int len, const char *msg) {
  if (!buf || len <= 0) return;
  int i = 0;
  for (; msg[i] && i < len - 1; ++i) buf[i] = msg[i];
  buf[i] = 0;
}

// Sets the shared-memory limit of the two passes and launches them.  Called on every call: the
// attribute belongs to the current context, which a host may have replaced since the last call.
template <int R, bool PER>
cudaError_t noalloc_launch(const FusedArgs &a, dim3 grid, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(k_pass_g<double, R, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem_g<double, R>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_pass_d<double, R, PER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_d<double, R>());
  if (e != cudaSuccess) return e;
  k_pass_g<double, R, PER><<<grid, dim3(TX, TY), smem_g<double, R>(), s>>>(a);
  k_pass_d<double, R, PER><<<grid, dim3(TX, TY), smem_d<double, R>(), s>>>(a);
  return cudaGetLastError();
}

}  // namespace
}  // namespace cruna

extern "C" int cruna_rhs_direct_noalloc(const cruna_config *cfg, const double *q, double *rhs, void *stream,
                                        char *errbuf, int errlen) {
  using namespace cruna;
  using namespace cruna::fz;
  if (!cfg || !q || !rhs) {
    noalloc_msg(errbuf, errlen, "null argument");
    return CRUNA_ERR_ARG;
  }
  if (cfg->abi_version != CRUNA_ABI_VERSION) {
    noalloc_msg(errbuf, errlen, "cruna_config.abi_version mismatch");
    return CRUNA_ERR_ARG;
  }
  for (int d = 0; d < 3; ++d)
    if (cfg->n[d] < 1) {
      noalloc_msg(errbuf, errlen, "geom.n must be >= 1");
      return CRUNA_ERR_ARG;
    }
  const long long npts = (long long)cfg->n[0] * cfg->n[1] * cfg->n[2];
  if (npts > kNoAllocMaxPoints) {
    noalloc_msg(errbuf, errlen,
                "grid too large for cruna_rhs_direct_noalloc: at most 131072 points (its static scratch)");
    return CRUNA_ERR_ARG;
  }
  if (cfg->precision != CRUNA_FP64) {
    noalloc_msg(errbuf, errlen, "cruna_rhs_direct_noalloc computes in FP64 only");
    return CRUNA_ERR_UNSUPPORTED;
  }
  if (!(cfg->gamma > 1.0) || !(cfg->R > 0.0) || !(cfg->W > 0.0) || !(cfg->T0 > 0.0) || !(cfg->Pr > 0.0)) {
    noalloc_msg(errbuf, errlen, "material.gamma must be > 1 and R, W, T0, Pr positive");
    return CRUNA_ERR_ARG;
  }
  // explicit derivative cores only (the compact cores need factor arrays); built on the stack
  LineOp ops[3];
  for (int d = 0; d < 3; ++d) {
    HostFactors hf;        // stays empty for explicit cores
    std::string err;       // short messages only; not filled on success
    if (!build_diff_op(cfg->diff[d], cfg->n[d], ops[d], hf, err)) {
      noalloc_msg(errbuf, errlen, "unsupported derivative scheme or grid size for this direction");
      return CRUNA_ERR_ARG;
    }
    if (ops[d].kind == OP_STENCIL && (ops[d].solve || ops[d].r > 4 || ops[d].nb > 2 || ops[d].bw > 5)) {
      noalloc_msg(errbuf, errlen, "cruna_rhs_direct_noalloc supports the explicit derivative cores only");
      return CRUNA_ERR_UNSUPPORTED;
    }
  }
  // an error left pending by the caller's earlier work would otherwise be read back (and cleared) as
  // this call's failure: report it as such and launch nothing
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess) {
    noalloc_msg(errbuf, errlen, "a CUDA error from earlier work is pending on this thread; nothing launched");
    return CRUNA_ERR_CUDA;
  }
  // the array's device address in the current context, resolved on every call (cheap, allocates
  // nothing): host code must not pass the array's name to a kernel, it is only a host-side stand-in,
  // and a cached address would go stale if the host switched contexts or reset the device
  void *scratch = nullptr;
  if (cudaGetSymbolAddress(&scratch, g_noalloc_scratch) != cudaSuccess || !scratch) {
    const cudaError_t e = cudaGetLastError();
    noalloc_msg(errbuf, errlen, e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver
                                    ? "no usable current CUDA device"
                                    : "cudaGetSymbolAddress of the static scratch array failed");
    return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? CRUNA_ERR_NODEVICE : CRUNA_ERR_CUDA;
  }
  Grid g{cfg->n[0], cfg->n[1], cfg->n[2], npts};
  FusedArgs a;
  a.g = g;
  for (int d = 0; d < 3; ++d) {
    const double L = cfg->x1[d] - cfg->x0[d];                    // grid_transform.f90:40-56
    const int m = diff_is_periodic(cfg->diff[d]) ? cfg->n[d] : cfg->n[d] - 1;
    a.op[d] = to_dir(ops[d], m > 0 ? L / m : INFINITY, cfg->heat_flux_dx != 0);
  }
  a.WoR = cfg->W / cfg->R;
  a.mu0 = cfg->mu0;
  a.T0 = cfg->T0;
  a.gamma = cfg->gamma;
  a.cp_over_pr = cfg->gamma * (cfg->R / cfg->W) / (cfg->gamma - 1.0) / cfg->Pr;
  a.p_ref = 0.0;
  a.T_ref = 0.0;
  a.q = q;
  a.gbuf = scratch;                 // every value of the 15 fields is written by pass G before use
  a.rhs = rhs;
  a.force = nullptr;
  a.stage = 0;
  a.dt = 0.0;
  a.q0 = nullptr;
  a.acc = nullptr;
  a.qnext = nullptr;
  int R = 0;
  for (int d = 0; d < 3; ++d) R = std::max(R, halo_of(ops[d]));
  const int Rl = R <= 2 ? 2 : 4;
  bool per = true;
  for (int d = 0; d < 3; ++d) per = per && ops[d].kind == OP_STENCIL && ops[d].periodic && ops[d].r == Rl;
  const int bx = (g.n1 + TX - 1) / TX, by = (g.n2 + TY - 1) / TY;
  int nz = 1;
  a.kc = z_chunk(g.n3, bx, by, Rl, nz);
  const dim3 grid(bx, by, nz);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (Rl == 2) e = per ? noalloc_launch<2, true>(a, grid, s) : noalloc_launch<2, false>(a, grid, s);
  else e = per ? noalloc_launch<4, true>(a, grid, s) : noalloc_launch<4, false>(a, grid, s);
  if (e != cudaSuccess) {
    noalloc_msg(errbuf, errlen, cudaGetErrorString(e));
    return CRUNA_ERR_CUDA;
  }
  return CRUNA_OK;
}
