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
template <typename T>
struct Prim {
  T u, v, w, t, p, ru, rv, rw;
};

template <typename T>
__device__ __forceinline__ Prim<T> prim_at(const FusedArgs &a, long long pt) {
  const long long N = a.g.N;
  const double r = a.q[pt], ru = a.q[pt + N], rv = a.q[pt + 2 * N], rw = a.q[pt + 3 * N], p = a.q[pt + 4 * N];
  // u = rho*u / rho etc. (ns_rho_rhou_p.f90:95-99, trafos.f90:57) as products with 1/rho:
  // one division per point instead of four, at most one rounding step away from the quotients
  const double ir = 1.0 / r;
  Prim<T> o;
  o.u = T(ru * ir);
  o.v = T(rv * ir);
  o.w = T(rw * ir);
  o.t = T(a.WoR * p * ir - a.T_ref);
  o.p = T(p - a.p_ref);
  o.ru = T(ru);
  o.rv = T(rv);
  o.rw = T(rw);
  return o;
}

template <typename T, int R>
__global__ void __launch_bounds__(TX *TY, 2) k_pass_g(const __grid_constant__ FusedArgs a) {
  constexpr int PW = TX + 2 * R, PH = TY + 2 * R, PS = PW * PH;
  constexpr int NS = ring_slots(R);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *plane = reinterpret_cast<T *>(smem_raw);          // [7][PH][PW]
  T *ring = plane + 7 * PS;                            // [NS][6][TY*TX]
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int k0 = blockIdx.z * a.kc;
  const int k1 = min(k0 + a.kc, a.g.n3);
  const DirOpF &ox = a.op[0], &oy = a.op[1], &oz = a.op[2];
  const int gi = gidx(ox, i0 + tx), gj = gidx(oy, j0 + ty);
  const long long n1 = a.g.n1, n12 = (long long)a.g.n1 * a.g.n2;
  const bool inside = (i0 + tx) < a.g.n1 && (j0 + ty) < a.g.n2;

  auto ring_at = [&](int slot, int f) -> T * { return ring + (slot * 6 + f) * (TX * TY) + tid; };
  auto load_ring = [&](int kk) {
    const int gk = gidx(oz, kk);
    if (gk < 0 || gi < 0 || gj < 0) return;
    const Prim<T> pr = prim_at<T>(a, gi + n1 * gj + n12 * gk);
    const int slot = ((kk % NS) + NS) % NS;
    *ring_at(slot, 0) = pr.u;
    *ring_at(slot, 1) = pr.v;
    *ring_at(slot, 2) = pr.w;
    *ring_at(slot, 3) = pr.t;
    *ring_at(slot, 4) = pr.p;
    *ring_at(slot, 5) = pr.rw;
  };
  for (int kk = k0 - R; kk < k0 + R; ++kk) load_ring(kk);
  // register prefetch of the raw state entering the ring next (plane k+R) and of rho*u, rho*v of the
  // current plane, so their latency overlaps the previous plane's arithmetic
  const bool col = gi >= 0 && gj >= 0;
  const long long colpt = gi + n1 * gj;
  double pf[5] = {0, 0, 0, 0, 0};
  double pruv[2] = {0, 0};
  int pf_k = -1;
  auto prefetch = [&](int kk, int kc) {
    const int gk = gidx(oz, kk);
    pf_k = (gk >= 0 && col) ? gk : -1;
    if (pf_k >= 0) {
      const long long pt = colpt + n12 * gk;
#pragma unroll
      for (int v = 0; v < 5; ++v) pf[v] = a.q[pt + v * a.g.N];
    }
    if (col && kc < k1) {
      const long long pt = colpt + n12 * kc;
      pruv[0] = a.q[pt + a.g.N];
      pruv[1] = a.q[pt + 2 * a.g.N];
    }
  };
  prefetch(k0 + R, k0);

  constexpr int nhalo = 2 * R * (TX + TY);
  for (int k = k0; k < k1; ++k) {
    if (pf_k >= 0) {
      const double ir = 1.0 / pf[0];
      const int sl = ((k + R) % NS + NS) % NS;
      *ring_at(sl, 0) = T(pf[1] * ir);
      *ring_at(sl, 1) = T(pf[2] * ir);
      *ring_at(sl, 2) = T(pf[3] * ir);
      *ring_at(sl, 3) = T(a.WoR * pf[4] * ir - a.T_ref);
      *ring_at(sl, 4) = T(pf[4] - a.p_ref);
      *ring_at(sl, 5) = T(pf[3]);
    }
    const int slot = k % NS;
    // centre of the plane from this thread's ring, plus rho*u and rho*v
    {
      T *c = plane + (ty + R) * PW + (tx + R);
      c[0 * PS] = *ring_at(slot, 0);
      c[1 * PS] = *ring_at(slot, 1);
      c[2 * PS] = *ring_at(slot, 2);
      c[3 * PS] = *ring_at(slot, 3);
      c[4 * PS] = *ring_at(slot, 4);
      c[5 * PS] = T(pruv[0]);
      c[6 * PS] = T(pruv[1]);
    }
    prefetch(k + R + 1, k + 1);
    // halo strips (no corners)
    for (int h = tid; h < nhalo; h += TX * TY) {
      int lx, ly;
      if (h < 2 * R * TY) {            // left / right strips
        const int side = h / (R * TY), e = h % (R * TY);
        ly = e / R;
        lx = side == 0 ? -R + e % R : TX + e % R;
      } else {                          // bottom / top strips
        const int e2 = h - 2 * R * TY;
        const int side = e2 / (R * TX), e = e2 % (R * TX);
        lx = e % TX;
        ly = side == 0 ? -R + e / TX : TY + e / TX;
      }
      const int hi = gidx(ox, i0 + lx), hj = gidx(oy, j0 + ly);
      if (hi < 0 || hj < 0) continue;
      const Prim<T> pr = prim_at<T>(a, hi + n1 * hj + n12 * k);
      T *c = plane + (ly + R) * PW + (lx + R);
      c[0 * PS] = pr.u; c[1 * PS] = pr.v; c[2 * PS] = pr.w; c[3 * PS] = pr.t;
      c[4 * PS] = pr.p; c[5 * PS] = pr.ru; c[6 * PS] = pr.rv;
    }
    __syncthreads();
    if (inside) {
      const int i = i0 + tx, j = j0 + ty;
      const T *c = plane + (ty + R) * PW + (tx + R);
      const T *U = c, *V = c + PS, *W = c + 2 * PS, *TT = c + 3 * PS, *P = c + 4 * PS, *RU = c + 5 * PS,
              *RV = c + 6 * PS;
      const T *zu = ring_at(slot, 0), *zv = ring_at(slot, 1), *zw = ring_at(slot, 2), *zt = ring_at(slot, 3),
              *zp = ring_at(slot, 4), *zrw = ring_at(slot, 5);
      // ring neighbours of slot: slot +- m (mod NS); build pointer with stride in units of T
      // since slots wrap, gather the column into registers first
      T cu[NS], cv[NS], cw[NS], ct[NS], cp[NS], crw[NS];
#pragma unroll
      for (int m = -R; m <= R; ++m) {
        const int sl = (slot + m + NS) % NS;
        cu[m + R] = *ring_at(sl, 0);
        cv[m + R] = *ring_at(sl, 1);
        cw[m + R] = *ring_at(sl, 2);
        ct[m + R] = *ring_at(sl, 3);
        cp[m + R] = *ring_at(sl, 4);
        crw[m + R] = *ring_at(sl, 5);
      }
      (void)zu; (void)zv; (void)zw; (void)zt; (void)zp; (void)zrw;
      const T sx = T(ox.scale), sy = T(oy.scale), sz = T(oz.scale);
      // velocity gradients (:102-112)
      const T ux = dsm<T, R>(ox, U, 1, i) * sx, uy = dsm<T, R>(oy, U, PW, j) * sy, uz = dsz<T, R>(oz, cu, k) * sz;
      const T vx = dsm<T, R>(ox, V, 1, i) * sx, vy = dsm<T, R>(oy, V, PW, j) * sy, vz = dsz<T, R>(oz, cv, k) * sz;
      const T wx = dsm<T, R>(ox, W, 1, i) * sx, wy = dsm<T, R>(oy, W, PW, j) * sy, wz = dsz<T, R>(oz, cw, k) * sz;
      // temperature gradient (:189-191)
      const T tgx = dsm<T, R>(ox, TT, 1, i) * T(ox.scale_h);
      const T tgy = dsm<T, R>(oy, TT, PW, j) * T(oy.scale_h);
      const T tgz = dsz<T, R>(oz, ct, k) * T(oz.scale_h);
      // viscosity and stresses (:115-128)
      const T Tabs = T(double(ct[R]) + a.T_ref);
      const T mu = T(a.mu0) * T(pow(double(Tabs) / a.T0, 1.5)) * (T(a.T0 + 110.4) / (Tabs + T(110.4)));
      const T mu_div = -(T(2.0 / 3.0) * mu * (ux + vy + wz));
      const T t11 = mu_div + T(2) * mu * ux;
      const T t22 = mu_div + T(2) * mu * vy;
      const T t33 = mu_div + T(2) * mu * wz;
      const T t12 = mu * (uy + vx);
      const T t13 = mu * (uz + wx);
      const T t23 = mu * (vz + wy);
      const T lam = mu * T(a.cp_over_pr);
      // friction work (:204-206)
      const T phi = t11 * ux + t12 * uy + t13 * uz + t12 * vx + t22 * vy + t23 * vz + t13 * wx + t23 * wy +
                    t33 * wz;
      // convective terms (:131-186)
      const T m1 = dsm<T, R>(ox, RU, 1, i) * sx, m2 = dsm<T, R>(oy, RV, PW, j) * sy,
              m3 = dsz<T, R>(oz, crw, k) * sz;
      const T px = dsm<T, R>(ox, P, 1, i) * sx, py = dsm<T, R>(oy, P, PW, j) * sy, pz = dsz<T, R>(oz, cp, k) * sz;
      const T a1x = dsm2<T, R>(ox, RU, U, 1, i) * sx, a1y = dsm2<T, R>(oy, RV, U, PW, j) * sy,
              a1z = dsz2<T, R>(oz, crw, cu, k) * sz;
      const T a2x = dsm2<T, R>(ox, RU, V, 1, i) * sx, a2y = dsm2<T, R>(oy, RV, V, PW, j) * sy,
              a2z = dsz2<T, R>(oz, crw, cv, k) * sz;
      const T a3x = dsm2<T, R>(ox, RU, W, 1, i) * sx, a3y = dsm2<T, R>(oy, RV, W, PW, j) * sy,
              a3z = dsz2<T, R>(oz, crw, cw, k) * sz;
      const T pref = T(a.p_ref);
      const T ex = pref * ux + dsm2<T, R>(ox, P, U, 1, i) * sx;
      const T ey = pref * vy + dsm2<T, R>(oy, P, V, PW, j) * sy;
      const T ez = pref * wz + dsz2<T, R>(oz, cp, cw, k) * sz;
      const T uc = cu[R], vc = cv[R], wc = cw[R];
      const double gt = a.gamma / (a.gamma - 1.0);
      const T c1 = -m1 - m2 - m3;
      const T c2 = -a1x - a1y - a1z - px;
      const T c3 = -a2x - a2y - a2z - py;
      const T c4 = -a3x - a3y - a3z - pz;
      T c5 = T(gt) * (-ex - ey - ez);
      c5 = c5 + uc * px + vc * py + wc * pz;
      T *go = static_cast<T *>(a.gbuf);
      const long long N = a.g.N, pt = i + n1 * j + n12 * k;
      go[pt + 0 * N] = c1;
      go[pt + 1 * N] = c2;
      go[pt + 2 * N] = c3;
      go[pt + 3 * N] = c4;
      go[pt + 4 * N] = c5;
      go[pt + 5 * N] = t11;
      go[pt + 6 * N] = t12;
      go[pt + 7 * N] = t13;
      go[pt + 8 * N] = t22;
      go[pt + 9 * N] = t23;
      go[pt + 10 * N] = t33;
      go[pt + 11 * N] = lam * tgx;
      go[pt + 12 * N] = lam * tgy;
      go[pt + 13 * N] = lam * tgz;
      go[pt + 14 * N] = phi;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------
// pass D
// plane fields: 0 t11, 1 t12, 2 t13, 3 t22, 4 t23, 5 hx, 6 hy ; ring fields: 0 t13, 1 t23, 2 t33, 3 hz
// ------------------------------------------------------------------------------------------------
template <typename T, int R>
__global__ void __launch_bounds__(TX *TY, 3) k_pass_d(const __grid_constant__ FusedArgs a) {
  constexpr int PW = TX + 2 * R, PH = TY + 2 * R, PS = PW * PH;
  constexpr int NS = ring_slots(R);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *plane = reinterpret_cast<T *>(smem_raw);          // [7][PH][PW]
  T *ring = plane + 7 * PS;                            // [NS][4][TY*TX]
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int k0 = blockIdx.z * a.kc;
  const int k1 = min(k0 + a.kc, a.g.n3);
  const DirOpF &ox = a.op[0], &oy = a.op[1], &oz = a.op[2];
  const int gi = gidx(ox, i0 + tx), gj = gidx(oy, j0 + ty);
  const long long N = a.g.N, n1 = a.g.n1, n12 = (long long)a.g.n1 * a.g.n2;
  const bool inside = (i0 + tx) < a.g.n1 && (j0 + ty) < a.g.n2;
  const T *G = static_cast<const T *>(a.gbuf);

  auto ring_at = [&](int slot, int f) -> T * { return ring + (slot * 4 + f) * (TX * TY) + tid; };
  auto load_ring = [&](int kk) {
    const int gk = gidx(oz, kk);
    if (gk < 0 || gi < 0 || gj < 0) return;
    const long long pt = gi + n1 * gj + n12 * gk;
    const int slot = ((kk % NS) + NS) % NS;
    *ring_at(slot, 0) = G[pt + 7 * N];
    *ring_at(slot, 1) = G[pt + 9 * N];
    *ring_at(slot, 2) = G[pt + 10 * N];
    *ring_at(slot, 3) = G[pt + 13 * N];
  };
  for (int kk = k0 - R; kk < k0 + R; ++kk) load_ring(kk);

  constexpr int pf[7] = {5, 6, 7, 8, 9, 11, 12};   // G fields of the plane
  constexpr int nhalo = 2 * R * (TX + TY);
  for (int k = k0; k < k1; ++k) {
    load_ring(k + R);
    const int slot = k % NS;
    if (gi >= 0 && gj >= 0) {
      const long long pt = gi + n1 * gj + n12 * k;
      T *c = plane + (ty + R) * PW + (tx + R);
#pragma unroll
      for (int f = 0; f < 7; ++f) c[f * PS] = G[pt + pf[f] * N];
    }
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
      // x-halo cells need t11,t12,t13,hx; y-halo cells need t12,t22,t23,hy; loading all 7 is simpler
#pragma unroll
      for (int f = 0; f < 7; ++f) c[f * PS] = G[pt + pf[f] * N];
    }
    __syncthreads();
    if (inside) {
      const int i = i0 + tx, j = j0 + ty;
      const T *c = plane + (ty + R) * PW + (tx + R);
      T z13[NS], z23[NS], z33[NS], zh[NS];
#pragma unroll
      for (int m = -R; m <= R; ++m) {
        const int sl = (slot + m + NS) % NS;
        z13[m + R] = *ring_at(sl, 0);
        z23[m + R] = *ring_at(sl, 1);
        z33[m + R] = *ring_at(sl, 2);
        zh[m + R] = *ring_at(sl, 3);
      }
      const T sx = T(ox.scale), sy = T(oy.scale), sz = T(oz.scale);
      const T v1x = dsm<T, R>(ox, c + 0 * PS, 1, i) * sx;       // d_x tau_11
      const T v1y = dsm<T, R>(oy, c + 1 * PS, PW, j) * sy;      // d_y tau_12
      const T v1z = dsz<T, R>(oz, z13, k) * sz;          // d_z tau_13
      const T v2x = dsm<T, R>(ox, c + 1 * PS, 1, i) * sx;       // d_x tau_21
      const T v2y = dsm<T, R>(oy, c + 3 * PS, PW, j) * sy;      // d_y tau_22
      const T v2z = dsz<T, R>(oz, z23, k) * sz;          // d_z tau_23
      const T v3x = dsm<T, R>(ox, c + 2 * PS, 1, i) * sx;       // d_x tau_31
      const T v3y = dsm<T, R>(oy, c + 4 * PS, PW, j) * sy;      // d_y tau_32
      const T v3z = dsz<T, R>(oz, z33, k) * sz;          // d_z tau_33
      const T qx = dsm<T, R>(ox, c + 5 * PS, 1, i) * T(ox.scale_h);   // d_x (lambda d_x T)
      const T qy = dsm<T, R>(oy, c + 6 * PS, PW, j) * T(oy.scale_h);
      const T qz = dsz<T, R>(oz, zh, k) * T(oz.scale_h);
      const long long pt = i + n1 * j + n12 * k;
      // assembly in the reference's order (:135, 143-149, 157-163, 171-177, 185-209)
      double r1 = double(G[pt]);
      double r2 = double(G[pt + N]);
      r2 = r2 + double(v1x); r2 = r2 + double(v1y); r2 = r2 + double(v1z);
      double r3 = double(G[pt + 2 * N]);
      r3 = r3 + double(v2x); r3 = r3 + double(v2y); r3 = r3 + double(v2z);
      double r4 = double(G[pt + 3 * N]);
      r4 = r4 + double(v3x); r4 = r4 + double(v3y); r4 = r4 + double(v3z);
      double r5 = double(G[pt + 4 * N]);
      r5 = r5 + double(qx); r5 = r5 + double(qy); r5 = r5 + double(qz);
      r5 = r5 + double(G[pt + 14 * N]);
      r5 = (a.gamma - 1.0) * r5;
      if (a.force) {                                              // :212
        r1 = r1 + a.force[pt]; r2 = r2 + a.force[pt + N]; r3 = r3 + a.force[pt + 2 * N];
        r4 = r4 + a.force[pt + 3 * N]; r5 = r5 + a.force[pt + 4 * N];
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

template <typename T, int R>
size_t smem_g() {
  return sizeof(T) * (7 * (TX + 2 * R) * (TY + 2 * R) + ring_slots(R) * 6 * TX * TY);
}
template <typename T, int R>
size_t smem_d() {
  return sizeof(T) * (7 * (TX + 2 * R) * (TY + 2 * R) + ring_slots(R) * 4 * TX * TY);
}

template <typename T, int R>
void launch_passes(cruna_ctx *c, FusedArgs &a, const double *q, double *rhs_or_null) {
  static bool configured = false;
  if (!configured) {
    CRUNA_CUDA_CHECK(cudaFuncSetAttribute(k_pass_g<T, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem_g<T, R>()));
    CRUNA_CUDA_CHECK(cudaFuncSetAttribute(k_pass_d<T, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem_d<T, R>()));
    configured = true;
  }
  const int bx = (c->g.n1 + TX - 1) / TX, by = (c->g.n2 + TY - 1) / TY;
  const int n3 = c->g.n3;
  // z chunks: enough blocks to fill the GPU a few times while keeping the 2R-plane preload small
  int nz = std::max(1, std::min(n3, (4 * 148 + bx * by - 1) / (bx * by)));
  int kc = (n3 + nz - 1) / nz;
  kc = std::max(kc, std::min(n3, 4 * R));
  nz = (n3 + kc - 1) / kc;
  a.kc = kc;
  dim3 grid(bx, by, nz), block(TX, TY);
  {
    ProfScope ps(c, "pass_g");
    k_pass_g<T, R><<<grid, block, smem_g<T, R>(), c->stream>>>(a);
    CRUNA_LAUNCH_CHECK(c);
  }
  (void)q;
  (void)rhs_or_null;
  {
    ProfScope ps(c, "pass_d");
    k_pass_d<T, R><<<grid, block, smem_d<T, R>(), c->stream>>>(a);
    CRUNA_LAUNCH_CHECK(c);
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
  if (fp32) {
    if (R <= 2) launch_passes<float, 2>(c, a, q, rhs);
    else launch_passes<float, 4>(c, a, q, rhs);
  } else {
    if (R <= 2) launch_passes<double, 2>(c, a, q, rhs);
    else launch_passes<double, 4>(c, a, q, rhs);
  }
  if (stage == 0 || split) {
    if (c->has_rhs_bc) bc_rhs(c, rhs, q);                          // :218
    if (split) rk_stage(c, stage, dt, rhs, q0, acc, qnext);
  }
}

}  // namespace cruna
