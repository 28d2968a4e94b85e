// Gradient of an objective through the direct and adjoint loops with binomial checkpointing in HBM.
//
// CRUNA's optimisation loop (src/main/cruna.f90:78-179) runs calc_direct, calc_objective,
// calc_adjoint with calc_objective_g as the adjoint source, then calc_grad; the direct trajectory is
// kept whole in memory Q(:,:,:,:,nt) (src/data/data_rhs.f90:25) or spilled per time subset to HDF5
// (computation_direct.f90:131, computation_adjoint.f90:58).  Here the trajectory is recomputed from
// a few snapshots kept in HBM: rev(a, b, s) produces Q(b) .. Q(a+1) in reverse order from the
// snapshot Q(a) with s free snapshots -- advance to a + k, store, reverse the right part with s - 1
// snapshots, run the adjoint step at the snapshot, reverse the left part with s snapshots.  k is
// chosen by a dynamic programme restricted to the binomial bounds (with t the least number of sweeps
// such that M(s, t) = C(s+1+t, t) - 1 >= n states, the right part holds at most M(s-1, t) and the left
// part at most M(s, t-1) states), which gives the minimal number of recomputed direct steps.
//
// Objectives (the reference leaves them to each case, src/opt/objective.f90:19-45):
//   plane_p2:        J = sum_{nt=1..T} dt * sum_plane w (p - p_inf)^2, adjoint source
//                    g = -dj/dq = (0,0,0,0, -2 w (p - p_inf)) on the plane (calc_objective_g; the sign makes
//                    the backward-integrated qs an approximation of dJ/dq)
//   kinetic_energy:  J = sum dV |rho u|^2 / (2 rho) at t_T, qs(T) = dJ/dq(T)
//   enstrophy:       J = sum dV |curl u|^2 / 2 at t_T (the solver's derivative operators), qs(T) = dJ/dq(T)
// Gradients (calc_grad, force.f90:41-45): dJ/df for a time-constant forcing added to the RHS is the
// time integral of qs (trapezoid over the adjoint trajectory), dJ/dq0 = qs(0).
// Discrete mode (cruna_set_adjoint_mode 1) replaces the reference's continuous adjoint step by the
// exact transpose of the direct loop step (discrete_adjoint.cu): J is the same sum over the same
// states, and dJ/dq0, dJ/df are its exact derivatives.
#include <algorithm>
#include <cmath>
#include <vector>

#include "cruna_internal.cuh"

namespace cruna {

namespace {

constexpr int RB = 256;   // reduction block
constexpr int RG = 592;   // reduction grid (4 x 148): fixed, so sums are deterministic

long long Mst(int s, int t) {
  // C(s+1+t, t) - 1, saturating
  double v = 1.0;
  for (int i = 1; i <= t; ++i) {
    v = v * (double)(s + 1 + i) / (double)i;
    if (v > 4e18) return (long long)4e18;
  }
  return (long long)std::llround(v) - 1;
}

// kbest[n*(S+1)+s] = optimal first checkpoint distance for n states and s free snapshots
void build_schedule(int n, int S, std::vector<int> &kbest, long long &cost_out) {
  const int W = S + 1;
  std::vector<long long> cost((size_t)(n + 1) * W, 0);
  kbest.assign((size_t)(n + 1) * W, 1);
  for (int s = 0; s <= S; ++s) {
    for (int m = 1; m <= n; ++m) {
      long long &c = cost[(size_t)m * W + s];
      if (s == 0) {
        c = (long long)m * (m + 1) / 2;
        continue;
      }
      int t = 0;
      while (Mst(s, t) < m) ++t;
      const long long lo = std::max<long long>(1, m - Mst(s - 1, t));
      const long long hi = std::min<long long>(m, Mst(s, t - 1) + 1);
      long long best = -1;
      int bk = (int)lo;
      for (long long k = lo; k <= hi; ++k) {
        const long long v = k + cost[(size_t)(m - k) * W + (s - 1)] + cost[(size_t)(k - 1) * W + s];
        if (best < 0 || v < best) {
          best = v;
          bk = (int)k;
        }
      }
      c = best;
      kbest[(size_t)m * W + s] = bk;
    }
  }
  cost_out = cost[(size_t)n * W + S];
}

// ---- objective kernels (deterministic two-level sums) --------------------------------------------
__global__ void k_plane_obj(Grid g, int normal, int index, double w, double p_inf, const double *q, double *gsrc,
                            double *partial, double gsign) {
  __shared__ double sh[RB];
  const long long n1 = g.n1, n2 = g.n2, n3 = g.n3;
  const long long na = normal == 0 ? n2 : n1, nb = normal == 2 ? n2 : n3;
  const long long cnt = na * nb;
  double acc = 0.0;
  for (long long t = blockIdx.x * (long long)RB + threadIdx.x; t < cnt; t += (long long)RG * RB) {
    const long long a = t % na, b = t / na;
    long long i, j, k;
    if (normal == 0) { i = index; j = a; k = b; }
    else if (normal == 1) { i = a; j = index; k = b; }
    else { i = a; j = b; k = index; }
    const long long p = i + n1 * (j + n2 * k);
    const double dp = q[p + 4 * g.N] - p_inf;
    acc += w * dp * dp;
    gsrc[p + 4 * g.N] = gsign * (2.0 * w * dp);
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = RB / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__global__ void k_ke_obj(Grid g, double dV, const double *q, double *qs_out, double *partial) {
  __shared__ double sh[RB];
  double acc = 0.0;
  const long long N = g.N;
  for (long long p = blockIdx.x * (long long)RB + threadIdx.x; p < N; p += (long long)RG * RB) {
    const double r = q[p], mu = q[p + N], mv = q[p + 2 * N], mw = q[p + 3 * N];
    acc += dV * 0.5 * (mu * mu + mv * mv + mw * mw) / r;
    if (qs_out) {
      const double u = mu / r, v = mv / r, w = mw / r;
      qs_out[p] = dV * (-0.5 * (u * u + v * v + w * w));
      qs_out[p + N] = dV * u;
      qs_out[p + 2 * N] = dV * v;
      qs_out[p + 3 * N] = dV * w;
      qs_out[p + 4 * N] = 0.0;
    }
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = RB / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

__global__ void k_sum_partials(const double *partial, int n, double *out, double scale, int accumulate) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += partial[i];
    out[0] = accumulate ? out[0] + scale * s : scale * s;
  }
}

__global__ void k_axpy(long long M, double a, const double *x, double *y, int overwrite) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < M; p += (long long)gridDim.x * blockDim.x)
    y[p] = overwrite ? a * x[p] : y[p] + a * x[p];
}

// u_i = (rho u_i) / rho, three fields
__global__ void k_velocity(long long N, const double *__restrict__ q, double *__restrict__ u) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
    const double r = q[p];
    u[p] = q[p + N] / r;
    u[p + N] = q[p + 2 * N] / r;
    u[p + 2 * N] = q[p + 3 * N] / r;
  }
}

// a = a - b (one field)
__global__ void k_sub(long long N, double *__restrict__ a, const double *__restrict__ b) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x)
    a[p] = a[p] - b[p];
}

// partial sums of dV * 0.5 |omega|^2 (fixed grid and block: deterministic)
__global__ void k_ens_obj(Grid g, double dV, const double *w, double *partial) {
  __shared__ double sh[RB];
  double acc = 0.0;
  const long long N = g.N;
  for (long long p = blockIdx.x * (long long)RB + threadIdx.x; p < N; p += (long long)RG * RB) {
    const double a = w[p], b = w[p + N], d = w[p + 2 * N];
    acc += dV * 0.5 * (a * a + b * b + d * d);
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = RB / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// lam(1..3) hold curl^T omega on entry; dZ/dq = (-sum u_i gu_i / rho, gu_i / rho, 0), gu = dV curl^T omega
__global__ void k_ens_grad(long long N, double dV, const double *__restrict__ q, const double *__restrict__ u,
                           double *__restrict__ lam) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
    const double r = q[p];
    const double g1 = dV * lam[p + N], g2 = dV * lam[p + 2 * N], g3 = dV * lam[p + 3 * N];
    lam[p] = -(u[p] * g1 + u[p + N] * g2 + u[p + 2 * N] * g3) / r;
    lam[p + N] = g1 / r;
    lam[p + 2 * N] = g2 / r;
    lam[p + 3 * N] = g3 / r;
    lam[p + 4 * N] = 0.0;
  }
}

}  // namespace

double cell_volume(const cruna_ctx *c) {
  double dV = 1.0;
  for (int d = 0; d < 3; ++d)
    if (c->cfg.n[d] > 1) dV *= c->dx[d];
  return dV;
}

// Z = sum dV |curl u|^2 / 2 with the context's derivative operators (h = dx) into J (scaled by 1,
// accumulated or not); lam (optional) = dZ/dq through the transposed operators.  Workspace: the stage
// buffers st[2] (u, a temporary, the transposes' scratch) and st[3] (omega), free between steps.
void enstrophy_objective(cruna_ctx *c, const double *q, double *lam, double *partial, double *J, int accumulate) {
  const long long N = c->g.N;
  double *u = c->st[2], *t = u + 3 * N, *scr = u + 4 * N, *w = c->st[3];
  const int blocks = (int)std::min<long long>((N + 255) / 256, 148LL * 16);
  k_velocity<<<blocks, 256, 0, c->stream>>>(N, q, u);
  CRUNA_LAUNCH_CHECK(c);
  const double *dx = c->dx;
  auto D = [&](int d, const double *f, double *out) { apply_diff(c, d, f, nullptr, out, dx[d], 1); };
  auto sub = [&](double *a, const double *b) {
    k_sub<<<blocks, 256, 0, c->stream>>>(N, a, b);
    CRUNA_LAUNCH_CHECK(c);
  };
  double *wx = w, *wy = w + N, *wz = w + 2 * N;
  const double *u1 = u, *u2 = u + N, *u3 = u + 2 * N;
  D(1, u3, wx); D(2, u2, t); sub(wx, t);   // D_y w - D_z v
  D(2, u1, wy); D(0, u3, t); sub(wy, t);   // D_z u - D_x w
  D(0, u2, wz); D(1, u1, t); sub(wz, t);   // D_x v - D_y u
  k_ens_obj<<<RG, RB, 0, c->stream>>>(c->g, cell_volume(c), w, partial);
  CRUNA_LAUNCH_CHECK(c);
  k_sum_partials<<<1, 32, 0, c->stream>>>(partial, RG, J, 1.0, accumulate);
  CRUNA_LAUNCH_CHECK(c);
  if (!lam) return;
  auto DT = [&](int d, const double *f, double *out) { diff_transpose(c, d, f, out, dx[d], scr); };
  double *g1 = lam + N, *g2 = lam + 2 * N, *g3 = lam + 3 * N;
  DT(2, wy, g1); DT(1, wz, t); sub(g1, t);   // D_z^T omega_y - D_y^T omega_z
  DT(0, wz, g2); DT(2, wx, t); sub(g2, t);   // D_x^T omega_z - D_z^T omega_x
  DT(1, wx, g3); DT(0, wy, t); sub(g3, t);   // D_y^T omega_x - D_x^T omega_y
  k_ens_grad<<<blocks, 256, 0, c->stream>>>(N, cell_volume(c), q, u, lam);
  CRUNA_LAUNCH_CHECK(c);
}

// the final-time objectives: J (overwritten) and, with lam, lam = dJ/dq
void terminal_objective(cruna_ctx *c, const cruna_objective *obj, const double *q, double *lam, double *partial,
                        double *J) {
  if (obj->kind == CRUNA_OBJ_ENSTROPHY) {
    enstrophy_objective(c, q, lam, partial, J, 0);
    return;
  }
  k_ke_obj<<<RG, RB, 0, c->stream>>>(c->g, cell_volume(c), q, lam, partial);
  CRUNA_LAUNCH_CHECK(c);
  k_sum_partials<<<1, 32, 0, c->stream>>>(partial, RG, J, 1.0, 0);
  CRUNA_LAUNCH_CHECK(c);
}

// kinetic energy and enstrophy of a state into out[0], out[1] (device)
void diagnostics_impl(cruna_ctx *c, const double *q, double *out, double *partial) {
  k_ke_obj<<<RG, RB, 0, c->stream>>>(c->g, cell_volume(c), q, nullptr, partial);
  CRUNA_LAUNCH_CHECK(c);
  k_sum_partials<<<1, 32, 0, c->stream>>>(partial, RG, out, 1.0, 0);
  CRUNA_LAUNCH_CHECK(c);
  enstrophy_objective(c, q, nullptr, partial, out + 1, 0);
}

struct GradientRun {
  cruna_ctx *c;
  int nsteps;
  const cruna_objective *obj;
  std::vector<int> kbest;
  int S;
  double *work;                    // current direct state
  std::vector<double *> slots;     // snapshot buffers
  std::vector<int> slot_step;      // step held by a slot, -1 free
  double *qs, *gsrc, *gf, *J, *partial;
  double *qN = nullptr;            // discrete mode: the final state Q(nsteps)
  bool discrete = false;
  long long advanced = 0;
  void (*direct_step)(cruna_ctx *, double *, int);
  void (*adjoint_step)(cruna_ctx *, double *, const double *, const double *, int);

  long long M5() const { return c->g.N * 5; }
  int slot_of(int step) const {
    for (size_t i = 0; i < slots.size(); ++i)
      if (slot_step[i] == step) return (int)i;
    return -1;
  }
  int take(int step) {
    for (size_t i = 0; i < slots.size(); ++i)
      if (slot_step[i] < 0) {
        slot_step[i] = step;
        return (int)i;
      }
    throw std::runtime_error("checkpoint schedule ran out of snapshots");
  }
  bool host_slots = false;         // snapshots in pinned host memory (cruna_set_snapshot_memory)
  // Host slots, when HBM has room for one more state: hcache holds the last slot stored or loaded.
  // A store copies work into it and drains it to the host on a copy stream while the direct steps
  // go on; a load of the cached slot (the restart right after a store, each restart of a leaf) is a
  // device copy.  The cache is overwritten only after its pending drain (d2h_done) has finished.
  double *hcache = nullptr;
  int hcache_slot = -1;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t cache_ready = nullptr, d2h_done = nullptr;
  ~GradientRun() {
    if (copy_stream) cudaStreamSynchronize(copy_stream);
    if (cache_ready) cudaEventDestroy(cache_ready);
    if (d2h_done) cudaEventDestroy(d2h_done);
    if (copy_stream) cudaStreamDestroy(copy_stream);
  }
  void enable_cache(double *buf) {
    CRUNA_CUDA_CHECK(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
    CRUNA_CUDA_CHECK(cudaEventCreateWithFlags(&cache_ready, cudaEventDisableTiming));
    CRUNA_CUDA_CHECK(cudaEventCreateWithFlags(&d2h_done, cudaEventDisableTiming));
    hcache = buf;
  }
  void copy(double *dst, const double *src) {
    if (dst == src) return;
    CRUNA_CUDA_CHECK(cudaMemcpyAsync(dst, src, sizeof(double) * c->g.N * 5, cudaMemcpyDefault, c->stream));
  }
  void fill_cache(const double *src, int s) {
    CRUNA_CUDA_CHECK(cudaStreamWaitEvent(c->stream, d2h_done, 0));
    copy(hcache, src);
    hcache_slot = s;
  }
  // dst <- snapshot slot s
  void load(double *dst, int s) {
    if (!hcache) return copy(dst, slots[s]);
    if (hcache_slot != s) fill_cache(slots[s], s);
    copy(dst, hcache);
  }
  // snapshot slot s <- work
  void store(int s) {
    if (!hcache) return copy(slots[s], work);
    fill_cache(work, s);
    CRUNA_CUDA_CHECK(cudaEventRecord(cache_ready, c->stream));
    CRUNA_CUDA_CHECK(cudaStreamWaitEvent(copy_stream, cache_ready, 0));
    CRUNA_CUDA_CHECK(cudaMemcpyAsync(slots[s], hcache, sizeof(double) * c->g.N * 5, cudaMemcpyDeviceToHost,
                                     copy_stream));
    CRUNA_CUDA_CHECK(cudaEventRecord(d2h_done, copy_stream));
  }
  // the state held by snapshot slot sm, where the kernels can read it (host slots go through work)
  const double *at_snapshot(int sm) {
    if (!host_slots) return slots[sm];
    load(work, sm);
    return work;
  }
  void advance(int a, int b) {
    for (int nt = a + 1; nt <= b; ++nt) {
      direct_step(c, work, nt);
      ++advanced;
    }
  }
  void axpy(double a, const double *x, double *y, bool overwrite) {
    k_axpy<<<(int)std::min<long long>((M5() + 255) / 256, 148LL * 32), 256, 0, c->stream>>>(M5(), a, x, y,
                                                                                             overwrite ? 1 : 0);
    CRUNA_LAUNCH_CHECK(c);
  }
  void plane_source(const double *q) {
    const int nd = obj->normal - 1;
    double w = 1.0;
    for (int d = 0; d < 3; ++d)
      if (d != nd && c->cfg.n[d] > 1) w *= c->dx[d];
    k_plane_obj<<<RG, RB, 0, c->stream>>>(c->g, nd, obj->index - 1, w, obj->p_inf, q, gsrc, partial, 1.0);
    CRUNA_LAUNCH_CHECK(c);
    k_sum_partials<<<1, 32, 0, c->stream>>>(partial, RG, J, c->cfg.dt, 1);
    CRUNA_LAUNCH_CHECK(c);
  }
  // discrete mode: the state Q(nt) is the input of step nt + 1, whose transpose maps the cotangent of
  // Q(nt + 1) to that of Q(nt); the objective's own term at Q(nt) is added after it
  void adjoint_discrete(int nt, const double *qnt) {
    const double dt = c->cfg.dt;
    const bool plane = obj->kind == CRUNA_OBJ_PLANE_P2;
    if (nt == nsteps - 1) {
      copy(qN, qnt);
      direct_step(c, qN, nsteps);
      ++advanced;
      if (plane) {
        plane_source(qN);
        axpy(dt, gsrc, qs, true);
      } else {
        terminal_objective(c, obj, qN, qs, partial, J);
      }
    }
    step_direct_vjp(c, qnt, qs, qs, gf, nt + 1);
    if (plane && nt >= 1) {
      plane_source(qnt);
      axpy(dt, gsrc, qs, false);
    }
  }
  // adjoint step nt on the direct state Q(nt) (computation_adjoint.f90:66-108)
  void adjoint(int nt, const double *qnt) {
    if (discrete) {
      adjoint_discrete(nt, qnt);
      return;
    }
    const double dt = c->cfg.dt;
    const bool plane = obj->kind == CRUNA_OBJ_PLANE_P2;
    if (nt == nsteps) {
      if (!plane) terminal_objective(c, obj, qnt, qs, partial, J);
      if (gf) axpy(0.5 * dt, qs, gf, true);
    }
    if (plane) {
      const int nd = obj->normal - 1;
      double w = 1.0;
      for (int d = 0; d < 3; ++d)
        if (d != nd && c->cfg.n[d] > 1) w *= c->dx[d];
      // CRUNA's adjoint stepper integrates dqs/dt = rhs_adjoint(qs) + g backwards (rk_o4_e.f90:62-105),
      // so qs approximates dJ/dq when the source is g = -dj/dq
      k_plane_obj<<<RG, RB, 0, c->stream>>>(c->g, nd, obj->index - 1, w, obj->p_inf, qnt, gsrc, partial, -1.0);
      CRUNA_LAUNCH_CHECK(c);
      k_sum_partials<<<1, 32, 0, c->stream>>>(partial, RG, J, dt, 1);
      CRUNA_LAUNCH_CHECK(c);
    }
    adjoint_step(c, qs, qnt, plane ? gsrc : nullptr, nt);
    if (gf) axpy(nt - 1 > 0 ? dt : 0.5 * dt, qs, gf, false);
  }
  void rev(int a, int b, int s) {
    const int n = b - a;
    if (n <= 0) return;
    const int sa = slot_of(a);
    if (s == 0) {
      for (int nt = b; nt > a; --nt) {
        load(work, sa);
        advance(a, nt);
        adjoint(nt, work);
      }
      return;
    }
    const int k = kbest[(size_t)n * (S + 1) + s];
    const int m = a + k;
    load(work, sa);
    advance(a, m);
    const int sm = take(m);
    store(sm);
    rev(m, b, s - 1);
    adjoint(m, at_snapshot(sm));
    slot_step[sm] = -1;
    rev(a, m - 1, s);
  }
};

// direct / adjoint loop bodies shared with the run loops (capi.cu)
void direct_loop_step(cruna_ctx *c, double *q, int nt);
void adjoint_loop_step(cruna_ctx *c, double *qs, const double *q0, const double *g, int nt);

long long gradient_impl(cruna_ctx *c, const double *q0, int nsteps, int nsnap, const cruna_objective *obj,
                        double *J_dev, double *grad_f, double *grad_q0, std::vector<void *> &scratch) {
  GraphScope graphs(c);
  GradientRun g;
  g.c = c;
  g.nsteps = nsteps;
  g.obj = obj;
  g.discrete = c->adjoint_mode == 1;
  // discrete mode reverses the step inputs Q(nsteps-1) .. Q(0); the continuous one Q(nsteps) .. Q(1)
  const int span = g.discrete ? nsteps - 1 : nsteps;
  g.S = std::min(nsnap - 1, std::max(span, 0));
  long long cost = 0;
  build_schedule(span, g.S, g.kbest, cost);
  const size_t bytes = sizeof(double) * (size_t)c->g.N * 5;
  auto alloc = [&](size_t b) {
    void *p = nullptr;
    CRUNA_CUDA_CHECK(cudaMalloc(&p, b));
    scratch.push_back(p);
    return static_cast<double *>(p);
  };
  const bool plane = obj->kind == CRUNA_OBJ_PLANE_P2;
  double *work = alloc(bytes);
  g.work = work;
  g.slots.resize(g.S + 1);
  g.slot_step.assign(g.S + 1, -1);
  g.host_slots = c->snapshot_host;
  for (int i = 0; i <= g.S; ++i) {
    if (g.host_slots) {  // pinning is slow (seconds per state at 768^3): the slots stay on the context
      if ((size_t)i == c->snap_pinned.size()) {
        void *p = nullptr;
        CRUNA_CUDA_CHECK(cudaMallocHost(&p, bytes));
        c->snap_pinned.push_back(p);
      }
      g.slots[i] = static_cast<double *>(c->snap_pinned[i]);
    } else {
      g.slots[i] = alloc(bytes);
    }
  }
  g.qs = alloc(bytes);
  g.gsrc = plane ? alloc(bytes) : nullptr;  // the plane objective's adjoint source
  g.partial = alloc(sizeof(double) * (RG + 1));
  g.J = J_dev;
  g.gf = grad_f;
  CRUNA_CUDA_CHECK(cudaMemsetAsync(g.qs, 0, bytes, c->stream));
  if (plane) CRUNA_CUDA_CHECK(cudaMemsetAsync(g.gsrc, 0, bytes, c->stream));
  CRUNA_CUDA_CHECK(cudaMemsetAsync(J_dev, 0, sizeof(double), c->stream));
  g.direct_step = direct_loop_step;
  g.adjoint_step = adjoint_loop_step;
  if (g.discrete) g.qN = alloc(bytes);
  if (g.host_slots && span > 0) {  // optional, last: without room for it every restart crosses PCIe
    void *p = nullptr;
    if (cudaMalloc(&p, bytes) == cudaSuccess) {
      scratch.push_back(p);
      g.enable_cache(static_cast<double *>(p));
    } else {
      (void)cudaGetLastError();
    }
  }
  g.slot_step[0] = 0;
  g.work = const_cast<double *>(q0);  // q0 is not read after this store (grad_q0 may alias it)
  g.store(0);
  g.work = work;
  if (g.discrete) {
    if (grad_f) CRUNA_CUDA_CHECK(cudaMemsetAsync(grad_f, 0, bytes, c->stream));
    g.rev(0, span, g.S);
    g.adjoint(0, g.at_snapshot(0));
  } else {
    g.rev(0, nsteps, g.S);
  }
  if (grad_q0) copy_state(c, grad_q0, g.qs, 5);
  return g.advanced;
}

// J of the direct loop from q0 alone (calc_direct + calc_objective, cruna.f90:90-117): the line search's
// objective evaluations
double objective_direct_impl(cruna_ctx *c, const double *q0, int nsteps, const cruna_objective *obj,
                             std::vector<void *> &scratch) {
  GraphScope graphs(c);
  auto alloc = [&](size_t b) {
    void *p = nullptr;
    CRUNA_CUDA_CHECK(cudaMalloc(&p, b));
    scratch.push_back(p);
    return static_cast<double *>(p);
  };
  const size_t bytes = sizeof(double) * (size_t)c->g.N * 5;
  const bool plane = obj->kind == CRUNA_OBJ_PLANE_P2;
  double *work = alloc(bytes), *gsrc = plane ? alloc(bytes) : nullptr,
         *partial = alloc(sizeof(double) * (RG + 1)), *J = alloc(sizeof(double));
  CRUNA_CUDA_CHECK(cudaMemsetAsync(J, 0, sizeof(double), c->stream));
  copy_state(c, work, q0, 5);
  const int nd = obj->normal - 1;
  double w = 1.0;
  for (int d = 0; d < 3; ++d)
    if (d != nd && c->cfg.n[d] > 1) w *= c->dx[d];
  for (int nt = 1; nt <= nsteps; ++nt) {
    direct_loop_step(c, work, nt);
    if (plane) {
      k_plane_obj<<<RG, RB, 0, c->stream>>>(c->g, nd, obj->index - 1, w, obj->p_inf, work, gsrc, partial, 1.0);
      CRUNA_LAUNCH_CHECK(c);
      k_sum_partials<<<1, 32, 0, c->stream>>>(partial, RG, J, c->cfg.dt, 1);
      CRUNA_LAUNCH_CHECK(c);
    }
  }
  if (!plane) terminal_objective(c, obj, work, nullptr, partial, J);
  double h = 0.0;
  CRUNA_CUDA_CHECK(cudaMemcpyAsync(&h, J, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
  return h;
}

void axpy_state(cruna_ctx *c, double a, const double *x, double *y) {
  const long long M = c->g.N * 5;
  k_axpy<<<(int)std::min<long long>((M + 255) / 256, 148LL * 32), 256, 0, c->stream>>>(M, a, x, y, 0);
  CRUNA_LAUNCH_CHECK(c);
}

}  // namespace cruna
