// Learned subgrid closure around the solver (no counterpart in the reference: CRUNA has no learned
// component): box filtering of a fine state with the exact subgrid stresses, the closure's features on
// a coarse state, and the closure inside the coarse direct RHS.
//
// Filtering (factor r per direction with more than one point): the coarse value is the mean over the
// r^3 fine points of rho, rho u_i and p; the subgrid stress is the Favre residual
//   tau_ij = mean(rho u_i u_j) - mean(rho u_i) mean(rho u_j) / mean(rho),
// so the filtered momentum equation reads d(rho u_i)/dt + d_j(rho u_i u_j)_resolved + ... = -d_j tau_ij.
// Features (12 per point): du_i/dx_j of the coarse velocity (u_x, u_y, u_z, v_x, ..., w_z, derivatives
// of the solver's own scheme), rho, T, the filter width; or, normalised, du_i/dx_j / g, rho, T, g delta
// with g = |grad u| (Frobenius), and the network's outputs scaled by rho (g delta)^2.  With a closure attached, every direct RHS
// evaluation adds -d_j tau_ij(model) to the momentum equations through the forcing hook (apply_force,
// src/opt/force.f90:27-31), on top of the caller's own forcing.
#include <algorithm>
#include <cmath>

#include "cruna_internal.cuh"
#include "ops_common.cuh"

namespace cruna {

namespace {

__global__ void k_box_filter(Grid fg, Grid cg, int r0, int r1, int r2, const double *__restrict__ q,
                             double *__restrict__ qc, float *__restrict__ tau) {
  const long long Nc = cg.N, Nf = fg.N;
  for (long long pc = blockIdx.x * (long long)blockDim.x + threadIdx.x; pc < Nc;
       pc += (long long)gridDim.x * blockDim.x) {
    const long long ic = pc % cg.n1, jc = (pc / cg.n1) % cg.n2, kc = pc / ((long long)cg.n1 * cg.n2);
    double s[5] = {0, 0, 0, 0, 0}, uu[6] = {0, 0, 0, 0, 0, 0};
    for (int c = 0; c < r2; ++c)
      for (int b = 0; b < r1; ++b)
        for (int a = 0; a < r0; ++a) {
          const long long pf = (ic * r0 + a) + fg.n1 * ((jc * r1 + b) + (long long)fg.n2 * (kc * r2 + c));
          const double rho = q[pf], m0 = q[pf + Nf], m1 = q[pf + 2 * Nf], m2 = q[pf + 3 * Nf];
          s[0] += rho;
          s[1] += m0;
          s[2] += m1;
          s[3] += m2;
          s[4] += q[pf + 4 * Nf];
          const double ir = 1.0 / rho;
          uu[0] += m0 * m0 * ir;
          uu[1] += m1 * m1 * ir;
          uu[2] += m2 * m2 * ir;
          uu[3] += m0 * m1 * ir;
          uu[4] += m0 * m2 * ir;
          uu[5] += m1 * m2 * ir;
        }
    const double inv = 1.0 / (double)(r0 * r1 * r2);
    for (int v = 0; v < 5; ++v) qc[pc + v * Nc] = s[v] * inv;
    const double rb = s[0] * inv, m[3] = {s[1] * inv, s[2] * inv, s[3] * inv};
    const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    for (int t = 0; t < 6; ++t) tau[pc * 6 + t] = (float)(uu[t] * inv - m[ia[t]] * m[ib[t]] / rb);
  }
}

// features from the generic workspace (u, T, grad u) and rho; normalised: grad u / |grad u| and
// |grad u| * delta in place of the raw gradients and the filter width
__global__ void k_features(long long N, const double *__restrict__ q, const double *__restrict__ t, double delta,
                           int norm, float *__restrict__ X) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    float *x = X + p * 12;
    double gr[9], s = 0.0;
    for (int g = 0; g < 9; ++g) {
      gr[g] = t[p + (long long)(F_UX + g) * N];
      s += gr[g] * gr[g];
    }
    const double gm = sqrt(s), inv = gm > 0.0 ? 1.0 / gm : 0.0;
    for (int g = 0; g < 9; ++g) x[g] = (float)(norm ? gr[g] * inv : gr[g]);
    x[9] = (float)q[p];
    x[10] = (float)t[p + (long long)F_T * N];
    x[11] = (float)(norm ? gm * delta : delta);
  }
}

// model stresses (point-major floats) -> six double fields tau_11, tau_22, tau_33, tau_12, tau_13, tau_23;
// normalised outputs are tau / (rho (|grad u| delta)^2), rho and |grad u| delta read back from the features
__global__ void k_tau_fields(long long N, const float *__restrict__ Y, const float *__restrict__ X, int norm,
                             double *__restrict__ tau) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    const double gd = (double)X[p * 12 + 11];
    const double sc = norm ? (double)X[p * 12 + 9] * gd * gd : 1.0;
    for (int t = 0; t < 6; ++t) tau[p + t * N] = (double)Y[p * 6 + t] * sc;
  }
}

// f = user forcing (or 0) with f_{1+i} -= sum_j d_j tau_ij; dtau[i*3 + j] = d_j tau_ij
__global__ void k_closure_force(long long N, const double *__restrict__ user, const double *__restrict__ dtau,
                                double *__restrict__ f) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x) {
    for (int v = 0; v < 5; ++v) f[p + v * N] = user ? user[p + v * N] : 0.0;
    for (int i = 0; i < 3; ++i) {
      const double div = dtau[p + (i * 3 + 0) * N] + dtau[p + (i * 3 + 1) * N] + dtau[p + (i * 3 + 2) * N];
      f[p + (1 + i) * N] -= div;
    }
  }
}

// slot of tau_ij among the six fields (order 11, 22, 33, 12, 13, 23)
int tau_index(int i, int j) {
  if (i == j) return i;
  const int a = std::min(i, j), b = std::max(i, j);
  return a == 0 ? (b == 1 ? 3 : 4) : 5;
}

void features(cruna_ctx *c, const double *q, double delta, float *X) {
  ensure_generic(c);
  generic_forward_gradients(c, q);
  const long long N = c->g.N;
  k_features<<<(int)std::min<long long>(nblocks(N), 148LL * 32), kThreads, 0, c->stream>>>(
      N, q, c->tmp, delta, c->closure_norm ? 1 : 0, X);
  CRUNA_LAUNCH_CHECK(c);
}

void ensure_closure_buffers(cruna_ctx *c) {
  const long long N = c->g.N;
  if (!c->cl_force) c->cl_force = dalloc(c, (size_t)N * 5);
  if (!c->cl_tau) c->cl_tau = dalloc(c, (size_t)N * 15);
  if (!c->cl_x) c->cl_x = reinterpret_cast<float *>(dalloc(c, (size_t)N * 6));  // 12 floats per point
  if (!c->cl_y) c->cl_y = reinterpret_cast<float *>(dalloc(c, (size_t)N * 3));  // 6 floats per point
}

}  // namespace

void closure_stage(cruna_ctx *c, const double *q) {
  if (!c->closure_mlp) return;
  if (closure_in_pass(c)) {                        // pass G adds the model stresses itself
    c->force = c->user_force;
    return;
  }
  const long long N = c->g.N;
  features(c, q, c->closure_delta, c->cl_x);
  mlp_forward_stream(c->closure_mlp, c->cl_x, c->cl_y, N, c->stream);
  const int blocks = (int)std::min<long long>(nblocks(N), 148LL * 32);
  k_tau_fields<<<blocks, kThreads, 0, c->stream>>>(N, c->cl_y, c->cl_x, c->closure_norm ? 1 : 0, c->cl_tau);
  CRUNA_LAUNCH_CHECK(c);
  double *dtau = c->cl_tau + 6 * N;
  for (int j = 0; j < 3; ++j) {  // d_j tau_ij of the three rows in one launch per direction
    if (c->dop[j].kind == OP_ZERO) {
      for (int i = 0; i < 3; ++i)
        CRUNA_CUDA_CHECK(cudaMemsetAsync(dtau + (i * 3 + j) * N, 0, sizeof(double) * N, c->stream));
      continue;
    }
    FieldSet fs;
    for (int i = 0; i < 3; ++i) fs.add(c->cl_tau + tau_index(i, j) * N, nullptr, dtau + (i * 3 + j) * N);
    apply_diff_set(c, j, fs, c->dx[j]);
  }
  k_closure_force<<<blocks, kThreads, 0, c->stream>>>(N, c->user_force, dtau, c->cl_force);
  CRUNA_LAUNCH_CHECK(c);
  c->force = c->cl_force;
}

}  // namespace cruna

using namespace cruna;

namespace {
template <class F>
int closure_guard(cruna_ctx *c, F &&f) {
  if (!c) return CRUNA_ERR_ARG;
  try {
    CRUNA_CUDA_CHECK(cudaSetDevice(c->device));
    return f();
  } catch (const ApiError &e) {
    c->err = e.msg;
    return e.code;
  } catch (const std::exception &e) {
    c->err = e.what();
    return CRUNA_ERR_CUDA;
  }
}
}  // namespace

extern "C" {

int cruna_box_filter_dev(cruna_ctx *c, int factor, const double *q, double *q_coarse, float *tau) {
  return closure_guard(c, [&]() -> int {
    if (!q || !q_coarse || !tau || factor < 1) throw ApiError{CRUNA_ERR_ARG, "bad box-filter arguments"};
    int r[3], nc[3];
    for (int d = 0; d < 3; ++d) {
      r[d] = c->cfg.n[d] > 1 ? factor : 1;
      if (c->cfg.n[d] % r[d] != 0) throw ApiError{CRUNA_ERR_ARG, "grid not divisible by the filter factor"};
      nc[d] = c->cfg.n[d] / r[d];
    }
    Grid cg{nc[0], nc[1], nc[2], (long long)nc[0] * nc[1] * nc[2]};
    k_box_filter<<<(int)std::min<long long>(nblocks(cg.N), 148LL * 32), kThreads, 0, c->stream>>>(
        c->g, cg, r[0], r[1], r[2], q, q_coarse, tau);
    CRUNA_LAUNCH_CHECK(c);
    return CRUNA_OK;
  });
}

int cruna_closure_features_dev(cruna_ctx *c, const double *q, double delta, float *X) {
  return closure_guard(c, [&]() -> int {
    if (!q || !X) throw ApiError{CRUNA_ERR_ARG, "null pointer"};
    features(c, q, delta, X);
    return CRUNA_OK;
  });
}

int cruna_set_closure_fused(cruna_ctx *c, int on) {
  return closure_guard(c, [&]() -> int {
    c->closure_fused = on != 0;                    // closure_stage picks the forcing before each RHS
    return CRUNA_OK;
  });
}

int cruna_set_closure_normalisation(cruna_ctx *c, int on) {
  return closure_guard(c, [&]() -> int {
    c->closure_norm = on != 0;
    return CRUNA_OK;
  });
}

int cruna_set_closure(cruna_ctx *c, cruna_mlp *mlp, double delta) {
  return closure_guard(c, [&]() -> int {
    if (mlp && !(delta > 0.0)) throw ApiError{CRUNA_ERR_ARG, "filter width must be positive"};
    if (mlp && c->adjoint_mode == 1)
      throw ApiError{CRUNA_ERR_UNSUPPORTED, "the discrete adjoint does not transpose the closure"};
    if (mlp && !c->closure_mlp) {
      ensure_closure_buffers(c);
      c->user_force = c->force;
    } else if (!mlp && c->closure_mlp) {
      c->force = c->user_force;
      c->user_force = nullptr;
    }
    c->closure_mlp = mlp;
    c->closure_delta = delta;
    return CRUNA_OK;
  });
}

}  // extern "C"
