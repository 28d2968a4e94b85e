// extern "C" entry points of the CRUNA B200 library (declared in include/cruna_b200.h).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

#include "cruna_internal.cuh"

using namespace cruna;

namespace cruna {

double *dalloc(cruna_ctx *c, size_t count) {
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, count * sizeof(double));
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw ApiError{CRUNA_ERR_NOMEM, std::string("cudaMalloc of ") + std::to_string(count * 8) +
                                        " bytes failed: " + cudaGetErrorString(e)};
  }
  c->allocations.push_back(p);
  return static_cast<double *>(p);
}

void ensure_generic(cruna_ctx *c) {
  if (!c->tmp) c->tmp = dalloc(c, (size_t)c->g.N * 60);
}

bool use_fused(const cruna_ctx *c) { return c->fused_ok && !c->force_generic; }

// z-slab mode: let the caller refresh the halo planes of `nfields` fields before a z-reading pass
void halo(cruna_ctx *c, const double *f, int nfields) {
  if (!c->halo_fn) return;
  if (c->halo_fn(c->halo_user, const_cast<double *>(f), nfields, (void *)c->stream) != 0)
    throw ApiError{CRUNA_ERR_CUDA, "halo exchange callback failed"};
}

}  // namespace cruna

namespace {

thread_local std::string g_init_error;

struct Status {
  int code;
};

template <class F>
int guarded(cruna_ctx *c, F &&f) {
  if (!c) return CRUNA_ERR_ARG;
  try {
    CRUNA_CUDA_CHECK(cudaSetDevice(c->device));
    int rc = f();
    return rc;
  } catch (const Status &s) {
    return s.code;
  } catch (const ApiError &e) {
    c->err = e.msg;
    return e.code;
  } catch (const std::bad_alloc &) {
    c->err = "host allocation failed";
    return CRUNA_ERR_NOMEM;
  } catch (const std::exception &e) {
    c->err = e.what();
    return CRUNA_ERR_CUDA;
  }
}

[[noreturn]] void fail(cruna_ctx *c, int code, const std::string &msg) {
  c->err = msg;
  throw Status{code};
}

template <class T>
T *upload(cruna_ctx *c, const std::vector<T> &v) {
  if (v.empty()) return nullptr;
  void *p = nullptr;
  CRUNA_CUDA_CHECK(cudaMalloc(&p, v.size() * sizeof(T)));
  c->allocations.push_back(p);
  CRUNA_CUDA_CHECK(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return static_cast<T *>(p);
}

void attach_factors(cruna_ctx *c, LineOp &op, const HostFactors &hf) {
  if (!op.solve) return;
  std::vector<double> inv(hf.d.size());
  for (size_t i = 0; i < hf.d.size(); ++i) inv[i] = 1.0 / hf.d[i];
  op.dl = upload(c, hf.dl);
  op.inv_d = upload(c, inv);
  op.du = upload(c, hf.du);
  op.du2 = upload(c, hf.du2);
  op.ipiv = upload(c, hf.ipiv);
  op.nopiv = 1;
  for (size_t i = 0; i + 1 < hf.ipiv.size(); ++i)
    if (hf.ipiv[i] != (int)i + 1) op.nopiv = 0;
  if (op.cyclic) {
    op.fbnorm = upload(c, hf.fbnorm);
    op.fbrat = hf.fbrat;
  }
}

long long N5(const cruna_ctx *c) { return c->g.N * 5; }

double *stage_in(cruna_ctx *c, int slot, const double *host, int nfields) {
  if (!c->io[slot]) c->io[slot] = dalloc(c, (size_t)N5(c));
  if (host)
    CRUNA_CUDA_CHECK(cudaMemcpyAsync(c->io[slot], host, sizeof(double) * c->g.N * nfields,
                                     cudaMemcpyHostToDevice, c->stream));
  return c->io[slot];
}

// grad_f of the host-pointer VJP entry points has its own buffer: io[3] may hold the forcing
double *stage_gf(cruna_ctx *c, const double *host) {
  if (!c->vjp_gf) c->vjp_gf = dalloc(c, (size_t)N5(c));
  CRUNA_CUDA_CHECK(cudaMemcpyAsync(c->vjp_gf, host, sizeof(double) * N5(c), cudaMemcpyHostToDevice, c->stream));
  return c->vjp_gf;
}

void stage_out(cruna_ctx *c, double *host, const double *dev, int nfields) {
  CRUNA_CUDA_CHECK(cudaMemcpyAsync(host, dev, sizeof(double) * c->g.N * nfields, cudaMemcpyDeviceToHost,
                                   c->stream));
  CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
}

// the reference state buffer (zeros until cruna_set_reference)
void ensure_reference(cruna_ctx *c) {
  if (c->qref) return;
  c->qref = dalloc(c, (size_t)N5(c));
  CRUNA_CUDA_CHECK(cudaMemsetAsync(c->qref, 0, sizeof(double) * N5(c), c->stream));
}

// the RHS buffer st[0]: the generic path's RHS and the fused path's RHS before RHS boundary conditions
double *rhs_buffer(cruna_ctx *c) {
  if (!c->st[0]) c->st[0] = dalloc(c, (size_t)N5(c));
  return c->st[0];
}

// time_stepper_direct (rk_o4_e.f90:17-58): q1 may alias q0
void step_direct(cruna_ctx *c, const double *q0, double *q1) {
  double *k = (use_fused(c) && !c->has_rhs_bc) ? nullptr : rhs_buffer(c);
  double *acc = c->st[1], *qa = c->st[2], *qb = c->st[3], *qbc = c->st[4];
  const double dt = c->cfg.dt;
  if (use_fused(c)) {
    halo(c, q0, 5);
    closure_stage(c, q0);
    rhs_direct_fused(c, q0, k, 1, q0, acc, qa, dt);
    halo(c, qa, 5);
    closure_stage(c, qa);
    rhs_direct_fused(c, qa, k, 2, q0, acc, qb, dt);
    halo(c, qb, 5);
    closure_stage(c, qb);
    rhs_direct_fused(c, qb, k, 3, q0, acc, qa, dt);
    halo(c, qa, 5);
    closure_stage(c, qa);
    rhs_direct_fused(c, qa, k, 4, q0, acc, q1, dt);
    return;
  }
  ensure_generic(c);
  halo(c, q0, 5);
  closure_stage(c, q0);
  rhs_direct_generic(c, q0, k, qbc);
  rk_stage(c, 1, dt, k, q0, acc, qa);
  halo(c, qa, 5);
  closure_stage(c, qa);
  rhs_direct_generic(c, qa, k, qbc);
  rk_stage(c, 2, dt, k, q0, acc, qb);
  halo(c, qb, 5);
  closure_stage(c, qb);
  rhs_direct_generic(c, qb, k, qbc);
  rk_stage(c, 3, dt, k, q0, acc, qa);
  halo(c, qa, 5);
  closure_stage(c, qa);
  rhs_direct_generic(c, qa, k, qbc);
  rk_stage(c, 4, dt, k, q0, acc, q1);
}

// time_stepper_adjoint (rk_o4_e.f90:62-105): dt -> -dt, q0 frozen; qs1 may alias qs0
void step_adjoint(cruna_ctx *c, const double *qs0, const double *q0, const double *g, double *qs1) {
  double *k = (use_fused(c) && !c->has_rhs_bc) ? nullptr : rhs_buffer(c);
  double *acc = c->st[1], *qa = c->st[2], *qb = c->st[3], *qbc = c->st[4];
  const double dt = -c->cfg.dt;
  halo(c, q0, 5);
  if (use_fused(c)) {
    halo(c, qs0, 5);
    rhs_adjoint_fused(c, qs0, q0, g, k, 1, qs0, acc, qa, dt);
    halo(c, qa, 5);
    rhs_adjoint_fused(c, qa, q0, g, k, 2, qs0, acc, qb, dt);
    halo(c, qb, 5);
    rhs_adjoint_fused(c, qb, q0, g, k, 3, qs0, acc, qa, dt);
    halo(c, qa, 5);
    rhs_adjoint_fused(c, qa, q0, g, k, 4, qs0, acc, qs1, dt);
    return;
  }
  ensure_generic(c);
  halo(c, qs0, 5);
  rhs_adjoint_generic(c, qs0, q0, g, k, qbc);
  rk_stage(c, 1, dt, k, qs0, acc, qa);
  halo(c, qa, 5);
  rhs_adjoint_generic(c, qa, q0, g, k, qbc);
  rk_stage(c, 2, dt, k, qs0, acc, qb);
  halo(c, qb, 5);
  rhs_adjoint_generic(c, qb, q0, g, k, qbc);
  rk_stage(c, 3, dt, k, qs0, acc, qa);
  halo(c, qa, 5);
  rhs_adjoint_generic(c, qa, q0, g, k, qbc);
  rk_stage(c, 4, dt, k, qs0, acc, qs1);
}

bool due(int freq, int nt) { return freq > 0 && nt % freq == 0; }

void check_or_fail(cruna_ctx *c, const double *q, int nt) {
  int f = check_state(c, q);
  if (f) {
    std::string what;
    if (f & 1) what += " non-finite value;";
    if (f & 2) what += " rho <= 0;";
    if (f & 4) what += " p <= 0;";
    fail(c, CRUNA_ERR_STATE, "state check failed after step " + std::to_string(nt) + ":" + what);
  }
}

int dir_index(cruna_ctx *c, int dir) {
  if (dir < 1 || dir > 3) fail(c, CRUNA_ERR_ARG, "dir must be 1, 2 or 3");
  return dir - 1;
}

}  // namespace

namespace cruna {

int prof_begin(cruna_ctx *c, const char *name) {
  if (!c->prof_on) return -1;
  auto take = [&]() {
    cudaEvent_t e;
    if (!c->prof_pool.empty()) {
      e = c->prof_pool.back();
      c->prof_pool.pop_back();
    } else {
      CRUNA_CUDA_CHECK(cudaEventCreate(&e));
    }
    return e;
  };
  if (c->prof_pending.size() >= 4096) prof_drain(c);
  cudaEvent_t a = take(), b = take();
  CRUNA_CUDA_CHECK(cudaEventRecord(a, c->stream));
  c->prof_pending.push_back({name, a, b});
  return (int)c->prof_pending.size() - 1;
}

void prof_end(cruna_ctx *c, int idx) {
  if (idx < 0 || idx >= (int)c->prof_pending.size()) return;
  cudaEventRecord(c->prof_pending[idx].b, c->stream);
}

void prof_drain(cruna_ctx *c) {
  if (c->prof_pending.empty()) return;
  CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
  for (auto &e : c->prof_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) {
      auto &acc = c->prof_acc[e.name];
      acc.first += 1;
      acc.second += ms;
    } else {
      cudaGetLastError();
    }
    c->prof_pool.push_back(e.a);
    c->prof_pool.push_back(e.b);
  }
  c->prof_pending.clear();
}

}  // namespace cruna

extern "C" {

void cruna_config_defaults(cruna_config *cfg) {
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->abi_version = CRUNA_ABI_VERSION;
  for (int d = 0; d < 3; ++d) {
    cfg->n[d] = 1;
    cfg->x0[d] = 0.0;
    cfg->x1[d] = 1.0;            // geom.x11 default (grid_transform.f90:34-36)
    cfg->diff[d] = CRUNA_DIFF_O4_E_C_P;
    cfg->filter[d] = CRUNA_FILTER_EMPTY;
    cfg->di_freq[d] = 0;
    cfg->ai_freq[d] = 0;
    cfg->sponge_length[d] = 0.3; // shape_functions.f90:98-100
  }
  cfg->filter_alpha = 0.35;      // filter_pen_core_o10_i_c_o.f90:179
  cfg->filter_strength = 0.2;
  cfg->gamma = 1.4;
  cfg->R = 8.3144598;            // parameter.f90:160
  cfg->W = 0.0289647;            // ns_rho_rhou_p_trafos.f90:24
  cfg->mu0 = 0.0;
  cfg->T0 = 273.0;               // ns_rho_rhou_p_trafos.f90:133
  cfg->Pr = 0.71;                // ns_rho_rhou_p_trafos.f90:159
  cfg->dt = 1e-3;
  cfg->heat_flux_dx = 0;
  cfg->precision = CRUNA_FP64;
  cfg->sponge_amplitude = 1.0;   // shape_functions.f90:102
  cfg->sponge_shape = 0;
  cfg->device = 0;
  cfg->check_every = 0;
}

}  // extern "C"

namespace cruna {
void set_global_error(const std::string &msg) { g_init_error = msg; }
}  // namespace cruna

extern "C" {

const char *cruna_last_error(const cruna_ctx *ctx) {
  return ctx ? ctx->err.c_str() : g_init_error.c_str();
}

int cruna_init(const cruna_config *cfg, const double *bc_table, int nbc, cruna_ctx **out) {
  if (!cfg || !out) {
    g_init_error = "null argument";
    return CRUNA_ERR_ARG;
  }
  *out = nullptr;
  if (cfg->abi_version != CRUNA_ABI_VERSION) {
    g_init_error = "cruna_config.abi_version mismatch";
    return CRUNA_ERR_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    g_init_error = "no CUDA device available";
    return CRUNA_ERR_NODEVICE;
  }
  cruna_ctx *c = new cruna_ctx();
  c->cfg = *cfg;
  c->device = cfg->device;
  int rc = guarded(c, [&]() -> int {
    for (int d = 0; d < 3; ++d)
      if (cfg->n[d] < 1) fail(c, CRUNA_ERR_ARG, "geom.n must be >= 1");
    if (cfg->precision != CRUNA_FP64 && cfg->precision != CRUNA_FP32_STENCIL)
      fail(c, CRUNA_ERR_ARG, "unknown precision");
    if (!(cfg->gamma > 1.0)) fail(c, CRUNA_ERR_ARG, "material.gamma must be > 1");
    if (!(cfg->R > 0.0) || !(cfg->W > 0.0) || !(cfg->T0 > 0.0) || !(cfg->Pr > 0.0))
      fail(c, CRUNA_ERR_ARG, "material.R, W, T0 and Pr must be positive");
    c->g = Grid{cfg->n[0], cfg->n[1], cfg->n[2], (long long)cfg->n[0] * cfg->n[1] * cfg->n[2]};
    CRUNA_CUDA_CHECK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    // dx rule: periodic dx = L/n, open dx = L/(n-1) (grid_transform.f90:40-56)
    for (int d = 0; d < 3; ++d) {
      const double L = cfg->x1[d] - cfg->x0[d];
      const int m = diff_is_periodic(cfg->diff[d]) ? cfg->n[d] : cfg->n[d] - 1;
      c->dx[d] = m > 0 ? L / m : INFINITY;
    }
    for (int d = 0; d < 3; ++d) {
      std::string err;
      HostFactors hf;
      if (!build_diff_op(cfg->diff[d], cfg->n[d], c->dop[d], hf, err))
        fail(c, CRUNA_ERR_ARG, "direction " + std::to_string(d + 1) + ": " + err);
      attach_factors(c, c->dop[d], hf);
      c->dhf[d] = hf;
      HostFactors hf2;
      if (!build_filter_op(cfg->filter[d], cfg->n[d], cfg->filter_alpha, cfg->filter_strength, c->fop[d],
                           hf2, err))
        fail(c, CRUNA_ERR_ARG, "direction " + std::to_string(d + 1) + ": " + err);
      attach_factors(c, c->fop[d], hf2);
      c->fhf[d] = hf2;
    }
    // boundary table (boundary_conditions.f90:461-610: inf -> n, clamp to the block)
    if (nbc < 0 || (nbc > 0 && !bc_table)) fail(c, CRUNA_ERR_ARG, "bad boundary table");
    for (int i = 0; i < nbc; ++i) {
      const double *r = bc_table + 10 * i;
      BCRow b{};
      b.type = (int)std::lround(r[0]);
      int lo[3], hi[3];
      for (int d = 0; d < 3; ++d) {
        double a = r[1 + 2 * d], e = r[2 + 2 * d];
        if (std::isinf(a)) a = cfg->n[d];
        if (std::isinf(e)) e = cfg->n[d];
        lo[d] = (int)std::lround(a);
        hi[d] = (int)std::lround(e);
      }
      bool member = true;
      for (int d = 0; d < 3; ++d)
        if (lo[d] > cfg->n[d] || hi[d] < 1) member = false;
      if (!member || b.type == 0) continue;
      for (int d = 0; d < 3; ++d) {
        lo[d] = std::max(lo[d], 1);
        hi[d] = std::min(hi[d], cfg->n[d]);
        if (lo[d] > hi[d]) fail(c, CRUNA_ERR_ARG, "empty boundary box in row " + std::to_string(i + 1));
      }
      b.is = lo[0] - 1; b.ie = hi[0] - 1; b.js = lo[1] - 1; b.je = hi[1] - 1; b.ks = lo[2] - 1; b.ke = hi[2] - 1;
      for (int d = 0; d < 3; ++d) b.k[d] = r[7 + d];
      b.comp = (int)std::lround(r[7]) - 1;
      switch (b.type) {
        case 100:
          if (b.comp < 0 || b.comp > 4) fail(c, CRUNA_ERR_ARG, "wall component must be 1..5");
          c->has_rhs_bc = true;
          break;
        case 200: {
          // characteristic_zero_grad_init (nonreflecting.f90:665-728)
          double nrm = std::sqrt(b.k[0] * b.k[0] + b.k[1] * b.k[1] + b.k[2] * b.k[2]);
          if (!(nrm > 0)) fail(c, CRUNA_ERR_ARG, "type 200 needs a non-zero k-vector");
          int lo2[3] = {b.is, b.js, b.ks}, hi2[3] = {b.ie, b.je, b.ke};
          for (int d = 0; d < 3; ++d) {
            double kd = b.k[d] / nrm;
            b.shift[d] = kd > 0 ? -1 : (kd < 0 ? 1 : 0);
            if (lo2[d] + b.shift[d] < 0 || hi2[d] + b.shift[d] >= cfg->n[d])
              fail(c, CRUNA_ERR_ARG, "type 200: inner neighbour outside the block");
          }
          c->has_q_bc = true;
          c->has_nonlocal_bc = true;
          break;
        }
        case 201:
          c->has_q_bc = true;
          break;
        case 204:
          c->has_rhs_bc = true;
          c->has_nonlocal_bc = true;
          break;
        case 400:
          c->has_rhs_bc = true;
          c->has_sponge = true;
          break;
        case 401:
          c->has_q_bc = true;
          c->has_sponge = true;
          break;
        case 202:  // characteristic on q with the normal-vector field, on the row's box
        case 203:  // zonal: the whole block, weighted by the sponge shape (boundary_conditions.f90:93-107)
        case 205:  // as 202 on the RHS
        case 206:  // as 203 on the RHS
          if (b.type == 203 || b.type == 206) {
            b.is = 0; b.ie = cfg->n[0] - 1; b.js = 0; b.je = cfg->n[1] - 1; b.ks = 0; b.ke = cfg->n[2] - 1;
            b.only = b.type == 203 ? (int)std::lround(r[7]) : 0;  // -1 outside_rhs_only, 1 inside_rhs_only
          }
          if (cfg->kvector < 0 || cfg->kvector > 2) fail(c, CRUNA_ERR_ARG, "kvector must be 0, 1 or 2");
          if (b.type <= 203) c->has_q_bc = true;
          else c->has_rhs_bc = true;
          if (!c->kvec) c->kvec = dalloc(c, (size_t)c->g.N * 3);
          break;
        default:
          fail(c, CRUNA_ERR_UNSUPPORTED, "boundary type " + std::to_string(b.type) +
                                             " is not available (supported: 0,100,200-206,400,401)");
      }
      c->bc.push_back(b);
    }
    // sponge shape factors (shape_functions.f90:69-150) as 1-D vectors
    {
      std::vector<double> f[3][2];
      for (int d = 0; d < 3; ++d) {
        const int n = cfg->n[d];
        f[d][0].assign(n, 1.0);
        f[d][1].assign(n, 1.0);
        const double L = cfg->sponge_length[d];
        if (!(L > 0.0)) continue;
        const double pi = 4.0 * std::atan(1.0);
        for (int i = 0; i < n; ++i) {
          const double x = (n > 1 ? (double)i * c->dx[d] : 0.0) + cfg->x0[d];
          auto fct = [&](double x0) {
            return cfg->sponge_shape == 0 ? 1.0 - ((x - x0) / L) * ((x - x0) / L)
                                          : 0.5 + 0.5 * std::cos((x - x0) * (pi / L));
          };
          double x0 = cfg->x0[d] + L;
          f[d][0][i] = x > x0 ? 1.0 : fct(x0);
          x0 = cfg->x1[d] - L;
          f[d][1][i] = x < x0 ? 1.0 : fct(x0);
        }
      }
      std::vector<double> sx(cfg->n[0]);
      for (int i = 0; i < cfg->n[0]; ++i) sx[i] = f[0][0][i] * f[0][1][i];
      c->sponge.sx = upload(c, sx);
      c->sponge.sym = upload(c, f[1][0]);
      c->sponge.syp = upload(c, f[1][1]);
      c->sponge.szm = upload(c, f[2][0]);
      c->sponge.szp = upload(c, f[2][1]);
      c->sponge.amp = cfg->sponge_amplitude;
    }
    if (c->kvec) build_kvector(c);
    // reference state (zero until cruna_set_reference), only where a boundary type reads it
    bool needs_ref = false;
    for (const BCRow &r : c->bc) needs_ref = needs_ref || (r.type >= 201 && r.type <= 206) || r.type >= 400;
    if (needs_ref) ensure_reference(c);
    // stage buffers: acc, two stage inputs and the step output always; the RHS buffer st[0] and the
    // BC copy st[4] on first use (the fused passes without RHS boundary conditions need neither)
    for (int i : {1, 2, 3, 5}) c->st[i] = dalloc(c, (size_t)N5(c));
    if (c->has_q_bc) c->st[4] = dalloc(c, (size_t)N5(c));
    void *fl = nullptr;
    CRUNA_CUDA_CHECK(cudaMalloc(&fl, sizeof(int) * 4));
    c->allocations.push_back(fl);
    c->flag = static_cast<int *>(fl);  // [0] state check, [1] a kernel's bounded wait ran out
    CRUNA_CUDA_CHECK(cudaMemsetAsync(fl, 0, sizeof(int) * 4, c->stream));
    c->fused_ok = fused_supported(c);
    c->filter_fused_ok = filter_fused_supported(c);
    CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    return CRUNA_OK;
  });
  if (rc != CRUNA_OK) {
    g_init_error = c->err;
    cruna_free(c);
    return rc;
  }
  *out = c;
  return CRUNA_OK;
}

int cruna_profile_enable(cruna_ctx *c, int on) {
  return guarded(c, [&]() -> int {
    if (!on) prof_drain(c);
    c->prof_on = on != 0;
    if (on) c->prof_acc.clear();
    return CRUNA_OK;
  });
}

int cruna_profile_report(cruna_ctx *c, char *buf, int buflen) {
  return guarded(c, [&]() -> int {
    prof_drain(c);
    std::string out;
    for (auto &kv : c->prof_acc)
      out += kv.first + " " + std::to_string(kv.second.first) + " " + std::to_string(kv.second.second) + "\n";
    if (buf && buflen > 0) {
      std::strncpy(buf, out.c_str(), (size_t)buflen - 1);
      buf[buflen - 1] = 0;
    }
    return (int)out.size();
  });
}

void cruna_free(cruna_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto &e : c->prof_pending) {
    cudaEventDestroy(e.a);
    cudaEventDestroy(e.b);
  }
  for (auto e : c->prof_pool) cudaEventDestroy(e);
  for (void *p : c->allocations) cudaFree(p);
  for (void *p : c->snap_pinned) cudaFreeHost(p);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int cruna_sync(cruna_ctx *c) {
  return guarded(c, [&]() -> int {
    CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    int waited = 0;
    CRUNA_CUDA_CHECK(cudaMemcpy(&waited, c->flag + 1, sizeof(int), cudaMemcpyDeviceToHost));
    if (waited) {
      CRUNA_CUDA_CHECK(cudaMemset(c->flag + 1, 0, sizeof(int)));
      fail(c, CRUNA_ERR_CUDA, "a kernel's bounded wait for its shared-memory copies ran out");
    }
    return CRUNA_OK;
  });
}

int cruna_get_dx(const cruna_ctx *c, double dx[3]) {
  if (!c || !dx) return CRUNA_ERR_ARG;
  for (int d = 0; d < 3; ++d) dx[d] = c->dx[d];
  return CRUNA_OK;
}

void *cruna_stream(cruna_ctx *c) { return c ? (void *)c->stream : nullptr; }

int cruna_rhs_path(const cruna_ctx *c) { return c ? (use_fused(c) ? 1 : 0) : CRUNA_ERR_ARG; }

int cruna_set_force_generic(cruna_ctx *c, int v) {
  if (!c) return CRUNA_ERR_ARG;
  c->force_generic = v != 0;
  return CRUNA_OK;
}

int cruna_set_tma_passes(cruna_ctx *c, int on) {
  if (!c) return CRUNA_ERR_ARG;
  c->tma_fused = on != 0;
  return CRUNA_OK;
}

int64_t cruna_kernel_launches(const cruna_ctx *c) { return c ? c->launches : -1; }

int cruna_set_reference_dev(cruna_ctx *c, const double *qref) {
  return guarded(c, [&]() -> int {
    if (!qref) fail(c, CRUNA_ERR_ARG, "qref is null");
    ensure_reference(c);
    copy_state(c, c->qref, qref, 5);
    return CRUNA_OK;
  });
}

int cruna_set_reference(cruna_ctx *c, const double *qref) {
  return guarded(c, [&]() -> int {
    if (!qref) fail(c, CRUNA_ERR_ARG, "qref is null");
    ensure_reference(c);
    CRUNA_CUDA_CHECK(cudaMemcpyAsync(c->qref, qref, sizeof(double) * N5(c), cudaMemcpyHostToDevice, c->stream));
    CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    return CRUNA_OK;
  });
}

// the forcing the kernels add: the caller's, or (with a closure) the closure's buffer, which adds it
static void point_forcing(cruna_ctx *c, double *user) {
  if (c->closure_mlp) c->user_force = user;
  else c->force = user;
}

int cruna_set_forcing_dev(cruna_ctx *c, const double *f) {
  return guarded(c, [&]() -> int {
    if (!f) {
      point_forcing(c, nullptr);
      return CRUNA_OK;
    }
    if (!c->io[3]) c->io[3] = dalloc(c, (size_t)N5(c));
    copy_state(c, c->io[3], f, 5);
    point_forcing(c, c->io[3]);
    return CRUNA_OK;
  });
}

int cruna_set_forcing(cruna_ctx *c, const double *f) {
  return guarded(c, [&]() -> int {
    if (!f) {
      point_forcing(c, nullptr);
      return CRUNA_OK;
    }
    if (!c->io[3]) c->io[3] = dalloc(c, (size_t)N5(c));
    CRUNA_CUDA_CHECK(cudaMemcpyAsync(c->io[3], f, sizeof(double) * N5(c), cudaMemcpyHostToDevice, c->stream));
    CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
    point_forcing(c, c->io[3]);
    return CRUNA_OK;
  });
}

int cruna_diff_dev(cruna_ctx *c, int dir, const double *in, double *out, int nfields, double h) {
  return guarded(c, [&]() -> int {
    const int d = dir_index(c, dir);
    if (!in || !out || nfields < 1) fail(c, CRUNA_ERR_ARG, "bad arguments to cruna_diff");
    if (in == out) fail(c, CRUNA_ERR_ARG, "cruna_diff does not work in place");
    const double hh = (std::isnan(h) || h <= 0.0) ? 1.0 : h;
    apply_diff(c, d, in, nullptr, out, hh, nfields);
    return CRUNA_OK;
  });
}

int cruna_diff(cruna_ctx *c, int dir, const double *in, double *out, int nfields, double h) {
  return guarded(c, [&]() -> int {
    const int d = dir_index(c, dir);
    if (!in || !out || nfields < 1 || nfields > 5) fail(c, CRUNA_ERR_ARG, "bad arguments to cruna_diff");
    const double hh = (std::isnan(h) || h <= 0.0) ? 1.0 : h;
    double *din = stage_in(c, 0, in, nfields);
    double *dout = stage_in(c, 1, nullptr, nfields);
    apply_diff(c, d, din, nullptr, dout, hh, nfields);
    stage_out(c, out, dout, nfields);
    return CRUNA_OK;
  });
}

int cruna_filter_dev(cruna_ctx *c, int dir, double *q, int nfields) {
  return guarded(c, [&]() -> int {
    const int d = dir_index(c, dir);
    if (!q || nfields < 1 || nfields > 5) fail(c, CRUNA_ERR_ARG, "bad arguments to cruna_filter");
    apply_filter(c, d, q, c->st[5], nfields);
    return CRUNA_OK;
  });
}

int cruna_filter(cruna_ctx *c, int dir, double *q, int nfields) {
  return guarded(c, [&]() -> int {
    const int d = dir_index(c, dir);
    if (!q || nfields < 1 || nfields > 5) fail(c, CRUNA_ERR_ARG, "bad arguments to cruna_filter");
    double *dq = stage_in(c, 0, q, nfields);
    apply_filter(c, d, dq, c->st[5], nfields);
    stage_out(c, q, dq, nfields);
    return CRUNA_OK;
  });
}

int cruna_rhs_direct_dev(cruna_ctx *c, const double *q, double *rhs, double /*t*/) {
  return guarded(c, [&]() -> int {
    if (!q || !rhs) fail(c, CRUNA_ERR_ARG, "null pointer");
    closure_stage(c, q);
    if (use_fused(c)) {
      rhs_direct_fused(c, q, rhs, 0, nullptr, nullptr, nullptr, 0.0);
    } else {
      ensure_generic(c);
      rhs_direct_generic(c, q, rhs, c->st[4]);
    }
    return CRUNA_OK;
  });
}

int cruna_rhs_direct(cruna_ctx *c, const double *q, double *rhs, double t) {
  return guarded(c, [&]() -> int {
    if (!q || !rhs) fail(c, CRUNA_ERR_ARG, "null pointer");
    double *dq = stage_in(c, 0, q, 5);
    double *dr = stage_in(c, 1, nullptr, 5);
    int rc = cruna_rhs_direct_dev(c, dq, dr, t);
    if (rc) return rc;
    stage_out(c, rhs, dr, 5);
    return CRUNA_OK;
  });
}

int cruna_rhs_adjoint_dev(cruna_ctx *c, const double *qs, const double *q, const double *g, double *rhs,
                          double /*t*/) {
  return guarded(c, [&]() -> int {
    if (!qs || !q || !rhs) fail(c, CRUNA_ERR_ARG, "null pointer");
    if (use_fused(c)) {
      rhs_adjoint_fused(c, qs, q, g, rhs, 0, nullptr, nullptr, nullptr, 0.0);
    } else {
      ensure_generic(c);
      rhs_adjoint_generic(c, qs, q, g, rhs, c->st[4]);
    }
    return CRUNA_OK;
  });
}

int cruna_rhs_adjoint(cruna_ctx *c, const double *qs, const double *q, const double *g, double *rhs,
                      double t) {
  return guarded(c, [&]() -> int {
    if (!qs || !q || !rhs) fail(c, CRUNA_ERR_ARG, "null pointer");
    double *dqs = stage_in(c, 0, qs, 5);
    double *dq = stage_in(c, 1, q, 5);
    double *dg = g ? stage_in(c, 2, g, 5) : nullptr;
    double *dr = c->st[5];
    int rc = cruna_rhs_adjoint_dev(c, dqs, dq, dg, dr, t);
    if (rc) return rc;
    stage_out(c, rhs, dr, 5);
    return CRUNA_OK;
  });
}

int cruna_step_direct_dev(cruna_ctx *c, const double *q0, double *q1, double /*t*/) {
  return guarded(c, [&]() -> int {
    if (!q0 || !q1) fail(c, CRUNA_ERR_ARG, "null pointer");
    step_direct(c, q0, q1);
    return CRUNA_OK;
  });
}

int cruna_step_direct(cruna_ctx *c, const double *q0, double *q1, double t) {
  return guarded(c, [&]() -> int {
    if (!q0 || !q1) fail(c, CRUNA_ERR_ARG, "null pointer");
    double *dq = stage_in(c, 0, q0, 5);
    step_direct(c, dq, dq);
    stage_out(c, q1, dq, 5);
    (void)t;
    return CRUNA_OK;
  });
}

int cruna_step_adjoint_dev(cruna_ctx *c, const double *qs0, const double *q0, const double *g, double *qs1,
                           double /*t*/) {
  return guarded(c, [&]() -> int {
    if (!qs0 || !q0 || !qs1) fail(c, CRUNA_ERR_ARG, "null pointer");
    step_adjoint(c, qs0, q0, g, qs1);
    return CRUNA_OK;
  });
}

int cruna_step_adjoint(cruna_ctx *c, const double *qs0, const double *q0, const double *g, double *qs1,
                       double t) {
  return guarded(c, [&]() -> int {
    if (!qs0 || !q0 || !qs1) fail(c, CRUNA_ERR_ARG, "null pointer");
    double *dqs = stage_in(c, 0, qs0, 5);
    double *dq = stage_in(c, 1, q0, 5);
    double *dg = g ? stage_in(c, 2, g, 5) : nullptr;
    step_adjoint(c, dqs, dq, dg, dqs);
    stage_out(c, qs1, dqs, 5);
    (void)t;
    return CRUNA_OK;
  });
}

int cruna_bc_q_dev(cruna_ctx *c, double *q, int outside) {
  return guarded(c, [&]() -> int {
    if (!q) fail(c, CRUNA_ERR_ARG, "null pointer");
    bc_q(c, q, outside);
    return CRUNA_OK;
  });
}
int cruna_bc_qs_dev(cruna_ctx *c, double *qs, const double *q, int outside) {
  return guarded(c, [&]() -> int {
    if (!qs || !q) fail(c, CRUNA_ERR_ARG, "null pointer");
    bc_qs(c, qs, q, outside);
    return CRUNA_OK;
  });
}
int cruna_bc_rhs_dev(cruna_ctx *c, double *rhs, const double *q) {
  return guarded(c, [&]() -> int {
    if (!rhs || !q) fail(c, CRUNA_ERR_ARG, "null pointer");
    bc_rhs(c, rhs, q);
    return CRUNA_OK;
  });
}
int cruna_bc_rhss_dev(cruna_ctx *c, double *rhss, const double *qs, const double *q) {
  return guarded(c, [&]() -> int {
    if (!rhss || !qs) fail(c, CRUNA_ERR_ARG, "null pointer");
    bc_rhss(c, rhss, qs, q);
    return CRUNA_OK;
  });
}

int cruna_bc_q(cruna_ctx *c, double *q, int outside) {
  return guarded(c, [&]() -> int {
    if (!q) fail(c, CRUNA_ERR_ARG, "null pointer");
    double *d = stage_in(c, 0, q, 5);
    bc_q(c, d, outside);
    stage_out(c, q, d, 5);
    return CRUNA_OK;
  });
}
int cruna_bc_qs(cruna_ctx *c, double *qs, const double *q, int outside) {
  return guarded(c, [&]() -> int {
    if (!qs || !q) fail(c, CRUNA_ERR_ARG, "null pointer");
    double *d = stage_in(c, 0, qs, 5);
    double *dq = stage_in(c, 1, q, 5);
    bc_qs(c, d, dq, outside);
    stage_out(c, qs, d, 5);
    return CRUNA_OK;
  });
}
int cruna_bc_rhs(cruna_ctx *c, double *rhs, const double *q) {
  return guarded(c, [&]() -> int {
    if (!rhs || !q) fail(c, CRUNA_ERR_ARG, "null pointer");
    double *d = stage_in(c, 0, rhs, 5);
    double *dq = stage_in(c, 1, q, 5);
    bc_rhs(c, d, dq);
    stage_out(c, rhs, d, 5);
    return CRUNA_OK;
  });
}
int cruna_bc_rhss(cruna_ctx *c, double *rhss, const double *qs, const double *q) {
  return guarded(c, [&]() -> int {
    if (!rhss || !qs) fail(c, CRUNA_ERR_ARG, "null pointer");
    double *d = stage_in(c, 0, rhss, 5);
    double *dqs = stage_in(c, 1, qs, 5);
    double *dq = q ? stage_in(c, 2, q, 5) : nullptr;
    bc_rhss(c, d, dqs, dq);
    stage_out(c, rhss, d, 5);
    return CRUNA_OK;
  });
}

static int diagnostics_common(cruna_ctx *c, const double *q_dev, double *ke, double *ens) {
  if (c->halo_fn) fail(c, CRUNA_ERR_UNSUPPORTED, "volume diagnostics over z slabs are not provided");
  if (!c->diag) c->diag = dalloc(c, 600);
  diagnostics_impl(c, q_dev, c->diag + 592, c->diag);
  double h[2] = {0.0, 0.0};
  CRUNA_CUDA_CHECK(cudaMemcpyAsync(h, c->diag + 592, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
  if (ke) *ke = h[0];
  if (ens) *ens = h[1];
  return CRUNA_OK;
}

// kinetic energy and enstrophy (the volume integrals a case's post-processing forms from snapshots)
int cruna_diagnostics_dev(cruna_ctx *c, const double *q, double *ke, double *ens) {
  return guarded(c, [&]() -> int {
    if (!q) fail(c, CRUNA_ERR_ARG, "null pointer");
    return diagnostics_common(c, q, ke, ens);
  });
}

int cruna_diagnostics(cruna_ctx *c, const double *q, double *ke, double *ens) {
  return guarded(c, [&]() -> int {
    if (!q) fail(c, CRUNA_ERR_ARG, "null pointer");
    return diagnostics_common(c, stage_in(c, 0, q, 5), ke, ens);
  });
}

int cruna_check_state_dev(cruna_ctx *c, const double *q) {
  return guarded(c, [&]() -> int {
    if (!q) fail(c, CRUNA_ERR_ARG, "null pointer");
    check_or_fail(c, q, 0);
    return CRUNA_OK;
  });
}

}  // extern "C"

namespace cruna {

// one step of the loop body of calc_direct (computation_direct.f90:76-95): time_stepper_direct,
// set_boundary_condition_q(outside_rhs) and the filters whose frequency divides nt; q in place
static void direct_loop_body(cruna_ctx *c, double *q, const int on[3]) {
  if (c->filter_fused_ok && !c->force_generic && (on[0] || on[1] || on[2])) {
    step_direct(c, q, c->st[5]);
    if (c->has_q_bc) bc_q(c, c->st[5], 1);
    if (on[2]) halo(c, c->st[5], 5);
    filter3_fused(c, c->st[5], q, on);
  } else {
    step_direct(c, q, q);
    if (c->has_q_bc) bc_q(c, q, 1);
    if (on[2]) halo(c, q, 5);
    for (int d = 0; d < 3; ++d)
      if (on[d]) apply_filter(c, d, q, c->st[5], 5);
  }
}

// one step of the loop body of calc_adjoint (computation_adjoint.f90:81-101): time_stepper_adjoint
// with the frozen direct state q0 and source g, set_boundary_condition_qs(outside_rhs), filters
static void adjoint_loop_body(cruna_ctx *c, double *qs, const double *q0, const double *g, const int on[3]) {
  if (c->filter_fused_ok && !c->force_generic && (on[0] || on[1] || on[2])) {
    step_adjoint(c, qs, q0, g, c->st[5]);
    if (c->has_q_bc) bc_qs(c, c->st[5], q0, 1);
    if (on[2]) halo(c, c->st[5], 5);
    filter3_fused(c, c->st[5], qs, on);
  } else {
    step_adjoint(c, qs, q0, g, qs);
    if (c->has_q_bc) bc_qs(c, qs, q0, 1);
    if (on[2]) halo(c, qs, 5);
    for (int d = 0; d < 3; ++d)
      if (on[d]) apply_filter(c, d, qs, c->st[5], 5);
  }
}

// the loop steps as the run loops and the gradient call them: nt selects the filters due; a step
// that repeats with the same buffers and filter pattern is replayed from a graph (step_graph.cu)
void direct_loop_step(cruna_ctx *c, double *q, int nt) {
  const int on[3] = {due(c->cfg.di_freq[0], nt), due(c->cfg.di_freq[1], nt), due(c->cfg.di_freq[2], nt)};
  graph_step(c, on[0] | on[1] << 1 | on[2] << 2, q, nullptr, nullptr, [&]() { direct_loop_body(c, q, on); });
}

void adjoint_loop_step(cruna_ctx *c, double *qs, const double *q0, const double *g, int nt) {
  const int on[3] = {due(c->cfg.ai_freq[0], nt), due(c->cfg.ai_freq[1], nt), due(c->cfg.ai_freq[2], nt)};
  graph_step(c, 8 | on[0] | on[1] << 1 | on[2] << 2, qs, q0, g,
             [&]() { adjoint_loop_body(c, qs, q0, g, on); });
}

long long gradient_impl(cruna_ctx *c, const double *q0, int nsteps, int nsnap, const cruna_objective *obj,
                        double *J_dev, double *grad_f, double *grad_q0, std::vector<void *> &scratch);
double objective_direct_impl(cruna_ctx *c, const double *q0, int nsteps, const cruna_objective *obj,
                             std::vector<void *> &scratch);
void axpy_state(cruna_ctx *c, double a, const double *x, double *y);

}  // namespace cruna

extern "C" {

// loop body of calc_direct (computation_direct.f90:64-107); traj is a device pointer or NULL
static int run_direct_impl(cruna_ctx *c, double *q, int nt0, int nsteps, double *traj, bool traj_host) {
  GraphScope graphs(c);
  for (int s = 1; s <= nsteps; ++s) {
    const int nt = nt0 + s;
    direct_loop_step(c, q, nt);
    if (traj) {                                                    // :98-100
      double *dst = traj + (long long)(s - 1) * N5(c);
      CRUNA_CUDA_CHECK(cudaMemcpyAsync(dst, q, sizeof(double) * N5(c),
                                       traj_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                       c->stream));
    }
    if (c->cfg.check_every > 0 && nt % c->cfg.check_every == 0) check_or_fail(c, q, nt);
  }
  return CRUNA_OK;
}

int cruna_run_direct_dev(cruna_ctx *c, double *q_io, int nt0, int nsteps, double *traj) {
  return guarded(c, [&]() -> int {
    if (!q_io || nsteps < 0) fail(c, CRUNA_ERR_ARG, "bad arguments to cruna_run_direct");
    return run_direct_impl(c, q_io, nt0, nsteps, traj, false);
  });
}

int cruna_run_direct(cruna_ctx *c, double *q_io, int nt0, int nsteps, double *traj) {
  return guarded(c, [&]() -> int {
    if (!q_io || nsteps < 0) fail(c, CRUNA_ERR_ARG, "bad arguments to cruna_run_direct");
    double *dq = stage_in(c, 0, q_io, 5);
    int rc = run_direct_impl(c, dq, nt0, nsteps, traj, true);
    if (rc) return rc;
    stage_out(c, q_io, dq, 5);
    return CRUNA_OK;
  });
}

// loop body of calc_adjoint (computation_adjoint.f90:60-108)
static int run_adjoint_impl(cruna_ctx *c, double *qs, const double *Q, const double *G, int nt_end,
                            int nsteps, bool host) {
  GraphScope graphs(c);
  const int nt_first = nt_end - nsteps + 1;
  for (int nt = nt_end; nt >= nt_first; --nt) {
    const long long off = (long long)(nt - nt_first) * N5(c);
    const double *q0 = Q + off;
    const double *g = G ? G + off : nullptr;
    if (host) {
      double *dq = stage_in(c, 1, Q + off, 5);
      q0 = dq;
      g = G ? stage_in(c, 2, G + off, 5) : nullptr;
    }
    adjoint_loop_step(c, qs, q0, g, nt);
    if (c->cfg.check_every > 0 && nt % c->cfg.check_every == 0) {
      int f = check_state(c, qs);
      if (f & 1) fail(c, CRUNA_ERR_STATE, "adjoint state not finite at step " + std::to_string(nt));
    }
  }
  return CRUNA_OK;
}

int cruna_run_adjoint_dev(cruna_ctx *c, double *qs_io, const double *Q_traj, const double *g_traj, int nt_end,
                          int nsteps) {
  return guarded(c, [&]() -> int {
    if (!qs_io || !Q_traj || nsteps < 0) fail(c, CRUNA_ERR_ARG, "bad arguments to cruna_run_adjoint");
    return run_adjoint_impl(c, qs_io, Q_traj, g_traj, nt_end, nsteps, false);
  });
}

int cruna_run_adjoint(cruna_ctx *c, double *qs_io, const double *Q_traj, const double *g_traj, int nt_end,
                      int nsteps) {
  return guarded(c, [&]() -> int {
    if (!qs_io || !Q_traj || nsteps < 0) fail(c, CRUNA_ERR_ARG, "bad arguments to cruna_run_adjoint");
    double *dqs = stage_in(c, 0, qs_io, 5);
    int rc = run_adjoint_impl(c, dqs, Q_traj, g_traj, nt_end, nsteps, true);
    if (rc) return rc;
    stage_out(c, qs_io, dqs, 5);
    return CRUNA_OK;
  });
}

static int gradient_common(cruna_ctx *c, const double *q0_dev, int nsteps, int nsnap, const cruna_objective *obj,
                           double *J, double *gf_dev, double *gq_dev, int64_t *direct_steps) {
  if (!q0_dev || !obj || !J || nsteps < 1 || nsnap < 1) fail(c, CRUNA_ERR_ARG, "bad arguments to cruna_gradient");
  if (c->halo_fn) fail(c, CRUNA_ERR_UNSUPPORTED, "objective reductions over z slabs are not provided");
  if (obj->kind != CRUNA_OBJ_PLANE_P2 && obj->kind != CRUNA_OBJ_KINETIC_ENERGY &&
      obj->kind != CRUNA_OBJ_ENSTROPHY)
    fail(c, CRUNA_ERR_ARG, "unknown objective kind");
  if (obj->kind == CRUNA_OBJ_PLANE_P2) {
    if (obj->normal < 1 || obj->normal > 3) fail(c, CRUNA_ERR_ARG, "objective plane normal must be 1..3");
    if (obj->index < 1 || obj->index > c->cfg.n[obj->normal - 1])
      fail(c, CRUNA_ERR_ARG, "objective plane index outside the grid");
  }
  std::vector<void *> scratch;
  double *Jd = nullptr;
  long long adv = 0;
  try {
    void *p = nullptr;
    CRUNA_CUDA_CHECK(cudaMalloc(&p, sizeof(double)));
    scratch.push_back(p);
    Jd = static_cast<double *>(p);
    adv = gradient_impl(c, q0_dev, nsteps, nsnap, obj, Jd, gf_dev, gq_dev, scratch);
    CRUNA_CUDA_CHECK(cudaMemcpyAsync(J, Jd, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
  } catch (...) {
    cudaStreamSynchronize(c->stream);
    for (void *q : scratch) cudaFree(q);
    throw;
  }
  for (void *q : scratch) cudaFree(q);
  if (direct_steps) *direct_steps = adv;
  return CRUNA_OK;
}

// optimisation loop of cruna.f90:78-179 on the device-resident forcing f (5N, updated in place):
// direct run and J, adjoint gradient (except in the last loop), ls_quadratic_fit
// (line_search.f90:23-127) when loop >= ls_start, update f <- f - alpha dJ/df
static int optimize_common(cruna_ctx *c, const double *q0, const cruna_objective *obj, int nsteps, int nsnap,
                           int maxloop, int ls_start, double alpha0, double *f, double *J_hist,
                           double *alpha_hist) {
  if (!q0 || !obj || !f || maxloop < 1 || nsteps < 1 || nsnap < 1 || !(alpha0 > 0.0))
    fail(c, CRUNA_ERR_ARG, "bad arguments to cruna_optimize");
  if (c->halo_fn) fail(c, CRUNA_ERR_UNSUPPORTED, "objective reductions over z slabs are not provided");
  if (obj->kind == CRUNA_OBJ_PLANE_P2 &&
      (obj->normal < 1 || obj->normal > 3 || obj->index < 1 || obj->index > c->cfg.n[obj->normal - 1]))
    fail(c, CRUNA_ERR_ARG, "bad objective plane");
  if (obj->kind != CRUNA_OBJ_PLANE_P2 && obj->kind != CRUNA_OBJ_KINETIC_ENERGY &&
      obj->kind != CRUNA_OBJ_ENSTROPHY)
    fail(c, CRUNA_ERR_ARG, "unknown objective kind");
  std::vector<void *> scratch;
  double *saved_user = c->closure_mlp ? c->user_force : c->force;
  try {
    auto alloc = [&]() {
      void *p = nullptr;
      CRUNA_CUDA_CHECK(cudaMalloc(&p, sizeof(double) * N5(c)));
      scratch.push_back(p);
      return static_cast<double *>(p);
    };
    double *gf = alloc(), *fb = alloc(), *Jd = nullptr;
    {
      void *p = nullptr;
      CRUNA_CUDA_CHECK(cudaMalloc(&p, sizeof(double)));
      scratch.push_back(p);
      Jd = static_cast<double *>(p);
    }
    for (int loop = 1; loop <= maxloop; ++loop) {
      point_forcing(c, f);
      double J = 0.0;
      if (loop == maxloop) {                                   // cruna.f90:127-133: stop after the objective
        std::vector<void *> sc;
        try {
          J = objective_direct_impl(c, q0, nsteps, obj, sc);
        } catch (...) {
          for (void *p : sc) cudaFree(p);
          throw;
        }
        for (void *p : sc) cudaFree(p);
        if (J_hist) J_hist[loop - 1] = J;
        break;
      }
      std::vector<void *> sc;
      try {
        gradient_impl(c, q0, nsteps, nsnap, obj, Jd, gf, nullptr, sc);
      } catch (...) {
        for (void *p : sc) cudaFree(p);
        throw;
      }
      for (void *p : sc) cudaFree(p);
      CRUNA_CUDA_CHECK(cudaMemcpyAsync(&J, Jd, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
      if (J_hist) J_hist[loop - 1] = J;
      double alpha = alpha0;
      if (loop >= ls_start) {                                  // ls_quadratic_fit
        const double a[3] = {0.0, 0.5 * alpha0, alpha0};
        double Js[3] = {J, 0.0, 0.0};
        copy_state(c, fb, f, 5);                               // backup_force
        for (int ls = 1; ls <= 2; ++ls) {
          copy_state(c, f, fb, 5);
          axpy_state(c, -a[ls], gf, f);                        // update_force with alpha = a[ls]
          std::vector<void *> s2;
          try {
            Js[ls] = objective_direct_impl(c, q0, nsteps, obj, s2);
          } catch (...) {
            for (void *p : s2) cudaFree(p);
            throw;
          }
          for (void *p : s2) cudaFree(p);
        }
        copy_state(c, f, fb, 5);                               // restore_force
        // dgesv of M c = Js, M rows (a^2, a, 1): Gaussian elimination with partial pivoting
        double M[3][4];
        for (int i = 0; i < 3; ++i) {
          M[i][0] = a[i] * a[i];
          M[i][1] = a[i];
          M[i][2] = 1.0;
          M[i][3] = Js[i];
        }
        bool singular = false;
        for (int col = 0; col < 3 && !singular; ++col) {
          int piv = col;
          for (int r = col + 1; r < 3; ++r)
            if (std::fabs(M[r][col]) > std::fabs(M[piv][col])) piv = r;
          if (M[piv][col] == 0.0) {
            singular = true;
            break;
          }
          if (piv != col)
            for (int k = 0; k < 4; ++k) std::swap(M[piv][k], M[col][k]);
          for (int r = col + 1; r < 3; ++r) {
            const double m = M[r][col] / M[col][col];
            for (int k = col; k < 4; ++k) M[r][k] -= m * M[col][k];
          }
        }
        if (!singular) {
          double x[3];
          for (int i = 2; i >= 0; --i) {
            double s = M[i][3];
            for (int k = i + 1; k < 3; ++k) s -= M[i][k] * x[k];
            x[i] = s / M[i][i];
          }
          alpha = -x[1] / (2.0 * x[0]);
          if (alpha > 10.0 * alpha0) alpha = 10.0 * alpha0;     // line_search.f90:103-112
        }
      }
      if (alpha_hist) alpha_hist[loop - 1] = alpha;
      axpy_state(c, -alpha, gf, f);                            // update_force
    }
    CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
  } catch (...) {
    cudaStreamSynchronize(c->stream);
    for (void *p : scratch) cudaFree(p);
    point_forcing(c, saved_user);
    throw;
  }
  for (void *p : scratch) cudaFree(p);
  point_forcing(c, saved_user);
  return CRUNA_OK;
}

int cruna_objective_value_dev(cruna_ctx *c, const double *q0, int nsteps, const cruna_objective *obj, double *J) {
  return guarded(c, [&]() -> int {
    if (!q0 || !obj || !J || nsteps < 1) fail(c, CRUNA_ERR_ARG, "bad arguments to cruna_objective_value");
    if (c->halo_fn) fail(c, CRUNA_ERR_UNSUPPORTED, "objective reductions over z slabs are not provided");
    if (obj->kind == CRUNA_OBJ_PLANE_P2 &&
        (obj->normal < 1 || obj->normal > 3 || obj->index < 1 || obj->index > c->cfg.n[obj->normal - 1]))
      fail(c, CRUNA_ERR_ARG, "bad objective plane");
    if (obj->kind != CRUNA_OBJ_PLANE_P2 && obj->kind != CRUNA_OBJ_KINETIC_ENERGY &&
      obj->kind != CRUNA_OBJ_ENSTROPHY)
      fail(c, CRUNA_ERR_ARG, "unknown objective kind");
    std::vector<void *> sc;
    try {
      *J = objective_direct_impl(c, q0, nsteps, obj, sc);
    } catch (...) {
      for (void *p : sc) cudaFree(p);
      throw;
    }
    for (void *p : sc) cudaFree(p);
    return CRUNA_OK;
  });
}

int cruna_objective_value(cruna_ctx *c, const double *q0, int nsteps, const cruna_objective *obj, double *J) {
  return guarded(c, [&]() -> int {
    if (!q0) fail(c, CRUNA_ERR_ARG, "null pointer");
    double *dq = stage_in(c, 0, q0, 5);
    return cruna_objective_value_dev(c, dq, nsteps, obj, J);
  });
}

int cruna_optimize_dev(cruna_ctx *c, const double *q0, const cruna_objective *obj, int nsteps, int nsnap,
                       int maxloop, int ls_start, double alpha0, double *f, double *J_hist, double *alpha_hist) {
  return guarded(c, [&]() -> int {
    return optimize_common(c, q0, obj, nsteps, nsnap, maxloop, ls_start, alpha0, f, J_hist, alpha_hist);
  });
}

int cruna_optimize(cruna_ctx *c, const double *q0, const cruna_objective *obj, int nsteps, int nsnap, int maxloop,
                   int ls_start, double alpha0, double *f, double *J_hist, double *alpha_hist) {
  return guarded(c, [&]() -> int {
    if (!q0 || !f) fail(c, CRUNA_ERR_ARG, "null pointer");
    double *dq = stage_in(c, 0, q0, 5), *df = stage_in(c, 1, f, 5);
    int rc = optimize_common(c, dq, obj, nsteps, nsnap, maxloop, ls_start, alpha0, df, J_hist, alpha_hist);
    stage_out(c, f, df, 5);
    return rc;
  });
}

int cruna_set_halo_exchange(cruna_ctx *c, int (*fn)(void *, double *, int, void *), void *user) {
  return guarded(c, [&]() -> int {
    if (fn && (c->dop[2].kind != OP_STENCIL || !c->dop[2].periodic || c->has_q_bc || c->has_rhs_bc))
      fail(c, CRUNA_ERR_UNSUPPORTED, "z slabs need a periodic z scheme and no boundary table");
    c->halo_fn = fn;
    c->halo_user = user;
    return CRUNA_OK;
  });
}

int cruna_set_snapshot_memory(cruna_ctx *c, int host) {
  return guarded(c, [&]() -> int {
    c->snapshot_host = host != 0;
    if (!c->snapshot_host && !c->snap_pinned.empty()) {  // give the pinned host slots back
      CRUNA_CUDA_CHECK(cudaStreamSynchronize(c->stream));
      for (void *p : c->snap_pinned) cudaFreeHost(p);
      c->snap_pinned.clear();
    }
    return CRUNA_OK;
  });
}

int cruna_set_adjoint_mode(cruna_ctx *c, int mode) {
  return guarded(c, [&]() -> int {
    if (mode != 0 && mode != 1) fail(c, CRUNA_ERR_ARG, "adjoint mode must be 0 (continuous) or 1 (discrete)");
    if (mode == 1 && c->cfg.precision != CRUNA_FP64)
      fail(c, CRUNA_ERR_UNSUPPORTED, "the discrete adjoint needs precision CRUNA_FP64");
    if (mode == 1 && c->closure_mlp)
      fail(c, CRUNA_ERR_UNSUPPORTED, "the discrete adjoint does not transpose the closure");
    c->adjoint_mode = mode;
    return CRUNA_OK;
  });
}

int cruna_rhs_direct_vjp_dev(cruna_ctx *c, const double *q, const double *lam, double *mu, double *grad_f) {
  return guarded(c, [&]() -> int {
    if (!q || !lam || !mu) fail(c, CRUNA_ERR_ARG, "null pointer");
    rhs_direct_vjp(c, q, lam, mu, grad_f);
    return CRUNA_OK;
  });
}

int cruna_rhs_direct_vjp(cruna_ctx *c, const double *q, const double *lam, double *mu, double *grad_f) {
  return guarded(c, [&]() -> int {
    if (!q || !lam || !mu) fail(c, CRUNA_ERR_ARG, "null pointer");
    double *dq = stage_in(c, 0, q, 5), *dl = stage_in(c, 1, lam, 5), *dm = stage_in(c, 2, nullptr, 5);
    double *dg = grad_f ? stage_gf(c, grad_f) : nullptr;
    rhs_direct_vjp(c, dq, dl, dm, dg);
    if (dg) stage_out(c, grad_f, dg, 5);
    stage_out(c, mu, dm, 5);
    return CRUNA_OK;
  });
}

int cruna_step_direct_vjp_dev(cruna_ctx *c, const double *q0, const double *lam1, double *lam0, double *grad_f,
                              int nt) {
  return guarded(c, [&]() -> int {
    if (!q0 || !lam1 || !lam0) fail(c, CRUNA_ERR_ARG, "null pointer");
    step_direct_vjp(c, q0, lam1, lam0, grad_f, nt);
    return CRUNA_OK;
  });
}

int cruna_step_direct_vjp(cruna_ctx *c, const double *q0, const double *lam1, double *lam0, double *grad_f,
                          int nt) {
  return guarded(c, [&]() -> int {
    if (!q0 || !lam1 || !lam0) fail(c, CRUNA_ERR_ARG, "null pointer");
    double *dq = stage_in(c, 0, q0, 5), *dl = stage_in(c, 1, lam1, 5), *dm = stage_in(c, 2, nullptr, 5);
    double *dg = grad_f ? stage_gf(c, grad_f) : nullptr;
    step_direct_vjp(c, dq, dl, dm, dg, nt);
    if (dg) stage_out(c, grad_f, dg, 5);
    stage_out(c, lam0, dm, 5);
    return CRUNA_OK;
  });
}

int cruna_gradient_dev(cruna_ctx *c, const double *q0, int nsteps, int nsnap, const cruna_objective *obj,
                       double *J, double *grad_f, double *grad_q0, int64_t *direct_steps) {
  return guarded(c, [&]() -> int {
    return gradient_common(c, q0, nsteps, nsnap, obj, J, grad_f, grad_q0, direct_steps);
  });
}

int cruna_gradient(cruna_ctx *c, const double *q0, int nsteps, int nsnap, const cruna_objective *obj, double *J,
                   double *grad_f, double *grad_q0, int64_t *direct_steps) {
  return guarded(c, [&]() -> int {
    if (!q0) fail(c, CRUNA_ERR_ARG, "null q0");
    double *dq0 = stage_in(c, 0, q0, 5);
    double *dgf = grad_f ? stage_in(c, 1, nullptr, 5) : nullptr;
    double *dgq = grad_q0 ? stage_in(c, 2, nullptr, 5) : nullptr;
    int rc = gradient_common(c, dq0, nsteps, nsnap, obj, J, dgf, dgq, direct_steps);
    if (rc) return rc;
    if (grad_f) stage_out(c, grad_f, dgf, 5);
    if (grad_q0) stage_out(c, grad_q0, dgq, 5);
    return CRUNA_OK;
  });
}

// restated LAPACK routines, exported so the test-suite can compare them with LAPACK itself
int cruna_lapack_dgttrf(int n, double *dl, double *d, double *du, double *du2, int *ipiv) {
  return lapack_dgttrf(n, dl, d, du, du2, ipiv);
}
void cruna_lapack_dgttrs(int n, const double *dl, const double *d, const double *du, const double *du2,
                         const int *ipiv, double *b) {
  lapack_dgttrs(n, dl, d, du, du2, ipiv, b);
}

}  // extern "C"
