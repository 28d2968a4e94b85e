// Internal declarations of the CRUNA B200 library: line operators, context, kernel launchers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/cruna_b200.h"

namespace cruna {

constexpr int kMaxR = 6;        // largest interior half-width (o10 filter: 5)
constexpr int kMaxRows = 5;     // largest number of explicit boundary rows at one end
constexpr int kMaxRowW = 12;    // widest boundary row (o10 filter: 11 points)

enum OpKind { OP_ZERO = 0, OP_COPY = 1, OP_STENCIL = 2 };

// One direction's derivative or filter operator on lines of n points: an explicit stencil part
// (interior + optional one-sided rows at both ends, or periodic wrap), optionally followed by a
// tridiagonal solve with LAPACK dgttrf factors and a Sherman-Morrison cyclic correction -- the
// structure shared by every src/diff/diff_pen_core_* and src/filter/filter_pen_core_* module.
struct LineOp {
  int n = 1;
  int kind = OP_ZERO;
  int periodic = 0;
  int antisym = 0;                 // 1: derivative (end rows mirror with a sign flip)
  int r = 0;                       // interior half-width
  double c[kMaxR + 1] = {0};       // interior coefficients c[0..r] (c[0] unused when antisym)
  int nb = 0;                      // explicit rows at each end (open lines)
  int bw = 0;                      // width of those rows
  int keep_ends = 0;               // row 0 copies the input (open filters)
  double brow[kMaxRows][kMaxRowW] = {{0}};
  double div = 1.0;                // explicit part is divided by (h * div): 12 for o4 explicit
  int solve = 0;                   // dgttrs follows
  int cyclic = 0;                  // Sherman-Morrison correction follows
  int nopiv = 0;                   // dgttrf interchanged no rows (ipiv[i] == i + 1 throughout)
  double blend = 0.0;              // >0: out = q - blend * (q - F q)
  double fbrat = 0.0;
  // device factor arrays (owned by the context)
  const double *dl = nullptr, *inv_d = nullptr, *du = nullptr, *du2 = nullptr, *fbnorm = nullptr;
  const int *ipiv = nullptr;
};

// Host-side copy of the factors (filled by the dgttrf restatement in schemes.cpp).
struct HostFactors {
  std::vector<double> dl, d, du, du2, fbnorm;
  std::vector<double> raw_dl, raw_d, raw_du;  // the tridiagonal matrix before dgttrf (for B^T)
  std::vector<int> ipiv;  // 1-based as LAPACK
  double fbrat = 0.0;
  int info = 0;
};

// Transpose of a line operator (discrete adjoint): out = scale * A^T (B^-T in) where the operator is
// B^-1 A.  A^T is kept as a band: band[j*(hi-lo+1) + (o-lo)] multiplies in[j+o] (wrapped on
// periodic lines); sop holds the factors of B^T (B itself when B is symmetric).
struct LineOpT {
  int n = 1;
  int kind = OP_ZERO;   // OP_ZERO, OP_COPY (identity) or OP_STENCIL (band)
  int periodic = 0;
  int lo = 0, hi = 0;
  const double *band = nullptr;
  int solve = 0;
  LineOp sop;
};

struct Grid {
  int n1, n2, n3;
  long long N;   // points per field
};

// builds the operators (schemes.cpp); return false + message on unsupported input
bool build_diff_op(int scheme, int n, LineOp &op, HostFactors &hf, std::string &err);
bool build_filter_op(int scheme, int n, double alpha, double strength, LineOp &op, HostFactors &hf,
                     std::string &err);
bool diff_is_periodic(int scheme);
// LAPACK dgttrf / dgttrs (no transpose) restated (schemes.cpp); exposed for tests through the C API
int lapack_dgttrf(int n, double *dl, double *d, double *du, double *du2, int *ipiv);
void lapack_dgttrs(int n, const double *dl, const double *d, const double *du, const double *du2,
                   const int *ipiv, double *b);

// error raised inside the library and returned by the extern "C" entry points as (code, message)
struct ApiError {
  int code;
  std::string msg;
};

struct BCRow {
  int type;
  int is, ie, js, je, ks, ke;  // 0-based inclusive
  double k[3];
  int comp;                    // wall component (0-based)
  int shift[3];                // type 200: offset of the aim plane
  int only = 0;                // type 203: -1 applies outside the RHS only, 1 inside only
};

// device sponge-shape factors: phi = (((sx[i]*sym[j])*syp[j])*szm[k])*szp[k]; shape = amp*(1-phi)
struct SpongeDev {
  const double *sx = nullptr, *sym = nullptr, *syp = nullptr, *szm = nullptr, *szp = nullptr;
  double amp = 0.0;
};

class StepGraphs;  // step_graph.cu

}  // namespace cruna

struct cruna_ctx {
  cruna_config cfg;
  cruna::Grid g;
  double dx[3];
  cruna::LineOp dop[3];   // derivative operators
  cruna::LineOp fop[3];   // filter operators
  std::vector<cruna::BCRow> bc;
  bool has_q_bc = false, has_rhs_bc = false, has_sponge = false, has_nonlocal_bc = false;
  cruna::SpongeDev sponge;
  cudaStream_t stream = nullptr;
  int device = 0;
  int64_t launches = 0;
  std::string err;
  bool force_generic = false;
  bool fused_ok = false;
  bool tma_fused = false;       // FP64 adjoint pass fed by TMA where the layout allows (cruna_set_tma_passes)
  bool filter_fused_ok = false;
  // FP32-stencil path: pressure / temperature offsets differenced in FP32 (set once per context)
  bool refs_set = false;
  double p_ref = 0.0, T_ref = 0.0;
  // kernel timing (cruna_profile_enable): events bracketing launches on the context's stream
  bool prof_on = false;
  struct ProfEntry {
    const char *name;
    cudaEvent_t a, b;
  };
  std::vector<ProfEntry> prof_pending;
  std::vector<cudaEvent_t> prof_pool;
  std::map<std::string, std::pair<long long, double>> prof_acc;
  // device memory
  std::vector<void *> allocations;
  double *qref = nullptr;        // 5N
  double *kvec = nullptr;        // 3N boundary normal vectors (zonal BC types 202/203/205/206)
  double *force = nullptr;       // 5N or null
  double *st[6] = {nullptr};     // state-sized work buffers
  double *io[4] = {nullptr};     // staging for host-pointer entry points (5N each)
  double *tmp = nullptr;         // generic-path temporaries (kGenericFields * N)
  double *fz = nullptr;          // fused-path intermediates
  float *fz32 = nullptr;         // fused-path FP32 intermediates
  double *red = nullptr;         // reduction scratch
  int *flag = nullptr;           // device error flag
  // discrete adjoint (discrete_adjoint.cu): host factors kept for the transposes, built on first use
  cruna::HostFactors dhf[3], fhf[3];
  bool vjp_ready = false;
  cruna::LineOpT dopT[3], fopT[3];
  bool dopT_built[3] = {false, false, false};  // transposed derivative operators (also for objectives)
  double *vjp_ws = nullptr;        // backward workspace (fields)
  double *vjp_st[12] = {nullptr};  // state-sized buffers of the transposed step
  std::vector<double *> vjp_save;  // per boundary row: box values before the row (q, aim / rhs)
  double *vjp_gf = nullptr;        // staging of grad_f for the host-pointer entry points (io[3] holds f)
  int adjoint_mode = 0;            // cruna_gradient: 0 continuous (reference), 1 discrete
  // z-slab decomposition: refreshes the halo planes of a state before a pass that reads z-neighbours
  int (*halo_fn)(void *user, double *fields, int nfields, void *stream) = nullptr;
  void *halo_user = nullptr;
  // learned subgrid closure (closure_ops.cu): active when mlp is set
  struct cruna_mlp *closure_mlp = nullptr;
  double closure_delta = 0.0;
  bool closure_norm = false;       // scale-free features / outputs (cruna_set_closure_normalisation)
  bool closure_fused = true;       // network evaluated inside the fused pass G (cruna_set_closure_fused)
  double *user_force = nullptr;    // the caller's forcing (cruna_set_forcing) while a closure is set
  double *cl_force = nullptr;      // forcing + closure stress divergence (5N)
  double *cl_tau = nullptr;        // model stresses (6N) and their derivatives (9N)
  float *cl_x = nullptr, *cl_y = nullptr;  // features (12N) and outputs (6N), point-major
  double *diag = nullptr;          // diagnostics reduction scratch (partials + 2 results)
  bool snapshot_host = false;      // gradient snapshots in pinned host memory instead of HBM
  std::vector<void *> snap_pinned;  // those host slots (one state each), kept for later gradient calls
  // step graphs (step_graph.cu): the cache of the current run call, or null outside one
  bool graphs_enabled = true;
  cruna::StepGraphs *graphs = nullptr;
  int64_t graph_captures = 0, graph_replays = 0;
};

namespace cruna {

// launch helpers (ops.cu)
void launch_line_stencil(cruna_ctx *c, const LineOp &op, int dir, const double *f1, const double *f2,
                         double *out, double scale, int nfields, double sign = 1.0);
void launch_line_solve(cruna_ctx *c, const LineOp &op, int dir, double *data, int nfields);
void apply_diff(cruna_ctx *c, int dir, const double *f1, const double *f2, double *out, double h,
                int nfields);
void apply_filter(cruna_ctx *c, int dir, double *q, double *scratch, int nfields);

// RHS / BC / RK (ops.cu, fused.cu)
// bc_mask: 1 applies the BC on q before, 2 the BC on the RHS after (3 = the reference order)
void rhs_direct_generic(cruna_ctx *c, const double *q, double *rhs, double *qbc_scratch, int bc_mask = 3);
void generic_forward_gradients(cruna_ctx *c, const double *q);  // primitives, grads, mu, tau into tmp
void rhs_adjoint_generic(cruna_ctx *c, const double *qs, const double *q, const double *g, double *rhs,
                         double *qsbc_scratch);
bool fused_supported(const cruna_ctx *c);
void rhs_direct_fused(cruna_ctx *c, const double *q, double *rhs, int stage, const double *q0,
                      double *acc, double *qnext, double dt);
void rhs_adjoint_fused(cruna_ctx *c, const double *qs, const double *q, const double *g, double *rhs,
                       int stage, const double *qs0, double *acc, double *qnext, double dt);
bool filter_fused_supported(const cruna_ctx *c);
void filter3_fused(cruna_ctx *c, const double *in, double *out, const int on[3]);
void build_kvector(cruna_ctx *c);  // normal-vector field of the zonal BC types (ops.cu)
void bc_q(cruna_ctx *c, double *q, int outside);
void bc_qs(cruna_ctx *c, double *qs, const double *q, int outside);
void bc_rhs(cruna_ctx *c, double *rhs, const double *q);
void bc_rhss(cruna_ctx *c, double *rhss, const double *qs, const double *q);
void rk_stage(cruna_ctx *c, int stage, double dt, const double *k, const double *q0, double *acc,
              double *qnext);
void copy_state(cruna_ctx *c, double *dst, const double *src, int nfields);
int check_state(cruna_ctx *c, const double *q);
// out = D_d^T in (one field) with grid spacing h, building the transposed operator on first use
// (discrete_adjoint.cu); scratch: one field
void diff_transpose(cruna_ctx *c, int d, const double *in, double *out, double h, double *scratch);
// kinetic energy and enstrophy of q into out[0], out[1] on the device (gradient.cu); partial: 592 doubles
void diagnostics_impl(cruna_ctx *c, const double *q, double *out, double *partial);

// step graphs (step_graph.cu): a GraphScope makes a graph cache live for one run call (an inner scope
// uses the outer one's); graph_step runs body() as the loop step keyed by (kind, a, b, d): eagerly at
// the key's first sighting, recorded at its second, replayed after that
class GraphScope {
 public:
  explicit GraphScope(cruna_ctx *c);
  ~GraphScope();
  GraphScope(const GraphScope &) = delete;
  GraphScope &operator=(const GraphScope &) = delete;

 private:
  cruna_ctx *c_;
  StepGraphs *own_ = nullptr;
};
void graph_step(cruna_ctx *c, int kind, const void *a, const void *b, const void *d,
                const std::function<void()> &body);
double *dalloc(cruna_ctx *c, size_t count);
void ensure_generic(cruna_ctx *c);
bool use_fused(const cruna_ctx *c);
// learned closure (closure_mlp.cu, closure_ops.cu)
void mlp_forward_stream(struct cruna_mlp *h, const float *X, float *Y, long long n, cudaStream_t stream);
void closure_stage(cruna_ctx *c, const double *q);  // sets c->force for the next direct RHS evaluation
bool closure_in_pass(const cruna_ctx *c);           // the fused pass G evaluates the closure itself
// discrete adjoint (discrete_adjoint.cu)
void rhs_direct_vjp(cruna_ctx *c, const double *q, const double *lam, double *mu, double *gf_acc);
void step_direct_vjp(cruna_ctx *c, const double *q0, const double *lam1, double *lam0, double *gf_acc,
                     int nt);
void add_fields(cruna_ctx *c, double *dst, const double *src, long long n);

// kernel timing helpers (capi.cu)
int prof_begin(cruna_ctx *c, const char *name);
void prof_end(cruna_ctx *c, int idx);
void prof_drain(cruna_ctx *c);
// one kernel family's launch: an NVTX range on the host (visible to a timeline profiler; the calls
// do nothing without one) and, while kernel timing is on, CUDA events on the context's stream
struct ProfScope {
  cruna_ctx *c;
  int idx;
  ProfScope(cruna_ctx *ctx, const char *name) : c(ctx), idx(prof_begin(ctx, name)) { nvtxRangePushA(name); }
  ~ProfScope() {
    prof_end(c, idx);
    nvtxRangePop();
  }
};

}  // namespace cruna

#define CRUNA_CUDA_CHECK(call)                                                     \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e_) \
                               + " at " + __FILE__ + ":" + std::to_string(__LINE__)); \
    }                                                                              \
  } while (0)

#define CRUNA_LAUNCH_CHECK(ctx)                                                   \
  do {                                                                            \
    (ctx)->launches++;                                                            \
    CRUNA_CUDA_CHECK(cudaGetLastError());                                         \
  } while (0)
