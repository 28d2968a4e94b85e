/*
 * cruna_b200.h -- C ABI of the B200 (sm_100a) implementation of CRUNA's direct and adjoint
 * compressible Navier-Stokes time step.
 *
 * Every entry point replaces one Fortran module procedure of CRUNA (cruna-toolkit/public); the
 * procedure it stands in for is cited beside it as file:line.  A Fortran host binds these with
 * iso_c_binding (one interface block per entry point, arguments passed by value or as c_ptr);
 * Python binds them with ctypes.
 *
 * Conventions
 *  - Arrays are Fortran-ordered (column-major) and contiguous: a field is f(n1,n2,n3), a state is
 *    q(n1,n2,n3,5) holding (rho, rho*u, rho*v, rho*w, p) -- src/data/data_rhs.f90:3-4.
 *  - Functions without a suffix take HOST pointers; they copy in, run on the context's stream and
 *    copy out before returning.  Functions ending in _dev take DEVICE pointers (on the context's
 *    device) and only enqueue work on the context's stream (cruna_sync waits for it).
 *  - Every function returns 0 on success and a negative CRUNA_ERR_* code on failure;
 *    cruna_last_error() gives the message.  The reference prints and calls stop_cruna instead
 *    (src/parallelism/mpi_cartesian.f90:327-336); a Fortran shim maps a non-zero status to stop_cruna.
 *  - One context = one device, one CUDA stream, one grid; a context is not thread-safe (the
 *    reference keeps the same state in module SAVE variables).
 */
#ifndef CRUNA_B200_H
#define CRUNA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CRUNA_ABI_VERSION 2

/* status codes */
#define CRUNA_OK 0
#define CRUNA_ERR_ARG (-1)       /* invalid argument, shape or configuration */
#define CRUNA_ERR_CUDA (-2)      /* a CUDA runtime call failed */
#define CRUNA_ERR_NOMEM (-3)     /* device allocation failed */
#define CRUNA_ERR_STATE (-4)     /* non-finite or non-physical state detected (rho <= 0, p <= 0, NaN) */
#define CRUNA_ERR_UNSUPPORTED (-5) /* boundary type / scheme / path not available */
#define CRUNA_ERR_NODEVICE (-6)  /* no CUDA device */
#define CRUNA_ERR_IO (-7)        /* a snapshot / restart file could not be opened, written, renamed or read,
                                    or is not a file of this library */
#define CRUNA_STOPPED 1          /* cruna_run_hpc: stopped by its wall-time or step budget after storing
                                    a snapshot and the restart file (not an error) */

/* derivative cores (selected at compile time in CRUNA by discretisation_x_core.f90) */
enum cruna_diff_scheme {
  CRUNA_DIFF_EMPTY = 0,          /* src/diff/diff_pen_core_empty.f90 */
  CRUNA_DIFF_O2_E_C_O = 1,       /* src/diff/diff_pen_core_o2_e_c_o.f90 */
  CRUNA_DIFF_O4_E_C_P = 2,       /* src/diff/diff_pen_core_o4_e_c_p.f90 */
  CRUNA_DIFF_O4_E_C_O = 3,       /* src/diff/diff_pen_core_o4_e_c_o.f90 */
  CRUNA_DIFF_O4_I_C_P_PADE = 4,  /* src/diff/diff_pen_core_o4_i_c_p_pade.f90 */
  CRUNA_DIFF_O4_I_C_O_PADE = 5,  /* src/diff/diff_pen_core_o4_i_c_o_pade.f90 */
  CRUNA_DIFF_O6_I_C_P = 6,       /* src/diff/diff_pen_core_o6_i_c_p.f90 */
  CRUNA_DIFF_O6_I_C_O = 7,       /* src/diff/diff_pen_core_o6_i_c_o.f90 */
  CRUNA_DIFF_O8_E_C_P = 8        /* no reference counterpart: 8th-order explicit central, periodic */
};

/* filter cores (filter_x_core.f90 selector in CRUNA) */
enum cruna_filter_scheme {
  CRUNA_FILTER_EMPTY = 0,        /* src/filter/filter_pen_core_empty.f90 */
  CRUNA_FILTER_O2_I_C_P = 1,     /* src/filter/filter_pen_core_o2_i_c_p.f90 */
  CRUNA_FILTER_O6_I_C_P = 2,     /* src/filter/filter_pen_core_o6_i_c_p.f90 */
  CRUNA_FILTER_O2_I_C_O = 3,     /* src/filter/filter_pen_core_o2_i_c_o.f90 */
  CRUNA_FILTER_O4_I_C_O = 4,     /* src/filter/filter_pen_core_o4_i_c_o.f90 */
  CRUNA_FILTER_O6_I_C_O = 5,     /* src/filter/filter_pen_core_o6_i_c_o.f90 */
  CRUNA_FILTER_O8_I_C_O = 6,     /* src/filter/filter_pen_core_o8_i_c_o.f90 */
  CRUNA_FILTER_O10_I_C_O = 7,    /* src/filter/filter_pen_core_o10_i_c_o.f90 */
  CRUNA_FILTER_O10_E_C_P = 8     /* no reference counterpart: explicit 10th-order periodic, blended */
};

/* arithmetic of the stencil / flux / filter work (the RK accumulation is FP64 in both) */
enum cruna_precision {
  CRUNA_FP64 = 0,                /* plain path: everything FP64 */
  CRUNA_FP32_STENCIL = 1         /* stencils, fluxes and filters in FP32 on FP64-stored state */
};

/*
 * Solver configuration: the hot-path keys of parameter.dat (src/parameter/parameter.f90:100-170,
 * ns_rho_rhou_p_trafos.f90, filter cores, shape_functions.f90) as one struct.
 */
typedef struct cruna_config {
  int32_t abi_version;           /* must be CRUNA_ABI_VERSION */
  int32_t n[3];                  /* geom.n1, geom.n2, geom.n3 */
  double x0[3];                  /* geom.x10, geom.x20, geom.x30 */
  double x1[3];                  /* geom.x11, geom.x21, geom.x31 */
  int32_t diff[3];               /* enum cruna_diff_scheme per direction */
  int32_t filter[3];             /* enum cruna_filter_scheme per direction */
  double filter_alpha;           /* filter.alpha */
  double filter_strength;        /* blend strength of CRUNA_FILTER_O10_E_C_P */
  int32_t di_freq[3];            /* filter.di1freq..di3freq (direct loop), <= 0 means never */
  int32_t ai_freq[3];            /* filter.ai1freq..ai3freq (adjoint loop), <= 0 means never */
  double gamma, R, W, mu0, T0, Pr; /* material.* */
  double dt;                     /* time.dt */
  int32_t heat_flux_dx;          /* 0: as the reference, heat-flux Dx calls use dx=1
                                    (ns_rho_rhou_p.f90:189-197); 1: scale them by the grid spacing */
  int32_t precision;             /* enum cruna_precision */
  double sponge_length[3];       /* sponge.length(1..3); <= 0 disables that direction */
  double sponge_amplitude;       /* sponge.amplitude */
  int32_t sponge_shape;          /* sponge.shape: 0 quadratic, 1 cos */
  int32_t device;                /* CUDA device ordinal */
  int32_t check_every;           /* >0: run-loops check rho>0, p>0, finiteness every N steps */
  int32_t kvector;               /* sponge.kvector for the zonal BC types 202/203/205/206
                                    (boundary_conditions.f90:414-420): 0 diagonal, 1 orthogonal,
                                    2 hedgehog (boundary_normal_vector.f90:37-261) */
} cruna_config;

typedef struct cruna_ctx cruna_ctx;

/* Fills *cfg with the reference's defaults (material.R = 8.3144598, W = 0.0289647, T0 = 273,
   Pr = 0.71, filter.alpha = 0.35, sponge length 0.3, amplitude 1, quadratic, ...). */
void cruna_config_defaults(cruna_config *cfg);

/*
 * Create a context: grid, dx rule (src/geometry/grid_transform.f90:40-56), LAPACK-identical
 * tridiagonal factors of every compact core (the SAVE'd dgttrf factors, e.g.
 * diff_pen_core_o6_i_c_p.f90:170-228), the sponge shape (shape_functions.f90:69-150) and the
 * boundary table.  bc_table holds nbc rows of 10 doubles
 * (type, is, ie, js, je, ks, ke, k1, k2, k3) with 1-based inclusive global indices, i.e.
 * boundary_conditions_array after init_boundary_conditions_array / modify_boundary_conditions_array
 * (boundary_conditions.f90:461-610).  Supported types: 0, 100, 200, 201, 204, 400, 401.
 */
int cruna_init(const cruna_config *cfg, const double *bc_table, int nbc, cruna_ctx **out);
void cruna_free(cruna_ctx *ctx);
const char *cruna_last_error(const cruna_ctx *ctx);   /* ctx may be NULL (init failures) */
int cruna_sync(cruna_ctx *ctx);
int cruna_get_dx(const cruna_ctx *ctx, double dx[3]);
/* The context's cudaStream_t as an opaque pointer (for callers that interleave their own work). */
void *cruna_stream(cruna_ctx *ctx);

/* data_reference qref (src/data/data_reference.f90): target of BC 201/204 and the sponges. */
int cruna_set_reference(cruna_ctx *ctx, const double *qref);
int cruna_set_reference_dev(cruna_ctx *ctx, const double *qref);

/* apply_force(rhs) (src/opt/force.f90:27-31): rhs += f after the interior RHS; f (n1,n2,n3,5);
   NULL clears the forcing. */
int cruna_set_forcing(cruna_ctx *ctx, const double *f);
int cruna_set_forcing_dev(cruna_ctx *ctx, const double *f);

/* Dx1/Dx2/Dx3(q_x, q, h) (src/diff/diff_i1_mpi_cartesian.f90:17-132) on nfields consecutive fields;
   dir = 1, 2 or 3; h <= 0 or NaN means "h not present" (dx = 1.0, diff_i1_mpi_cartesian.f90:93-97). */
int cruna_diff(cruna_ctx *ctx, int dir, const double *in, double *out, int nfields, double h);
int cruna_diff_dev(cruna_ctx *ctx, int dir, const double *in, double *out, int nfields, double h);

/* filter_i1/2/3(q) (src/filter/filter_i1_mpi_cartesian.f90:18-97) in place on nfields fields. */
int cruna_filter(cruna_ctx *ctx, int dir, double *q, int nfields);
int cruna_filter_dev(cruna_ctx *ctx, int dir, double *q, int nfields);

/* right_hand_side_direct_3d(rhs, q_in, t) -- src/equations/ns_rho_rhou_p.f90:31-253 */
int cruna_rhs_direct(cruna_ctx *ctx, const double *q, double *rhs, double t);
int cruna_rhs_direct_dev(cruna_ctx *ctx, const double *q, double *rhs, double t);

/* right_hand_side_adjoint_3d(rhs, qs_in, q, g, t) -- ns_rho_rhou_p.f90:257-536 (continuous,
   inviscid adjoint as in CRUNA); g may be NULL (zero). */
int cruna_rhs_adjoint(cruna_ctx *ctx, const double *qs, const double *q, const double *g,
                      double *rhs, double t);
int cruna_rhs_adjoint_dev(cruna_ctx *ctx, const double *qs, const double *q, const double *g,
                          double *rhs, double t);

/* time_stepper_direct(q1, q0, t) -- src/time/rk_o4_e.f90:17-58 (classical RK4) */
int cruna_step_direct(cruna_ctx *ctx, const double *q0, double *q1, double t);
int cruna_step_direct_dev(cruna_ctx *ctx, const double *q0, double *q1, double t);

/* time_stepper_adjoint(qs1, qs0, q0, g, t) -- rk_o4_e.f90:62-105 (dt -> -dt, q0 frozen) */
int cruna_step_adjoint(cruna_ctx *ctx, const double *qs0, const double *q0, const double *g,
                       double *qs1, double t);
int cruna_step_adjoint_dev(cruna_ctx *ctx, const double *qs0, const double *q0, const double *g,
                           double *qs1, double t);

/* set_boundary_condition_q(q, outside_rhs)      boundary_conditions.f90:52-136
   set_boundary_condition_qs(qs, q, outside_rhs) boundary_conditions.f90:140-224
   set_boundary_condition_rhs(rhs, q)            boundary_conditions.f90:228-298
   set_boundary_condition_rhss(rhss, qs, q)      boundary_conditions.f90:302-377 (q may be NULL,
                                                 as in the NS adjoint RHS; a 400 sponge is then off) */
int cruna_bc_q(cruna_ctx *ctx, double *q, int outside_rhs);
int cruna_bc_qs(cruna_ctx *ctx, double *qs, const double *q, int outside_rhs);
int cruna_bc_rhs(cruna_ctx *ctx, double *rhs, const double *q);
int cruna_bc_rhss(cruna_ctx *ctx, double *rhss, const double *qs, const double *q);
int cruna_bc_q_dev(cruna_ctx *ctx, double *q, int outside_rhs);
int cruna_bc_qs_dev(cruna_ctx *ctx, double *qs, const double *q, int outside_rhs);
int cruna_bc_rhs_dev(cruna_ctx *ctx, double *rhs, const double *q);
int cruna_bc_rhss_dev(cruna_ctx *ctx, double *rhss, const double *qs, const double *q);

/*
 * Loop body of calc_direct (src/main/computation_direct.f90:64-107), nsteps steps starting after
 * step nt0: time_stepper_direct -> set_boundary_condition_q(outside_rhs) -> filter_i1/2/3 when
 * mod(nt, di_freq) == 0.  q_io holds q0 on entry and q(nt0+nsteps) on return.  traj, if not NULL,
 * receives the state after every step: traj[(s)*N*5 ...] for s = 0..nsteps-1 (the Q(:,:,:,:,nt)
 * store of computation_direct.f90:102).
 */
int cruna_run_direct(cruna_ctx *ctx, double *q_io, int nt0, int nsteps, double *traj);
int cruna_run_direct_dev(cruna_ctx *ctx, double *q_io, int nt0, int nsteps, double *traj);

/*
 * Loop body of calc_adjoint (src/main/computation_adjoint.f90:60-108) for nt = nt_end..nt_end-nsteps+1:
 * q0 = Q(nt), g = calc_objective_g(q0) (here: the caller's g_traj slice or zero), adjoint step,
 * set_boundary_condition_qs(outside_rhs), filters when mod(nt, ai_freq) == 0.  Q_traj holds the
 * direct states Q(nt_end-nsteps+1 .. nt_end) in that order; g_traj the matching sources (or NULL).
 */
int cruna_run_adjoint(cruna_ctx *ctx, double *qs_io, const double *Q_traj, const double *g_traj,
                      int nt_end, int nsteps);
int cruna_run_adjoint_dev(cruna_ctx *ctx, double *qs_io, const double *Q_traj, const double *g_traj,
                          int nt_end, int nsteps);

/*
 * Objectives and gradients of CRUNA's optimisation loop (src/main/cruna.f90:78-179): calc_direct,
 * calc_objective, calc_adjoint with calc_objective_g as the adjoint source, calc_grad.  The reference
 * leaves objective and gradient to each case (src/opt/objective.f90:19-45, src/opt/force.f90:41-45);
 * these are the library's built-in ones:
 *   CRUNA_OBJ_PLANE_P2       J = sum_{nt=1..T} dt * sum_{plane x_normal = index} dA (p - p_inf)^2,
 *                            adjoint source g = (0,0,0,0, 2 dA (p - p_inf)) on the plane
 *   CRUNA_OBJ_KINETIC_ENERGY J = sum dV |rho u|^2 / (2 rho) at the final time, qs(T) = dJ/dq
 *   CRUNA_OBJ_ENSTROPHY      J = sum dV |curl u|^2 / 2 at the final time (the curl taken with the
 *                            context's derivative operators, h = dx), qs(T) = dJ/dq (through the
 *                            transposed operators)
 */
enum cruna_objective_kind { CRUNA_OBJ_PLANE_P2 = 1, CRUNA_OBJ_KINETIC_ENERGY = 2, CRUNA_OBJ_ENSTROPHY = 3 };
typedef struct cruna_objective {
  int32_t kind;       /* enum cruna_objective_kind */
  int32_t normal;     /* plane normal direction 1..3 (CRUNA_OBJ_PLANE_P2) */
  int32_t index;      /* 1-based plane index */
  int32_t reserved;
  double p_inf;       /* reference pressure */
} cruna_objective;

/* Volume diagnostics of a state: kinetic energy sum dV |rho u|^2 / (2 rho) and enstrophy
   sum dV |curl u|^2 / 2 (either output pointer may be NULL); deterministic reductions. */
int cruna_diagnostics(cruna_ctx *ctx, const double *q, double *kinetic_energy, double *enstrophy);
int cruna_diagnostics_dev(cruna_ctx *ctx, const double *q, double *kinetic_energy, double *enstrophy);

/* J, dJ/df for the time-constant forcing set by cruna_set_forcing (the time integral of the adjoint
   state, trapezoid rule) and dJ/dq0 = qs(0), from nsteps direct steps and the matching adjoint steps
   of the run loops above.  The direct trajectory is recomputed from nsnap snapshots held in HBM
   (binomial schedule, minimal recomputation; nsnap > nsteps keeps every state); *direct_steps
   receives the number of direct steps executed.  grad_f / grad_q0 may be NULL. */
int cruna_gradient(cruna_ctx *ctx, const double *q0, int nsteps, int nsnap, const cruna_objective *obj, double *J,
                   double *grad_f, double *grad_q0, int64_t *direct_steps);
/* Where cruna_gradient keeps its nsnap snapshots: 0 = HBM (default), 1 = pinned host memory (copied
   over PCIe when stored and restored; frees nsnap states of HBM for grids whose states fill the GPU).
   Pinned slots stay allocated on the context for later gradient calls until it is freed or this is
   set back to 0.  In the _dev variant grad_q0 may alias q0: q0 is read only before the first step. */
int cruna_set_snapshot_memory(cruna_ctx *ctx, int host);
int cruna_gradient_dev(cruna_ctx *ctx, const double *q0, int nsteps, int nsnap, const cruna_objective *obj,
                       double *J, double *grad_f, double *grad_q0, int64_t *direct_steps);

/* z-slab decomposition (replaces the reference's MPI pencil transposes, transpose_mpi_cartesian.f90,
   for runs over several GPUs): the context holds one slab of the global grid extended by H >= 2R halo
   planes on each side (n3 = nz_local + 2H, periodic z scheme of half-width R), and before every pass
   that reads z-neighbours (each RK stage of the direct and adjoint steps, the frozen direct state of
   an adjoint step, the z filter) the library calls fn(user, fields, nfields, stream): it must refresh
   the H lowest and H highest planes of each of the nfields fields (device pointer, Fortran layout)
   with the neighbouring slabs' interior planes, ordered on `stream` (a cudaStream_t).  Interior results
   are then exactly the single-domain ones; halo planes hold no meaningful values between calls.
   fn returns 0 on success.  NULL detaches. */
int cruna_set_halo_exchange(cruna_ctx *ctx, int (*fn)(void *user, double *fields, int nfields, void *stream),
                            void *user);

/* Adjoint used by cruna_gradient: 0 = the reference's continuous inviscid adjoint step
   (right_hand_side_adjoint_3d, ns_rho_rhou_p.f90:257-536, integrated by time_stepper_adjoint,
   rk_o4_e.f90:62-105; the default), 1 = the exact discrete adjoint (no counterpart in the reference):
   the transpose of the direct loop step, so dJ/dq0 and dJ/df are the exact derivatives of the J the
   direct loop produces.  Mode 1 needs precision CRUNA_FP64; it runs the generic line-operator kernels
   and keeps about 160 doubles per grid point of device memory. */
int cruna_set_adjoint_mode(cruna_ctx *ctx, int mode);

/* Discrete adjoint of right_hand_side_direct_3d (ns_rho_rhou_p.f90:31-253; no counterpart in the
   reference): mu = (d rhs/d q)^T lam at q, through the BC on q, every derivative, the viscous terms,
   the forcing and the BC on the RHS.  grad_f (may be NULL) is accumulated with (d rhs/d f)^T lam. */
int cruna_rhs_direct_vjp(cruna_ctx *ctx, const double *q, const double *lam, double *mu, double *grad_f);
int cruna_rhs_direct_vjp_dev(cruna_ctx *ctx, const double *q, const double *lam, double *mu, double *grad_f);

/* Discrete adjoint of loop step nt of calc_direct (computation_direct.f90:64-107: time_stepper_direct,
   BC on q outside the RHS, filters when mod(nt, freq) == 0) at its input q0 (no counterpart in the
   reference): lam0 = (d q1/d q0)^T lam1; grad_f (may be NULL) accumulates (d q1/d f)^T lam1.
   lam0 may alias lam1. */
int cruna_step_direct_vjp(cruna_ctx *ctx, const double *q0, const double *lam1, double *lam0, double *grad_f,
                          int nt);
int cruna_step_direct_vjp_dev(cruna_ctx *ctx, const double *q0, const double *lam1, double *lam0,
                              double *grad_f, int nt);

/* ---- learned subgrid closure (no counterpart in the reference: CRUNA has no learned component) ----
   An MLP 12 -> 64 -> 64 -> 6 (GELU) from normalised features (the 9 velocity-gradient components
   du_i/dx_j in the order (u_x, u_y, u_z, v_x, ..., w_z), density, temperature, filter width) to the 6
   subgrid-stress components (tau_11, tau_22, tau_33, tau_12, tau_13, tau_23).  FP32 master parameters
   (order W1[64][12], b1[64], W2[64][64], b2[64], W3[6][64], b3[6]); the kernels run BF16 operands with
   FP32 accumulation on the tcgen05 tensor cores.  X is n x 12 and Y n x 6, row-major FP32 device
   arrays; outputs are in physical units (network output times out_scale). */
#define CRUNA_MLP_NPARAMS 5382
typedef struct cruna_mlp cruna_mlp;
int cruna_mlp_create(int device, uint64_t seed, cruna_mlp **out);
void cruna_mlp_free(cruna_mlp *mlp);
const char *cruna_mlp_last_error(const cruna_mlp *mlp);
int cruna_mlp_set_params(cruna_mlp *mlp, const float *params);   /* host array, resets Adam state */
int cruna_mlp_get_params(cruna_mlp *mlp, float *params);
/* x_normalised = (x - in_mean) / in_scale; y = network output * out_scale */
int cruna_mlp_set_scaling(cruna_mlp *mlp, const float *in_mean, const float *in_scale, const float *out_scale);
int cruna_mlp_forward_dev(cruna_mlp *mlp, const float *X, float *Y, long long n);
/* loss = mean over n x 6 of (y/out_scale - Y/out_scale)^2 and its gradient (host, 5382 floats);
   n a multiple of 128 */
int cruna_mlp_grad_dev(cruna_mlp *mlp, const float *X, const float *Y, int n, float *grad, float *loss);
/* Adam (lr, beta 0.9 / 0.999, eps 1e-8) over `steps` mini-batches of `batch` samples (a multiple of
   128) drawn without replacement per epoch (seeded shuffle); loss_hist (host, steps floats) may be NULL */
int cruna_mlp_train_dev(cruna_mlp *mlp, const float *X, const float *Y, long long n, int batch, int steps,
                        float lr, uint64_t seed, float *loss_hist);

/* Box filter of a fine state by `factor` in every direction with more than one point (grid sizes
   divisible by it): q_coarse (5 fields on the coarse grid) holds the means of rho, rho u_i and p; tau
   (n_coarse x 6 floats, point-major, point order i fastest) the Favre subgrid stresses
   mean(rho u_i u_j) - mean(rho u_i) mean(rho u_j) / mean(rho).  ctx is the fine grid's context. */
int cruna_box_filter_dev(cruna_ctx *ctx, int factor, const double *q, double *q_coarse, float *tau);
/* Closure features of a coarse state (n x 12 floats, point-major): du_i/dx_j with the context's
   derivative scheme, rho, T, delta. */
int cruna_closure_features_dev(cruna_ctx *ctx, const double *q, double delta, float *X);
/* Scale-free closure (0 default, 1 on): with g = |grad u| (Frobenius norm of the coarse velocity
   gradient) at each point, features 0..8 become grad u / g and feature 11 becomes g * delta, and the
   network's outputs are read as tau_ij / (rho (g delta)^2) and multiplied back.  Affects
   cruna_closure_features_dev and the closure inside the RHS; a network trained on normalised pairs
   then carries over while the flow decays. */
int cruna_set_closure_normalisation(cruna_ctx *ctx, int on);
/* Attach (mlp != NULL) or detach the closure: every direct RHS evaluation of ctx then adds
   -d_j tau_ij(model) to the momentum equations, on top of the forcing set with cruna_set_forcing.  The
   MLP must outlive the attachment; the discrete adjoint (mode 1) is unavailable while attached. */
int cruna_set_closure(cruna_ctx *ctx, cruna_mlp *mlp, double delta);
/* Where the attached closure runs on the fused (explicit-scheme) RHS path: on = 1 (default) inside the
   flux pass -- the pass that forms the viscous stresses evaluates the network on the tensor cores for
   each plane tile of 128 points (features from its own velocity gradients, BF16 operands, FP32
   accumulators in TMEM) and subtracts the model stresses from the stresses it writes, so the
   divergence pass differentiates both at once; on = 0 as separate launches (features, network, stress
   divergence) through the forcing hook.  The generic path always uses the separate launches.  Both
   agree up to the BF16 rounding of the network's inputs. */
int cruna_set_closure_fused(cruna_ctx *ctx, int on);

/* J of the objective after nsteps direct loop steps from q0 (calc_direct + calc_objective,
   cruna.f90:90-117), without the adjoint: what finite-difference checks and line searches evaluate. */
int cruna_objective_value(cruna_ctx *ctx, const double *q0, int nsteps, const cruna_objective *obj, double *J);
int cruna_objective_value_dev(cruna_ctx *ctx, const double *q0, int nsteps, const cruna_objective *obj,
                              double *J);

/* Optimisation loop of cruna.f90:78-179 on a time-constant forcing f (5 fields, updated in place):
   per loop the direct run and J (J_hist[loop-1]); except in the last loop the gradient dJ/df
   (cruna_gradient with the context's adjoint mode, nsnap snapshots), for loop >= ls_start the
   quadratic line search of ls_quadratic_fit (line_search.f90:23-127: J at alpha0/2 and alpha0, dgesv
   of [alpha^2, alpha, 1], alpha = -b/2a capped at 10 alpha0, alpha0 when singular; alpha_hist), and
   update_force as steepest descent f <- f - alpha dJ/df (force.f90:76-81 leaves the update to the
   case).  The context's own forcing is restored afterwards.  J_hist (maxloop) and alpha_hist
   (maxloop - 1) are host arrays and may be NULL. */
int cruna_optimize(cruna_ctx *ctx, const double *q0, const cruna_objective *obj, int nsteps, int nsnap,
                   int maxloop, int ls_start, double alpha0, double *f, double *J_hist, double *alpha_hist);
int cruna_optimize_dev(cruna_ctx *ctx, const double *q0, const cruna_objective *obj, int nsteps, int nsnap,
                       int maxloop, int ls_start, double alpha0, double *f, double *J_hist, double *alpha_hist);

/* State check used by the run loops: returns CRUNA_ERR_STATE if any rho <= 0, p <= 0 or a
   non-finite value is found in q (device pointer). */
int cruna_check_state_dev(cruna_ctx *ctx, const double *q);

/* Which RHS implementation the context uses: 1 = fused explicit kernels, 0 = generic line-operator
   sequence (compact schemes, 204/200 boundary types).  force_generic=1 selects the generic one. */
int cruna_rhs_path(const cruna_ctx *ctx);
int cruna_set_force_generic(cruna_ctx *ctx, int force_generic);
/* FP64 fused adjoint pass: on = 1 feeds it by TMA (cp.async.bulk.tensor tiles, column boxes and RK
   inputs into shared memory, z columns in registers) where the layout allows it (n1 even, 16-byte
   aligned states); on = 0 (default) keeps the per-thread-load kernel, which measures faster on B200
   (1.35 against 1.40 ms per launch at 256^3).  Both give the same results to rounding. */
int cruna_set_tma_passes(cruna_ctx *ctx, int on);

/* Number of kernels this library enqueued since the context was created (for launch accounting). */
int64_t cruna_kernel_launches(const cruna_ctx *ctx);

/* Allocation-free direct RHS.  No counterpart in the reference: it exists for callers that cannot
   allocate device memory where they evaluate the RHS -- a host whose device memory belongs to
   another allocator (a framework's caching pool) or a time loop that must keep a fixed footprint
   decided at start-up -- and therefore cannot create a context (cruna_init allocates).
   It evaluates right_hand_side_direct_3d for the explicit derivative cores (FP64, no boundary table,
   no forcing) from cfg alone: q and rhs are device pointers (n1*n2*n3*5 doubles each) on the
   current device and the work is enqueued on `stream` (a cudaStream_t, NULL = default stream).
   Its intermediate (15 doubles per point) is a static device array of 131072 points (15.7 MB) that
   every GPU loading the library keeps until exit; larger grids are rejected with CRUNA_ERR_ARG.
   Every call resolves that array's address in the current context and sets the two kernels'
   shared-memory limit (neither allocates).  The first call on a device also loads the library's
   device code there; with lazy module loading that is when the array is mapped, so that call can fail
   for lack of memory: make it at start-up, before any stream capture.  All calls share the array, so
   calls that overlap on the GPU race; serialise them (one stream, or events).  Each call overwrites
   every intermediate value it reads.  A CUDA error already pending on the calling thread is reported
   (CRUNA_ERR_CUDA) and left pending, and nothing is launched.  On failure a message is written to
   errbuf (errlen bytes, may be NULL). */
int cruna_rhs_direct_noalloc(const cruna_config *cfg, const double *q, double *rhs, void *stream, char *errbuf,
                             int errlen);

/*
 * Snapshot / restart files and the direct main loop with restart (src/main/cruna_hpc.f90:99-299).
 * The reference writes HDF5 (src/io/hdf5_single.f90:659-774: dataset "data" (n1,n2,n3,5) FP64 plus
 * "params"); this library writes the same content in a flat binary container under the reference's
 * file names (src/helper/io_helper.f90:11-15, 426-432) with ".bin" in place of ".h5":
 *   data_direct_snapshot__BB_IIIII_SS_TTTTTTT.bin   (world block, block image, subset, time step)
 *   restartfile.bin                                 (the int32 pair (ns, nt) of the last restart point)
 * Layout: 64-byte header (magic "CRUNAB2D", int32 version 1, int32 element size 8 or 4, int64 dims[4],
 * int64 params length, int64 0), the params text ("key = value" lines), the data in Fortran order.
 * Files are written to "<name>.tmp" and renamed.  A file that cannot be opened, written, renamed or
 * read, or that is not a file of this library, gives CRUNA_ERR_IO; bad arguments and a shape that differs
 * from the expected one give CRUNA_ERR_ARG.  Context-free functions report errors through
 * cruna_last_error(NULL).
 */
/* Writes the file name of `type` ("data_direct_snapshot", "data_adjoint_snapshot", "data_direct",
   "data_adjoint", "restartfile") into buf; returns its length (or a negative error). */
int cruna_io_fname(char *buf, int buflen, const char *workdir, const char *type, int world_block, int block_image,
                   int ns, int nt);
/* store_4d_rk (hdf5_single.f90:659-774) / its load: dims = Fortran shape; on read, dims is checked against
   the file when data is non-NULL, else filled from it (params, if given, receives the params text). */
int cruna_write_snapshot(const char *path, const int64_t dims[4], const double *data, const char *params);
int cruna_read_snapshot(const char *path, int64_t dims[4], double *data, char *params, int params_len);
/* restartfile with (ns, nt) (cruna_hpc.f90:196-199); read returns 1 when found, 0 when the file does not
   exist (the reference then starts from 0, :127-131), negative on error */
int cruna_write_restart(const char *workdir, int ns, int nt);
int cruna_read_restart(const char *workdir, int *ns, int *nt);
/* First subset and step after a restart point (cruna_hpc.f90:143-145):
   nt_total = (ns-1)*steps + nt + 1, s0 = nt_total/steps + 1, nt0 = nt_total - (s0-1)*steps. */
int cruna_restart_start(int ns, int nt, int steps, int *s0, int *nt0);
/* data_direct_snapshot of the context's grid at (ns, nt) from / to a HOST state (n1*n2*n3*5 doubles). */
int cruna_store_snapshot(cruna_ctx *ctx, const char *workdir, const char *type, const double *q, int ns, int nt);
int cruna_load_snapshot(cruna_ctx *ctx, const char *workdir, const char *type, double *q, int ns, int nt);

typedef struct cruna_hpc_opts {
  const char *workdir;   /* io.workdirectory (NULL or "" = ".") */
  int32_t steps;         /* time.steps: steps per subset */
  int32_t subsets;       /* time.subsets */
  int32_t dsfreq;        /* io.dsfreq: snapshot + restart file every dsfreq steps, and the initial and
                            final snapshots; <= 0: no files except at a budget stop */
  int32_t restart;       /* init.restart: continue from restartfile.bin when it exists */
  double walltime;       /* run.walltime in seconds of elapsed time (the reference: hours of CPU time);
                            <= 0: none */
  int32_t max_steps;     /* steps this call may take (<= 0: unlimited); reaching it acts like the wall time */
  int32_t reserved;
} cruna_hpc_opts;
/* The direct main loop of cruna_hpc (cruna_hpc.f90:99-299): store the initial condition as snapshot
   (1, 0), on restart load (ns, nt) from restartfile.bin and the matching snapshot, then run the subset
   and step loops from cruna_restart_start (time_stepper_direct, BC q outside, filters on the step index
   within the subset), storing a snapshot and the restart file every dsfreq steps; when the wall-time or
   step budget runs out before the end, store both at the current step and return CRUNA_STOPPED.  As in
   the reference, nt0 applies to every subset after a restart.  q_io (HOST) holds the initial condition
   on entry and the last state on return; *ns_out / *nt_out receive the last (subset, step) done. */
int cruna_run_hpc(cruna_ctx *ctx, double *q_io, const cruna_hpc_opts *opts, int *ns_out, int *nt_out);

/* Kernel timing: while enabled, each kernel family (fused passes, filters, stage updates, generic
   line operators) is bracketed by CUDA events on the context's stream.  cruna_profile_report drains
   them and writes lines "name launches total_ms" into buf; it returns the length of the full report. */
int cruna_profile_enable(cruna_ctx *ctx, int on);
int cruna_profile_report(cruna_ctx *ctx, char *buf, int buflen);

/* Step graphs: inside one call of cruna_run_direct*, cruna_run_adjoint*, cruna_gradient*,
   cruna_objective_value* or cruna_optimize*, a loop step (time step, boundary update and the filters
   due at that step) that repeats with the same buffers and filter pattern is recorded once as a CUDA
   graph on the context's stream and replayed after that; the first step of each kind runs eagerly.
   Results are bit-identical to eager launches.  Graphs are on by default and off while kernel timing
   or a halo exchange is set; a capture the runtime refuses turns them off for the rest of the call
   and the step runs eagerly.  cruna_graph_stats returns the counts of captures and of replays since
   the context was created (either pointer may be NULL). */
int cruna_set_graphs(cruna_ctx *ctx, int on);
int cruna_graph_stats(cruna_ctx *ctx, int64_t *captured, int64_t *replayed);

/* The library's restatement of LAPACK dgttrf / dgttrs('N', nrhs=1), which every compact core of the
   reference calls (e.g. diff_pen_core_o6_i_c_p.f90:135,213,219); exported so callers and tests can
   compare its factors with their LAPACK.  ipiv is 1-based as in LAPACK. */
int cruna_lapack_dgttrf(int n, double *dl, double *d, double *du, double *du2, int *ipiv);
void cruna_lapack_dgttrs(int n, const double *dl, const double *d, const double *du, const double *du2,
                         const int *ipiv, double *b);

#ifdef __cplusplus
}
#endif
#endif /* CRUNA_B200_H */
