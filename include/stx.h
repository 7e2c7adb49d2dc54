/*
 * stx.h -- C ABI of the B200 multi-species reacting step (libstx.so).
 *
 * The entry points replace the device work that the reference's GPU equation
 * object (src/multideal/multideal_gpu.F90, type equation_multideal_gpu_object,
 * :164-211) launches from its type-bound procedures.  Every array argument uses
 * the reference's own layout, so a Fortran host can pass its allocations as-is:
 *
 *   w      (1-ng:nx+ng, 1-ng:ny+ng, 1-ng:nz+ng, nv)      column-major, i fastest
 *   w_aux  (1-ng:nx+ng, 1-ng:ny+ng, 1-ng:nz+ng, nv_aux)
 *   fl, fln, fl_sav  (1:nx, 1:ny, 1:nz, nv)
 *   fluid_mask (1-ng:nx+ng, 1-ng:ny+ng, 1-ng:nz+ng) int32, 0 = fluid (may be NULL)
 *
 * with nv = ns+4 and the reference's index map (src/multideal/index_define.h):
 * species 1..ns, I_U..I_E = ns+1..ns+4; in w_aux the species mass fractions
 * 1..ns, J_U=ns+1, J_V, J_W, J_H, J_T, J_P, J_C, J_MU, J_DUC, J_DIV, J_R, J_Z,
 * J_K_COND=ns+13 and rho*D_k at ns+13+k.  Indices in arguments are the
 * reference's 1-based Fortran indices.
 *
 * All field pointers are device pointers; every call is asynchronous on the
 * caller's stream and allocates nothing on the device, except stx_ctx_create
 * (tables, scratch) and stx_compute_dt / stx_advance_solution_host, which say
 * so.  Return value: 0 on success, a negative STX_E_* code otherwise.  Kernels
 * never trap: iteration caps (Newton, Rosenbrock) set bits in the context's
 * device status word, read with stx_status().
 */
#ifndef STX_H
#define STX_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STX_ABI_VERSION 1

/* error codes */
#define STX_OK            0
#define STX_E_INVALID    -1   /* bad argument (null pointer, range, unsupported option) */
#define STX_E_CUDA       -2   /* a CUDA runtime call failed */
#define STX_E_NOMEM      -3   /* device allocation failed (stx_ctx_create only) */
#define STX_E_UNSUPPORTED -4  /* option outside the supported hot path (e.g. IBM, LES, NR BCs) */
#define STX_E_TOO_LARGE  -5   /* problem larger than the fixed scratch of stx_rosenbrock_krylov_noalloc */
#define STX_E_LOCAL_MEM  -6   /* stx_rosenbrock_krylov_noalloc: cudaLimitStackSize below the kernel's local frame */

/* status bits accumulated on the device (stx_status) */
#define STX_ST_NEWTON_CAP     0x1u  /* a Newton T(e) inversion hit its 10-iteration cap */
#define STX_ST_ROS_STEPS_CAP  0x2u  /* a Rosenbrock cell hit ros_maxsteps */
#define STX_ST_ROS_TRY_CAP    0x4u  /* a full-Jacobian Rosenbrock step exhausted ros_maxtry */
#define STX_ST_NONFINITE      0x8u  /* a non-finite value was produced */
#define STX_ST_WAIT_TIMEOUT   0x10u /* a kernel gave up waiting for its tensor-memory copies (the
                                       sweep's result is then incomplete); never expected */

/* Property tables: the arrays set_fluid_prop / set_fluid_prop_cantera build
 * (src/multideal/multideal.F90:2714-3318), in their Fortran layouts. */
typedef struct stx_tables {
  int32_t ns, nr;
  int32_t indx_cp_l, indx_cp_r, nsetcv, num_t_tab;
  double  t_min_tab, dt_tab, R_univ;
  const double *mw, *mwinv, *rgas;             /* (ns) */
  const double *trange;                        /* (ns, nsetcv+1) */
  const double *cp_coeff, *cv_coeff;           /* (indx_cp_l:indx_cp_r+2, ns, nsetcv), times R_k */
  const double *visc, *lambda;                 /* (num_t_tab+1, ns) */
  const double *diffbin;                       /* (num_t_tab+1, ns, ns), at p0 */
  const int32_t *reac_ty, *is_rev;             /* (nr) */
  const double *arr_a, *arr_b, *arr_ea;        /* (nr, 2), SI kmol units, Ea in J/kmol */
  const double *falloff;                       /* (nr, 5) */
  const double *tb_eff, *r_coeffs, *p_coeffs;  /* (nr, ns) */
  const double *kc_tab;                        /* (num_t_tab+1, nr), clamped to [tiny, huge] */
  /* Bilger mixture fraction (multideal.F90:955-1060); n_eoi == 1 gives Z = 0.5 */
  int32_t n_eoi;
  const double *aw_eoi, *coeff_eoi;            /* (n_eoi) */
  const int32_t *nainsp;                       /* (ns, n_eoi) */
  const double *beta0;                         /* (2) */
} stx_tables;

/* Grid: local coordinates and metrics (src/field.F90:300-347). */
typedef struct stx_grid {
  int32_t nx, ny, nz, ng;
  const double *x, *y, *z;                     /* (1-ng:n+ng) */
  const double *dcsidx, *detady, *dzitdz;      /* (n) = 1/dxg */
  const double *dcsidxs, *detadys, *dzitdzs;   /* (n) squares */
} stx_grid;

/* Numerics and controls (multideal.ini keys, bc_preproc, runge_kutta_initialize). */
typedef struct stx_params {
  int32_t nv_aux;
  double  p0, rho0, u0, eps_sensor, tol_iter_nr;
  int32_t ep_order, nkeep, weno_scheme, weno_version, flux_splitting;
  int32_t sensor_type, visc_order, conservative_viscous;
  double  sensor_threshold;
  int32_t bctags[6];                           /* xmin,xmax,ymin,ymax,zmin,zmax: 0 periodic, 1 free stream
                                                  (xmin), 2 extrapolation, 4 subsonic extrapolation at p0,
                                                  5 symmetry (y), 6 isothermal wall (y), 7 open outflow,
                                                  8 adiabatic wall */
  int32_t bctags_nr[6];                        /* characteristic treatment of the face (bc_nr): 0 none,
                                                  1 non-reflecting, 2 relaxed to the outer ghost, 3 relaxed
                                                  to winf, 6 reflecting wall */
  int32_t force_zero_flux[6];
  int32_t eul_imin, eul_imax, eul_jmin, eul_jmax, eul_kmin, eul_kmax;
  int32_t enable_chemistry;                    /* 0 off, 1 explicit source, 2 implicit Rosenbrock */
  int32_t rosenbrock_version;                  /* 1 full Jacobian, 2 ROK4 Krylov */
  int32_t operator_splitting;                  /* 1 "simpler", 2 Strang */
  int32_t ros_maxsteps, ros_maxtry;
  double  ros_eps;
  int32_t nrk;                                 /* 3: Wray RK3 */
  double  rhork[4], gamrk[4];
  const double *winf;                          /* (nv) free-stream state for bc tag 1, may be NULL */
  double  T_wall;                              /* wall temperature of bc tag 6 ([flow] T_wall) */
} stx_params;

/* Field set of one solve (all device pointers). */
typedef struct stx_fields {
  double *w, *w_aux, *fl, *fln, *fl_sav;       /* fl_sav only for operator_splitting == 1 */
  const int32_t *fluid_mask;                   /* may be NULL: every cell is fluid */
} stx_fields;

typedef struct stx_ctx stx_ctx;

/* Version of this ABI (STX_ABI_VERSION). */
int stx_abi_version(void);
/* Human-readable text of an STX_E_* code. */
const char *stx_strerror(int code);

/* Create a context on the current CUDA device: validates parameters, copies the
 * tables and the grid to device memory, allocates scratch.  Replaces the table
 * upload of multideal_gpu.F90:1361-1424 and the stream set-up of :1468. */
int stx_ctx_create(const stx_params *par, const stx_tables *tab, const stx_grid *grid, stx_ctx **out);
/* A context for another grid and parameter set on the same mechanism: it uses
 * base's device tables (no table upload or repacking) and has its own grid,
 * scratch, counters and status word; it starts in base's precision form
 * (stx_set_precision).  base must outlive every context created
 * from it.  No counterpart in the reference (one solve per process); for
 * callers that run many solves of one mechanism, e.g. a request server. */
int stx_ctx_create_like(const stx_ctx *base, const stx_params *par, const stx_grid *grid, stx_ctx **out);
/* stx_ctx_create_like with the context's uploads (grid, parameters, scratch
 * zero fills) enqueued on the caller's stream instead of waited for: the call
 * returns once its pageable host data has been staged, and the context may be
 * used at once on `stream`, on another stream after `stream` has reached this
 * point.  Nothing else is synchronised, so a server that admits a request while
 * other work runs on the device (seconds-long batched reactor launches) does
 * not wait for that work.  No counterpart in the reference. */
int stx_ctx_create_like_on(const stx_ctx *base, const stx_params *par, const stx_grid *grid, void *stream,
                           stx_ctx **out);
int stx_ctx_destroy(stx_ctx *ctx);

/* Ghost exchange with neighbouring subdomains (the MPI half of the reference's
 * bcswap, base_gpu.F90:1132-1264).  A face whose bctags entry is
 * STX_BC_EXCHANGE is an interface: the library neither swaps it periodically
 * nor applies a boundary condition to it.  After the local periodic swap of
 * every stx_bcswap call (and so of every swap inside stx_rk_sync,
 * stx_advance_solution and stx_update_ghost(do_swap = 1)) the library calls
 * fn(user, stream, field, nvar) with the swapped fields (nvar consecutive
 * ghosted fields) and the stream the call runs on; fn fills the interface
 * ghosts (enqueued on that stream, or done) and returns 0, or an error that
 * the library returns.  A context with an exchange cannot be captured
 * (stx_graph_create returns STX_E_UNSUPPORTED).  fn = NULL removes it. */
#define STX_BC_EXCHANGE (-1)
typedef int (*stx_exchange_fn)(void *user, void *stream, double *field, int nvar);
int stx_set_exchange(stx_ctx *ctx, stx_exchange_fn fn, void *user);

/* eval_aux_cuf (kernels_gpu.F90:6154-6308): species clip written back into w,
 * primitives, Newton T(e), c, Bilger Z, Mathur lambda, Wilke mu, Bird rho*D_k,
 * over the 1-based box [istart,iend]x[jstart,jend]x[kstart,kend]. */
int stx_eval_aux(stx_ctx *ctx, void *stream, double *w, double *w_aux,
                 int istart, int iend, int jstart, int jend, int kstart, int kend);
/* compute_aux (multideal_gpu.F90:361-443): central/ghost selection as in the reference. */
int stx_compute_aux(stx_ctx *ctx, void *stream, double *w, double *w_aux, int central, int ghost);
/* eval_aux2_cuf (kernels_gpu.F90:6310-6382): div/3 and the Ducros sensor. */
int stx_eval_aux2(stx_ctx *ctx, void *stream, double *w_aux);
/* bcextr_var_cuf (kernels_gpu.F90:5147-5207) on one ghosted scalar field. */
int stx_bcextr_var(stx_ctx *ctx, void *stream, double *var);
/* base_gpu%bcswap / bcswap_var (base_gpu.F90:1132-1264) on one GPU: periodic
 * self-exchange of the ng ghost layers of nvar consecutive ghosted fields. */
int stx_bcswap(stx_ctx *ctx, void *stream, double *field, int nvar);
/* update_ghost (multideal_gpu.F90:1165-1238): the ghost fills of every face's bc
 * tag, then, with do_swap = 1, the periodic swap (as in the reference).  Tags 4
 * (bcextr_sub_cuf) and 6 (bcwall_cuf) read and write w_aux (the mass fractions
 * of the cells they use, the Newton guess of tag 6): stx_update_ghost_aux takes
 * it; stx_update_ghost returns STX_E_INVALID for them. */
int stx_update_ghost(stx_ctx *ctx, void *stream, double *w, int do_swap);
int stx_update_ghost_aux(stx_ctx *ctx, void *stream, double *w, double *w_aux, int do_swap);
/* bc_nr (multideal_gpu.F90:1116-1163, kernels_gpu.F90:4330-4793): the
 * characteristic treatment of the boundary cells of every face with
 * bctags_nr > 0, added to fl (the faces' cells are outside the eul_* range of
 * the convective sweeps).  stx_rk_sync calls it after the viscous fluxes. */
int stx_bc_nr(stx_ctx *ctx, void *stream, const double *w_aux, const double *w, double *fl);

/* euler_x/y/z (multideal_gpu.F90:877-1044): hybrid central-KEEP / WENO face
 * fluxes (kernels_gpu.F90:88-2063) fused with the divergence update
 * euler_*_update_cuf (:732-793): fl += (fhat_i - fhat_{i-1}) * dxi/dx over
 * cells [imin,imax].  overwrite != 0 stores instead of accumulating, which
 * equals the reference's fl = 0 followed by the update. */
int stx_euler_x(stx_ctx *ctx, void *stream, const double *w_aux, double *fl, int imin, int imax, int overwrite);
int stx_euler_y(stx_ctx *ctx, void *stream, const double *w_aux, double *fl, int jmin, int jmax, int overwrite);
int stx_euler_z(stx_ctx *ctx, void *stream, const double *w_aux, double *fl, int kmin, int kmax, int overwrite);
/* visflx (multideal_gpu.F90:300-359): mode 1 = staggered visflx_x/y/z_cuf with
 * mixture-averaged diffusion (kernels_gpu.F90:3658-4031) fused with their
 * divergence; mode 2 = visflx_reduced_cuf (:3539-3656). */
int stx_visflx(stx_ctx *ctx, void *stream, const double *w_aux, double *fl, int mode);

/* RK bookkeeping (kernels_gpu.F90:11-86, 3297-3355). */
int stx_init_flux(stx_ctx *ctx, void *stream, double *fl, double *fln, double rhodt);
int stx_init_flux_simpler(stx_ctx *ctx, void *stream, double *fl, double *fln, const double *fl_sav, double rhodt);
int stx_sav_flx(stx_ctx *ctx, void *stream, const double *fl, double *fl_sav);
int stx_update_flux(stx_ctx *ctx, void *stream, const double *fl, double *fln, double gamdt);
int stx_update_simpler_flux(stx_ctx *ctx, void *stream, const double *fl, double *fln, const double *fl_sav, double gamdt);
int stx_update_field(stx_ctx *ctx, void *stream, double *w, const double *fln, const int32_t *fluid_mask);
/* update_flux + update_field fused: fln -= gamdt*(fl - fl_sav?); w += fln (masked). */
int stx_rk_finish(stx_ctx *ctx, void *stream, double *w, const double *fl, double *fln,
                  const double *fl_sav, const int32_t *fluid_mask, double gamdt, int simpler);

/* compute_dt_cuf (kernels_gpu.F90:6075-6152): the nine CFL maxima.  Writes
 * out9 (host memory) after synchronising the stream. */
int stx_compute_dt(stx_ctx *ctx, void *stream, const double *w_aux, const int32_t *fluid_mask, double out9[9]);

/* compute_residual (multideal_gpu.F90:1585-1615, kernels_gpu.F90:5991-6011,
 * 6038-6073) on one process: out7 = {residual_rhou = sqrt(sum over fluid
 * interior cells of (fln(I_U)/dt)^2 / (nx ny nz)), rhomin, rhomax, tmin, tmax,
 * pmin, pmax}, the figures print_progress writes every print_control steps.
 * The sum is formed in a fixed order (the same result on every call).  Writes
 * out7 (host memory) after synchronising the stream. */
int stx_compute_residual(stx_ctx *ctx, void *stream, const double *fln, const double *w_aux,
                         const int32_t *fluid_mask, double dt, double out7[7]);

/* Chemistry.  rosenbrock (multideal_gpu.F90:694-753 -> kernels_gpu.F90:8928-9501),
 * rosenbrock_krylov (:755-837 -> :10360-11205), compute_chemistry (:9503-9674). */
int stx_rosenbrock(stx_ctx *ctx, void *stream, double *w, double *w_aux,
                   double dttry, double time_start, double time_end);
int stx_rosenbrock_krylov(stx_ctx *ctx, void *stream, double *w, const double *w_aux, const double *fl_sav,
                          double dttry, double time_start, double time_end, int simpler);
int stx_compute_chemistry(stx_ctx *ctx, void *stream, double *w, double *w_aux, double *fl);

/* Whole steps.  rk_sync (multideal_gpu.F90:536-621) and advance_solution
 * (:1853-1931) sequenced on the caller's stream; *dt is the step size
 * (advance_solution halves and restores it for "simpler" splitting exactly
 * as the reference does).  No host synchronisation inside: capture-safe. */
int stx_rk_sync(stx_ctx *ctx, void *stream, const stx_fields *f, double dt, int simpler);
int stx_advance_solution(stx_ctx *ctx, void *stream, const stx_fields *f, double dt, double time);

/* Precision form of a context.  STX_PREC_FP64 (the default) is the reference's
 * FP64 method throughout.  STX_PREC_MIXED computes the central face fluxes,
 * the viscous / heat / diffusion face fluxes and the transport properties
 * (Wilke, Mathur, Bird) in FP32 and accumulates the RK residual in FP64; the
 * T(e) Newton inversion, the WENO faces, the Arrhenius rates, K_c and the
 * chemistry integration stay FP64.  The reference has no mixed form (it builds
 * all-FP32 or all-FP64, SINGLE_PRECISION). */
#define STX_PREC_FP64  0
#define STX_PREC_MIXED 1
int stx_set_precision(stx_ctx *ctx, int mode);

/* Captured steps for fixed-dt runs (cfl < 0 in multideal.ini).  The reference
 * launches ~50 kernels per step from its host loop (multideal_gpu.F90:1745-1806);
 * stx_graph_create captures nsteps iterations of that loop (compute_aux(1,0),
 * advance_solution, compute_aux(1,0), time += dt) into one CUDA graph on the
 * fields f; stx_graph_launch sets the simulation time on the device and replays
 * them on the stream (the chemistry windows read that time, so results equal the
 * step-by-step calls bit for bit).  Requires iter_dt_recompute = 1.  The graph
 * holds the field pointers and the context: keep both alive while it exists. */
typedef struct stx_graph stx_graph;
int stx_graph_create(stx_ctx *ctx, const stx_fields *f, double dt, int nsteps, stx_graph **out);
/* Captured steps for CFL-driven runs (cfl > 0, iter_dt_recompute = 1): each
 * captured step also forms the nine CFL maxima (compute_dt_cuf,
 * kernels_gpu.F90:6075-6152) and dt = cfl / max in device memory, which the
 * step's kernels read (the reference reads the maxima back to its host loop,
 * multideal_gpu.F90:1756), so nsteps steps replay with no host round trip and
 * give the step-by-step results bit for bit.  One rank only (no exchange). */
int stx_graph_create_cfl(stx_ctx *ctx, const stx_fields *f, double cfl, int nsteps, stx_graph **out);
int stx_graph_launch(stx_graph *g, void *stream, double time);
/* After a launch on `stream`: the simulation time and the last step size (the
 * fixed dt of a fixed-dt graph).  Synchronises the stream. */
int stx_graph_state(stx_graph *g, void *stream, double *time, double *dt);
int stx_graph_destroy(stx_graph *g);

/* n independent adiabatic constant-pressure 0-D reactors integrated by ROK4 in
 * one persistent launch (work stealing over reactors).  The reference's batch
 * reactor (examples/batch_reactor, flow_init 8) is one constant-volume cell run
 * through the whole solver; this is its batched, constant-pressure counterpart:
 * state Y_k, h = sum Y_k h_k(T0) and p fixed, T from h by the Newton iteration of
 * get_mixture_temperature_from_h_roe_dev (kernels_gpu.F90:6810-6900).  Device
 * arrays: T0, p0 (n); Y0, Y (n, ns) with the reactor index fastest; outputs T,
 * t_ign (first accepted time with T > ign_factor T0, or -1), t_end (time
 * reached), nsteps (ROK4 steps).  Integration ends at min(t_max,
 * end_factor t_ign); max_steps caps the steps of each reactor
 * (STX_ST_ROS_STEPS_CAP).  Uses the context's tables and work counter.  With
 * the context in the mixed precision form (stx_set_precision) the reactors run
 * the FP32/FP64-split form: the Krylov basis and the stage vectors stored in
 * FP32, the state, every right-hand side and the error control in FP64 (one
 * thread per reactor for every batch size). */
int stx_batch0d_integrate(stx_ctx *ctx, void *stream, int n, const double *T0, const double *p0, const double *Y0,
                          double t_max, double dttry, double ign_factor, double end_factor, int max_steps, double *Y,
                          double *T, double *t_ign, double *t_end, int32_t *nsteps);

/* Allocation-free ROK4 update, for callers that cannot call cudaMalloc (device
 * memory owned by another runtime or a fixed pool, or a path that must not
 * allocate while work is in flight).  No counterpart in the reference: it is
 * stx_rosenbrock_krylov without a context.  par supplies tol_iter_nr,
 * ros_maxsteps; tab holds DEVICE pointers to the caller's tables in the
 * reference's layouts (kc_tab included); grid supplies nx, ny, nz, ng only.
 * status is a device word that receives STX_ST_* bits, or NULL.
 * Its scratch is a 4-byte file-scope device array (the work-stealing cell
 * counter) loaded with the library on each device and kept until the process
 * exits; it allocates nothing.  At most 2^31 cells per call (STX_E_TOO_LARGE
 * beyond).  Calls share the scratch: each call clears it first, and calls that
 * overlap on the GPU race on it.
 * Set-up: the first call on a device loads the kernel (the CUDA runtime's module
 * load, once per device) and looks up the scratch's device address, so make it
 * before any stream capture.  The address stays valid for the life of the
 * device's primary context: do not call again on a device after resetting it
 * (cudaDeviceReset).  stream must belong to the current device (STX_E_INVALID
 * otherwise).
 * Local memory: the kernel's per-thread working set lives in local memory,
 * which the driver backs with cudaLimitStackSize bytes for every thread the
 * device can hold, and grows by a device allocation when a launch needs more.
 * So that no call allocates, a call whose kernel needs more than the current
 * limit launches nothing and returns STX_E_LOCAL_MEM.  Raise the limit once at
 * initialisation, e.g. cudaDeviceSetLimit(cudaLimitStackSize, 4608) for up to
 * 14 species or 12288 for 53 (this build's frames: 2624 B at 9 species, 3360 B
 * at 14, 9744 B at 53; the call checks the kernel's actual figure). */
int stx_rosenbrock_krylov_noalloc(const stx_params *par, const stx_tables *tab_dev, const stx_grid *grid,
                                  void *stream, double *w, const double *w_aux, const double *fl_sav,
                                  double dttry, double time_start, double time_end, int simpler, uint32_t *status);

/* Launch choices of a context that leave the method unchanged: the candidates
 * compute the same face fluxes and cell updates (equal up to rounding between
 * sweep kinds; bit for bit between WENO placements and CTA counts), so a fixed
 * tuning gives reproducible results.  No counterpart in the reference. */
typedef struct stx_tuning {
  int32_t sweep_kind[3];     /* convective sweep x, y, z: 0 staged shared-memory tiles, 1 one face per thread */
  int32_t weno_list[3];      /* 1: the faces the Ducros sensor marks are listed and computed by full warps;
                                0: computed in line by the sweep */
  int32_t chem_ctas_per_sm;  /* persistent CTAs per SM of the cell chemistry (ROK4); 0: its occupancy limit;
                                -1: the plain launch, one thread per cell and no work stealing (the
                                same per-cell arithmetic: the results are the same bit for bit) */
  int32_t chem_ctas_max;     /* out: that occupancy limit */
  int32_t batch_ctas_max;    /* most CTAs of one stx_batch0d_integrate launch; 0: no cap (a server running
                                several reactor launches at once caps each, leaving room for other work) */
  float sweep_ms[3];         /* out (stx_autotune): time of the chosen sweep kernels, ms */
  float chem_ms;             /* out (stx_autotune): time of the chosen chemistry launch, ms (stx_autotune tries
                                the persistent CTA counts from the limit down, then the plain launch) */
} stx_tuning;
int stx_get_tuning(stx_ctx *ctx, stx_tuning *out);
int stx_set_tuning(stx_ctx *ctx, const stx_tuning *t);
/* The autotuner: times every candidate of stx_tuning on the caller's fields
 * (f->w and f->w_aux as after compute_aux; neither is modified -- the sweeps
 * write a scratch residual, the chemistry runs on a scratch copy of w over
 * [0, dt_chem]), keeps the fastest in the context and returns the choice.
 * Synchronises the stream; call it outside any stream capture. */
int stx_autotune(stx_ctx *ctx, void *stream, const stx_fields *f, double dt_chem, stx_tuning *out);

/* Device status word (OR of STX_ST_* bits since the last reset); synchronises the stream. */
int stx_status(stx_ctx *ctx, void *stream, uint32_t *bits, int reset);

/* The same read without a synchronisation: enqueues on the stream the copy of the
 * status word into *bits (pinned host memory, or device memory) and then, if
 * reset, its reset.  *bits holds the value once the stream has reached this
 * point (an event recorded after the call has completed). */
int stx_status_enqueue(stx_ctx *ctx, void *stream, uint32_t *bits, int reset);

/* Instrumentation: kernel classes whose launches are counted and, while
 * profiling is on, timed with CUDA events recorded on the launching stream. */
#define STX_K_EVAL_AUX 0   /* eval_aux */
#define STX_K_DUCROS   1   /* eval_aux2 */
#define STX_K_GHOST    2   /* bcswap, bcextr_var, update_ghost faces */
#define STX_K_EULER    3   /* fused convective flux + divergence */
#define STX_K_VISC     4   /* viscous / diffusion fluxes, both modes */
#define STX_K_RK       5   /* RK bookkeeping */
#define STX_K_CHEM     6   /* Rosenbrock / ROK4 / explicit source */
#define STX_K_DT       7   /* CFL reduction */
#define STX_NK         8
typedef struct stx_kprof {
  int64_t launches;    /* kernel launches since the last stx_profile_enable */
  int64_t timed;       /* entry-point calls timed with events */
  double  ms;          /* summed event time of the timed calls */
  double  bytes;       /* algorithmic HBM bytes of those calls: every field the
                          kernel must read or write, once (FP64) */
} stx_kprof;
/* Reset the counters; on != 0 also records events around every launch. */
int stx_profile_enable(stx_ctx *ctx, int on);
/* Synchronises the device and fills out[STX_NK]. */
int stx_profile_read(stx_ctx *ctx, stx_kprof *out);

#ifdef __cplusplus
}
#endif
#endif /* STX_H */
