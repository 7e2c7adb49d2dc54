// stx_kernels.cuh -- launchers shared between the translation units of libstx.so.
#pragma once
#include "stx_common.cuh"

int launch_eval_aux(const DevCtx &c, cudaStream_t s, double *w, double *wa, int i0, int i1, int j0, int j1, int k0, int k1);
int launch_eval_aux2(const DevCtx &c, cudaStream_t s, double *wa);
int launch_bcextr_var(const DevCtx &c, cudaStream_t s, double *v);
int launch_bcswap(const DevCtx &c, cudaStream_t s, double *f, int nvar, const int *periodic);
int launch_bc_face(const DevCtx &c, cudaStream_t s, double *w, int ilat, int tag, const double *winf);
// ghost fills that need the thermodynamics and w_aux (bc tags 4 and 6)
int launch_bc_face_thermo(const DevCtx &c, cudaStream_t s, double *w, double *wa, int ilat, int tag);
// characteristic boundary treatment of face ilat (bc_nr_lat_*), added to fl
int launch_bc_nr(const DevCtx &c, cudaStream_t s, const double *wa, const double *w, double *fl, const double *winf,
                 int ilat, int nr_type);
// scale: with c.p.dt_d set (captured CFL-driven steps), rhodt / gamdt are the RK
// coefficient and the kernels form coefficient * (scale * dt) from the device dt
int launch_init_flux(const DevCtx &c, cudaStream_t s, double *fl, double *fln, const double *fl_sav, double rhodt,
                     double scale = 1.0);
int launch_update_flux(const DevCtx &c, cudaStream_t s, const double *fl, double *fln, const double *fl_sav, double gamdt,
                       double scale = 1.0);
int launch_copy(const DevCtx &c, cudaStream_t s, const double *a, double *b);
int launch_update_field(const DevCtx &c, cudaStream_t s, double *w, const double *fl, double *fln, const double *fl_sav,
                        const int32_t *mask, double gamdt, int fused, double scale = 1.0);
// the step size from the nine CFL maxima (bit patterns, as k_compute_dt leaves
// them): *dt = cfl / max, the host's operations
int launch_dt_from_max(cudaStream_t s, const unsigned long long *max9, double cfl, double *dt);
// *t = *t + *dt (the time advance of a captured CFL-driven step)
int launch_time_advance(cudaStream_t s, double *t, const double *dt);
int launch_compute_dt(const DevCtx &c, cudaStream_t s, const double *wa, const int32_t *mask, unsigned long long *out9);
// compute_residual + rho/T/p extrema: STX_RES_BLOCKS partial sums in part, 6 extrema in mm
#define STX_RES_BLOCKS 296
int launch_residual_minmax(const DevCtx &c, cudaStream_t s, const double *fln, const double *wa, const int32_t *mask,
                           double dt, double *part, unsigned long long *mm);

// Scratch of the listed WENO faces (stx_euler.cu): a counter, the ids of the
// faces the Ducros sensor marks, and their fluxes by face id (nv x cap).
struct WenoScratch {
  unsigned int *count;
  int *list;
  double *fh;
  long long cap;      // faces the buffers hold (0: no scratch)
};
// faces of the largest sweep of a grid (the listed-WENO scratch size)
long long weno_scratch_faces(const DevGrid &g);

// once per context, before any capture: kernel attributes of the staged sweeps
int launch_euler_setup(int ns);
// cg: a device-resident copy of c, for the out-of-line WENO face fluxes;
// ws: the listed-WENO scratch (null or cap 0: WENO faces computed in line)
int launch_euler(const DevCtx &c, const DevCtx *cg, cudaStream_t s, int dir, const double *wa, double *fl, int nmin,
                 int nmax, int overwrite, const WenoScratch *ws);
int launch_visflx(const DevCtx &c, cudaStream_t s, int dir, const double *wa, double *fl);
int launch_visflx_reduced(const DevCtx &c, cudaStream_t s, const double *wa, double *fl);

// occupancy limit (CTAs per SM) of the ROK4 cell kernel for ns species
int chem_ctas_limit(int ns);
// cg: the device-resident copy of c (stx_ctx::dctx_d)
int launch_rok4(const DevCtx &c, const DevCtx *cg, cudaStream_t s, double *w, const double *wa, const double *fl_sav,
                double dttry, double t0, double t1, int simpler, unsigned int *counter);
int launch_rosenbrock(const DevCtx &c, cudaStream_t s, double *w, double *wa, double dttry, double t0, double t1,
                      unsigned int *counter);
int launch_chem_explicit(const DevCtx &c, cudaStream_t s, double *w, double *wa, double *fl);
// cg: the device-resident context (its ros_maxsteps is not read: c's is the cap)
int launch_batch0d(const DevCtx &c, const DevCtx *cg, cudaStream_t s, int n, const double *T0, const double *p0,
                   const double *Y0, double t_max, double dttry, double ign, double endf, double *Y, double *T,
                   double *t_ign, double *t_end, int *nsteps, unsigned int *counter);
// once per device and species count: shared-memory split of the persistent
// warp-per-reactor kernel
int launch_batch0d_setup(int ns);
// one warp per reactor (ns <= 32, nr <= 64, and unless force, no more reactors
// than resident warps; STX_E_UNSUPPORTED otherwise)
int launch_batch0d_warp(const DevCtx &c, cudaStream_t s, int n, const double *T0, const double *p0, const double *Y0,
                        double t_max, double dttry, double ign, double endf, double *Y, double *T, double *t_ign,
                        double *t_end, int *nsteps, unsigned int *counter, int force);
