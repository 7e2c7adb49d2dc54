/*
 * stx_oracle.h -- CPU oracle for the multi-species reacting step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C FP64 restatement of the
 * reference's CUDA-Fortran kernels (src/multideal/kernels_gpu.F90) and of the
 * host sequencing in src/multideal/multideal_gpu.F90, used as the parity
 * checker for the CUDA path and as the timed CPU baseline.  Nothing in the
 * product links or calls it: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load liboracle.so.
 *
 * The functions take the same parameter structs as the C ABI (include/stx.h)
 * but HOST pointers, and use the same Fortran layouts and 1-based indices.
 * Parity of the oracle itself is pinned by tests against the reference's own
 * outputs: the thermo constants of examples/laminar_premix_flame/data.dat and
 * the 0-D reactor trajectories of examples/syngas_mech_eval/OUTPUT/.
 */
#ifndef STX_ORACLE_H
#define STX_ORACLE_H
#include "../include/stx.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ox_ctx ox_ctx;

ox_ctx *ox_ctx_create(const stx_params *par, const stx_tables *tab, const stx_grid *grid);
void    ox_ctx_destroy(ox_ctx *c);
void    ox_set_threads(int n);
uint32_t ox_status(ox_ctx *c, int reset);

void ox_eval_aux(ox_ctx *c, double *w, double *w_aux, int istart, int iend, int jstart, int jend, int kstart, int kend);
void ox_compute_aux(ox_ctx *c, double *w, double *w_aux, int central, int ghost);
void ox_eval_aux2(ox_ctx *c, double *w_aux);
void ox_bcextr_var(ox_ctx *c, double *var);
void ox_bcswap(ox_ctx *c, double *field, int nvar);
void ox_update_ghost(ox_ctx *c, double *w, int do_swap);
void ox_update_ghost_aux(ox_ctx *c, double *w, double *w_aux, int do_swap);
void ox_bc_nr(ox_ctx *c, const double *w_aux, const double *w, double *fl);
void ox_compute_residual(ox_ctx *c, const double *fln, const double *wa, const int32_t *mask, double dt,
                         double out7[7]);
/* face fluxes into fhat (ghosted, nv) for faces [face_lo, face_hi], then the update over [imin, imax] */
void ox_euler(ox_ctx *c, int dir, const double *w_aux, double *fhat, double *fl, int nmin, int nmax);
void ox_visflx(ox_ctx *c, const double *w_aux, double *fl, double *fhat, int mode);
void ox_init_flux(ox_ctx *c, double *fl, double *fln, double rhodt);
void ox_init_flux_simpler(ox_ctx *c, double *fl, double *fln, const double *fl_sav, double rhodt);
void ox_sav_flx(ox_ctx *c, const double *fl, double *fl_sav);
void ox_update_flux(ox_ctx *c, const double *fl, double *fln, double gamdt);
void ox_update_simpler_flux(ox_ctx *c, const double *fl, double *fln, const double *fl_sav, double gamdt);
void ox_update_field(ox_ctx *c, double *w, const double *fln, const int32_t *fluid_mask);
void ox_compute_dt(ox_ctx *c, const double *w_aux, const int32_t *fluid_mask, double out9[9]);
void ox_rosenbrock(ox_ctx *c, double *w, double *w_aux, double dttry, double time_start, double time_end);
void ox_rosenbrock_krylov(ox_ctx *c, double *w, const double *w_aux, const double *fl_sav,
                          double dttry, double time_start, double time_end, int simpler);
void ox_compute_chemistry(ox_ctx *c, double *w, double *w_aux, double *fl);
/* whole steps; fhat is caller scratch (ghosted, nv) */
void ox_rk_sync(ox_ctx *c, const stx_fields *f, double *fhat, double dt, int simpler);
void ox_advance_solution(ox_ctx *c, const stx_fields *f, double *fhat, double dt, double time);

/* single-cell chemistry, for tests of the kernels' per-cell contracts */
void ox_krylov_cell(ox_ctx *c, double *wcell, double T_start, double Z, const double *fl_sav_cell,
                    double dttry, double time_start, double time_end, int simpler);
void ox_rosenbrock_cell(ox_ctx *c, double *wcell, double *Y, double *T, double dttry,
                        double time_start, double time_end);
double ox_temperature_from_e(ox_ctx *c, double ee, double T_start, const double *Y);

/* n adiabatic constant-pressure 0-D reactors (the batched-reactor workload);
 * Y0 / Y are (n, ns) with the reactor index fastest */
void ox_batch0d_cp(ox_ctx *c, int n, const double *T0, const double *p0, const double *Y0, double t_max,
                   double dttry, double ign_factor, double end_factor, int max_steps, double *Y, double *T,
                   double *t_ign, double *t_end, int32_t *nsteps);

#ifdef __cplusplus
}
#endif
#endif
