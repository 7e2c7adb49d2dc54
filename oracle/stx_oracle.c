/*
 * stx_oracle.c -- CPU FP64 oracle (test infrastructure, see stx_oracle.h).
 *
 * Each function restates the reference routine cited beside it, in the same
 * order of operations, so that the oracle reproduces the reference arithmetic
 * (up to the rounding of libm's exp/pow/log, which differ from CUDA's by an ulp
 * or two).  Cells are independent in every kernel, so the loops are split
 * over OpenMP threads without changing any result.
 */
#include "stx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXNS 64
#define MAXNV (MAXNS + 4)
#define MMAX 4      /* M_max, src/multideal/index_define.h:27 */
#define NSTAGE 4    /* nstep, src/multideal/index_define.h:4 */

struct ox_ctx {
  stx_params p;
  stx_tables t;
  stx_grid g;
  int ns, nv, ncp, nxg, nyg, nzg;
  size_t npg, npi, ntab1;
  double cd1[5][5];            /* coeff_deriv1(l, lmax) -> cd1[l][lmax] */
  double *wk_a, *wk_b;         /* Wilke pair factors (ns*ns) */
  double *trange, *cp, *cv, *mw, *mwinv, *rgas;
  uint32_t status;
};

void ox_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

uint32_t ox_status(ox_ctx *c, int reset) {
  uint32_t s = c->status;
  if (reset) c->status = 0;
  return s;
}

/* ---------------------------------------------------------------- indexing */
#define NS (c->ns)
#define I_U (NS + 1)
#define I_V (NS + 2)
#define I_W (NS + 3)
#define I_E (NS + 4)
#define J_U (NS + 1)
#define J_V (NS + 2)
#define J_W (NS + 3)
#define J_H (NS + 4)
#define J_T (NS + 5)
#define J_P (NS + 6)
#define J_C (NS + 7)
#define J_MU (NS + 8)
#define J_DUC (NS + 9)
#define J_DIV (NS + 10)
#define J_R (NS + 11)
#define J_Z (NS + 12)
#define J_K_COND (NS + 13)
#define J_D_START (NS + 13)

static inline size_t gi(const ox_ctx *c, int i, int j, int k) {
  int ng = c->g.ng;
  return (size_t)(i + ng - 1) + (size_t)c->nxg * ((size_t)(j + ng - 1) + (size_t)c->nyg * (size_t)(k + ng - 1));
}
static inline size_t fi(const ox_ctx *c, int i, int j, int k) {
  return (size_t)(i - 1) + (size_t)c->g.nx * ((size_t)(j - 1) + (size_t)c->g.ny * (size_t)(k - 1));
}
#define WG(a, p, m) ((a)[(p) + (size_t)((m) - 1) * c->npg])
#define WF(a, p, m) ((a)[(p) + (size_t)((m) - 1) * c->npi])
#define TRANGE(lsp, jm) (c->trange[(size_t)((jm) - 1) * NS + (lsp) - 1])
#define CPC(arr, l, lsp, m) ((arr)[((size_t)((m) - 1) * NS + (lsp) - 1) * c->ncp + ((l) - c->t.indx_cp_l)])
#define VISC(it, lsp) (c->t.visc[(size_t)((lsp) - 1) * c->ntab1 + (it) - 1])
#define LAMB(it, lsp) (c->t.lambda[(size_t)((lsp) - 1) * c->ntab1 + (it) - 1])
#define DIFF(it, l, m) (c->t.diffbin[(((size_t)(m) - 1) * NS + (l) - 1) * c->ntab1 + (it) - 1])
#define KC(it, lr) (c->t.kc_tab[(size_t)((lr) - 1) * c->ntab1 + (it) - 1])
#define RX(arr, lr, j) ((arr)[(size_t)((j) - 1) * c->t.nr + (lr) - 1])

/* Fortran real**integer */
static inline double ipow(double x, int n) {
  double r = 1.0;
  int u = n < 0 ? -n : n;
  for (int q = 0; q < u; q++) r *= x;
  return n < 0 ? 1.0 / r : r;
}
static inline double dmax(double a, double b) { return a > b ? a : b; }
static inline double dmin(double a, double b) { return a < b ? a : b; }

/* ---------------------------------------------------------------- context */
ox_ctx *ox_ctx_create(const stx_params *par, const stx_tables *tab, const stx_grid *grid) {
  ox_ctx *c = (ox_ctx *)calloc(1, sizeof(ox_ctx));
  c->p = *par;
  c->t = *tab;
  c->g = *grid;
  c->ns = tab->ns;
  c->nv = tab->ns + 4;
  c->ncp = tab->indx_cp_r - tab->indx_cp_l + 3;
  c->nxg = grid->nx + 2 * grid->ng;
  c->nyg = grid->ny + 2 * grid->ng;
  c->nzg = grid->nz + 2 * grid->ng;
  c->npg = (size_t)c->nxg * c->nyg * c->nzg;
  c->npi = (size_t)grid->nx * grid->ny * grid->nz;
  c->ntab1 = (size_t)tab->num_t_tab + 1;
  c->trange = (double *)tab->trange;
  c->cp = (double *)tab->cp_coeff;
  c->cv = (double *)tab->cv_coeff;
  c->mw = (double *)tab->mw;
  c->mwinv = (double *)tab->mwinv;
  c->rgas = (double *)tab->rgas;
  /* grid.F90:135-160 coefficient table, column lmax = order/2 */
  memset(c->cd1, 0, sizeof(c->cd1));
  c->cd1[1][1] = 0.5;
  c->cd1[1][2] = 2.0 / 3.0;  c->cd1[2][2] = -1.0 / 12.0;
  c->cd1[1][3] = 0.75;       c->cd1[2][3] = -0.15;      c->cd1[3][3] = 1.0 / 60.0;
  c->cd1[1][4] = 4.0 / 5.0;  c->cd1[2][4] = -1.0 / 5.0; c->cd1[3][4] = 4.0 / 105.0; c->cd1[4][4] = -1.0 / 280.0;
  /* Wilke pair factors of kernels_gpu.F90:6272-6273 (functions of the molecular weights only) */
  c->wk_a = (double *)malloc(sizeof(double) * NS * NS);
  c->wk_b = (double *)malloc(sizeof(double) * NS * NS);
  for (int l = 1; l <= NS; l++)
    for (int m = 1; m <= NS; m++) {
      c->wk_a[(l - 1) * NS + m - 1] = 1.0 / sqrt(1.0 + c->mw[l - 1] * c->mwinv[m - 1]);
      c->wk_b[(l - 1) * NS + m - 1] = pow(c->mw[m - 1] * c->mwinv[l - 1], 0.25);
    }
  return c;
}

void ox_ctx_destroy(ox_ctx *c) {
  if (!c) return;
  free(c->wk_a);
  free(c->wk_b);
  free(c);
}

/* ---------------------------------------------------------------- thermo */
/* Numerical-Recipes locate used by every thermo routine (e.g. kernels_gpu.F90:6397-6415) */
static inline int locate_range(const ox_ctx *c, double T, int lsp) {
  int nset = c->t.nsetcv;
  int jl = 0, ju = nset + 2;
  while (ju - jl > 1) {
    int jm = (ju + jl) / 2;
    if (T >= TRANGE(lsp, jm)) jl = jm; else ju = jm;
  }
  if (jl < 1) jl = 1;
  if (jl > nset) jl = nset;
  return jl;
}

/* get_cp_dev / get_cp_roe_dev (kernels_gpu.F90:6384-6480) */
static double mix_cp(const ox_ctx *c, double tt, const double *Y) {
  int nrange[MAXNS];
  for (int lsp = 1; lsp <= NS; lsp++) nrange[lsp - 1] = 1;
  if (c->t.nsetcv > 1)
    for (int lsp = 1; lsp <= NS; lsp++) nrange[lsp - 1] = locate_range(c, tt, lsp);
  double cploc = 0.0;
  for (int l = c->t.indx_cp_l; l <= c->t.indx_cp_r; l++) {
    double tpow = ipow(tt, l);
    double cp_l = 0.0;
    for (int lsp = 1; lsp <= NS; lsp++) cp_l = cp_l + CPC(c->cp, l, lsp, nrange[lsp - 1]) * Y[lsp - 1];
    cploc = cploc + cp_l * tpow;
  }
  return cploc;
}

/* get_mixture_temperature_from_e_dev (kernels_gpu.F90:6532-6622); the _krylov and
 * Roe-inlined copies (:10977-11059, :3082-3157) are the same iteration.  With the
 * cp table in place of cv it is get_mixture_temperature_from_h_roe_dev
 * (:6810-6900), T from the mixture enthalpy. */
static double temperature_from_poly(ox_ctx *c, const double *coef, double ee, double T_start, const double *Y);
double ox_temperature_from_e(ox_ctx *c, double ee, double T_start, const double *Y) {
  return temperature_from_poly(c, c->cv, ee, T_start, Y);
}
static double temperature_from_poly(ox_ctx *c, const double *coef, double ee, double T_start, const double *Y) {
  int nrange[MAXNS];
  int nset = c->t.nsetcv;
  const int max_iter = 10;
  for (int lsp = 1; lsp <= NS; lsp++) nrange[lsp - 1] = 1;
  if (nset > 1)
    for (int lsp = 1; lsp <= NS; lsp++) nrange[lsp - 1] = locate_range(c, T_start, lsp);
  double T_old = T_start, tt = T_start;
  int conv = 0;
  for (int iter = 1; iter <= max_iter; iter++) {
    if (nset > 1) {
      for (int lsp = 1; lsp <= NS; lsp++) {
        int nl = nrange[lsp - 1];
        if (T_old < TRANGE(lsp, nl)) nrange[lsp - 1] = nrange[lsp - 1] - 1;
        else if (T_old > TRANGE(lsp, nl + 1)) nrange[lsp - 1] = nrange[lsp - 1] + 1;
        if (nrange[lsp - 1] < 1) nrange[lsp - 1] = 1;
        if (nrange[lsp - 1] > nset) nrange[lsp - 1] = nset;
      }
    }
    double sumb = 0.0;
    for (int lsp = 1; lsp <= NS; lsp++) sumb = sumb + CPC(coef, c->t.indx_cp_r + 1, lsp, nrange[lsp - 1]) * Y[lsp - 1];
    double ebar = ee - sumb;
    double den = 0.0, num = 0.0;
    for (int l = c->t.indx_cp_l; l <= c->t.indx_cp_r; l++) {
      double T_pow = ipow(T_old, l);
      double tden = T_pow, tnum;
      if (l == -1) {
        tnum = log(T_old);
      } else {
        double T_powp = T_old * T_pow;
        tnum = T_powp / (l + 1.0);
      }
      double cv_l = 0.0;
      for (int lsp = 1; lsp <= NS; lsp++) cv_l = cv_l + CPC(coef, l, lsp, nrange[lsp - 1]) * Y[lsp - 1];
      num = num + cv_l * tnum;
      den = den + cv_l * tden;
    }
    tt = T_old + (ebar - num) / den;
    if (fabs(tt - T_old) < c->p.tol_iter_nr) { conv = 1; break; }
    T_old = tt;
  }
  if (!conv) c->status |= STX_ST_NEWTON_CAP;
  return tt;
}

/* get_species_h_from_temperature_dev / _e_ (kernels_gpu.F90:7104-7183) */
static double species_poly_int(const ox_ctx *c, const double *arr, double tt, int isp) {
  int nr = 1;
  if (c->t.nsetcv > 1) nr = locate_range(c, tt, isp);
  double hh = CPC(arr, c->t.indx_cp_r + 1, isp, nr);
  for (int l = c->t.indx_cp_l; l <= c->t.indx_cp_r; l++) {
    if (l == -1) hh = hh + CPC(arr, l, isp, nr) * log(tt);
    else hh = hh + CPC(arr, l, isp, nr) / (l + 1.0) * ipow(tt, l + 1);
  }
  return hh;
}

/* get_mixture_e_from_temperature_dev (kernels_gpu.F90:7047-7102): the mixture's
 * internal energy at tt with the mass fractions in w_aux(p, 1..ns) */
static double mixture_e_wa(const ox_ctx *c, double tt, const double *wa, size_t p) {
  int nrange[MAXNS];
  for (int lsp = 1; lsp <= NS; lsp++) nrange[lsp - 1] = c->t.nsetcv > 1 ? locate_range(c, tt, lsp) : 1;
  double ee = 0.0;
  for (int lsp = 1; lsp <= NS; lsp++) ee = ee + CPC(c->cv, c->t.indx_cp_r + 1, lsp, nrange[lsp - 1]) * WG(wa, p, lsp);
  for (int l = c->t.indx_cp_l; l <= c->t.indx_cp_r; l++) {
    double tprod = l == -1 ? log(tt) : ipow(tt, l + 1) / (l + 1.0);
    double cv_l = 0.0;
    for (int lsp = 1; lsp <= NS; lsp++) cv_l = cv_l + CPC(c->cv, l, lsp, nrange[lsp - 1]) * WG(wa, p, lsp);
    ee = ee + cv_l * tprod;
  }
  return ee;
}
/* get_rho_from_w_dev (:6902-6915) and get_rmixture (:6917-6931) */
static double rho_from_w(const ox_ctx *c, const double *w, size_t p) {
  double rho = WG(w, p, 1);
  for (int lsp = 2; lsp <= NS; lsp++) rho = rho + WG(w, p, lsp);
  return rho;
}
static double rmix_wa(const ox_ctx *c, const double *wa, size_t p) {
  double rm = c->rgas[0] * WG(wa, p, 1);
  for (int lsp = 2; lsp <= NS; lsp++) rm = rm + c->rgas[lsp - 1] * WG(wa, p, lsp);
  return rm;
}

/* ---------------------------------------------------------------- eval_aux */
/* eval_aux_cuf body (kernels_gpu.F90:6188-6302) for one point */
static void aux_point(ox_ctx *c, double *w, double *wa, size_t p) {
  double Y[MAXNS];
  for (int lsp = 1; lsp <= NS; lsp++) WG(w, p, lsp) = dmax(WG(w, p, lsp), 0.0);
  double rho = WG(w, p, 1);
  for (int lsp = 2; lsp <= NS; lsp++) rho = rho + WG(w, p, lsp);
  double ri = 1.0 / rho;
  for (int lsp = 1; lsp <= NS; lsp++) { Y[lsp - 1] = WG(w, p, lsp) * ri; WG(wa, p, lsp) = Y[lsp - 1]; }
  double rhou = WG(w, p, I_U), rhov = WG(w, p, I_V), rhow = WG(w, p, I_W), rhoe = WG(w, p, I_E);
  double uu = rhou * ri, vv = rhov * ri, ww = rhow * ri;
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double ee = rhoe * ri - qq;
  double tt = ox_temperature_from_e(c, ee, WG(wa, p, J_T), Y);
  double rmixtloc = c->rgas[0] * Y[0];
  for (int lsp = 2; lsp <= NS; lsp++) rmixtloc = rmixtloc + c->rgas[lsp - 1] * Y[lsp - 1];
  double cploc = mix_cp(c, tt, Y);
  double gamloc = cploc / (cploc - rmixtloc);
  double pp = rho * tt * rmixtloc;
  double cc = sqrt(gamloc * pp * ri);
  WG(wa, p, J_R) = rho;
  WG(wa, p, J_U) = uu;
  WG(wa, p, J_V) = vv;
  WG(wa, p, J_W) = ww;
  WG(wa, p, J_H) = (rhoe + pp) * ri;
  WG(wa, p, J_T) = tt;
  WG(wa, p, J_P) = pp;
  WG(wa, p, J_C) = cc;
  /* Bilger mixture fraction (:6228-6243) */
  if (c->t.n_eoi != 1) {
    double Beta = 0.0;
    for (int le = 1; le <= c->t.n_eoi; le++) {
      double yatm = 0.0;
      for (int lsp = 1; lsp <= NS; lsp++)
        if (Y[lsp - 1] > 1e-14)
          yatm = yatm + c->t.nainsp[(size_t)(le - 1) * NS + lsp - 1] * c->t.aw_eoi[le - 1] * Y[lsp - 1] * c->mwinv[lsp - 1];
      Beta = Beta + c->t.coeff_eoi[le - 1] * yatm / c->t.aw_eoi[le - 1];
    }
    WG(wa, p, J_Z) = (Beta - c->t.beta0[1]) / (c->t.beta0[0] - c->t.beta0[1]);
  } else {
    WG(wa, p, J_Z) = 0.5;
  }
  int itt = (int)((tt - c->t.t_min_tab) / c->t.dt_tab) + 1;
  if (itt < 1) itt = 1;
  if (itt > c->t.num_t_tab) itt = c->t.num_t_tab;
  double tloc = c->t.t_min_tab + (itt - 1) * c->t.dt_tab;
  double dtt = (tt - tloc) / c->t.dt_tab;
  /* Mathur conductivity (:6252-6264) */
  double mwmixt = c->t.R_univ / rmixtloc;
  double k_cond = 0.0, k_cond2 = 0.0;
  for (int lsp = 1; lsp <= NS; lsp++) {
    double dlam = LAMB(itt + 1, lsp) - LAMB(itt, lsp);
    double klsp = LAMB(itt, lsp) + dlam * dtt;
    double xlsp = Y[lsp - 1] * mwmixt * c->mwinv[lsp - 1];
    k_cond = k_cond + xlsp * klsp;
    k_cond2 = k_cond2 + xlsp / klsp;
  }
  k_cond = 0.5 * (k_cond + 1.0 / k_cond2);
  /* Wilke viscosity (:6266-6281) */
  double mu = 0.0;
  for (int lsp = 1; lsp <= NS; lsp++) {
    double dmu = VISC(itt + 1, lsp) - VISC(itt, lsp);
    double mulsp = VISC(itt, lsp) + dmu * dtt;
    double mu_den = 0.0;
    for (int msp = 1; msp <= NS; msp++) {
      dmu = VISC(itt + 1, msp) - VISC(itt, msp);
      double mumsp = VISC(itt, msp) + dmu * dtt;
      double t1 = 1.0 + sqrt(mumsp / mulsp) * c->wk_b[(lsp - 1) * NS + msp - 1];
      double phi_lm = c->wk_a[(lsp - 1) * NS + msp - 1] * (t1 * t1);
      mu_den = mu_den + Y[msp - 1] * phi_lm * c->mwinv[msp - 1];
    }
    mu = mu + mulsp * Y[lsp - 1] * c->mwinv[lsp - 1] / mu_den;
  }
  mu = sqrt(8.0) * mu;
  WG(wa, p, J_MU) = mu;
  WG(wa, p, J_K_COND) = k_cond;
  /* Bird diffusion (:6286-6302) */
  for (int lsp = 1; lsp <= NS; lsp++) {
    double diff_den = 0.0;
    for (int msp = 1; msp <= NS; msp++) {
      if (msp != lsp) {
        double ddiff = DIFF(itt + 1, lsp, msp) - DIFF(itt, lsp, msp);
        double diff_ij = DIFF(itt, lsp, msp) + ddiff * dtt;
        double xmsp = Y[msp - 1] * mwmixt * c->mwinv[msp - 1];
        diff_den = diff_den + xmsp / diff_ij;
      }
    }
    if (diff_den > 1.0e-15) WG(wa, p, J_D_START + lsp) = (1.0 - Y[lsp - 1]) / diff_den * c->p.p0 / pp * rho;
    else WG(wa, p, J_D_START + lsp) = 0.0;
  }
}

void ox_eval_aux(ox_ctx *c, double *w, double *w_aux, int istart, int iend, int jstart, int jend, int kstart, int kend) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = kstart; k <= kend; k++)
    for (int j = jstart; j <= jend; j++)
      for (int i = istart; i <= iend; i++) aux_point(c, w, w_aux, gi(c, i, j, k));
}

/* compute_aux (multideal_gpu.F90:361-443) without LES */
void ox_compute_aux(ox_ctx *c, double *w, double *wa, int central, int ghost) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz, ng = c->g.ng;
  if (central == 1 && ghost == 1) {
    ox_eval_aux(c, w, wa, 1 - ng, nx + ng, 1 - ng, ny + ng, 1 - ng, nz + ng);
  } else if (central == 1 && ghost == 0) {
    ox_eval_aux(c, w, wa, 1, nx, 1, ny, 1, nz);
  } else if (central == 0 && ghost == 1) {
    ox_eval_aux(c, w, wa, 1 - ng, 0, 1 - ng, ny + ng, 1 - ng, nz + ng);
    ox_eval_aux(c, w, wa, nx + 1, nx + ng, 1 - ng, ny + ng, 1 - ng, nz + ng);
    ox_eval_aux(c, w, wa, 1 - ng, nx + ng, 1 - ng, 0, 1 - ng, nz + ng);
    ox_eval_aux(c, w, wa, 1 - ng, nx + ng, ny + 1, ny + ng, 1 - ng, nz + ng);
    ox_eval_aux(c, w, wa, 1 - ng, nx + ng, 1 - ng, ny + ng, 1 - ng, 0);
    ox_eval_aux(c, w, wa, 1 - ng, nx + ng, 1 - ng, ny + ng, nz + 1, nz + ng);
  }
  if (ghost == 1) ox_eval_aux2(c, wa);
}

/* eval_aux2_cuf (kernels_gpu.F90:6310-6382) */
void ox_eval_aux2(ox_ctx *c, double *wa) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz;
  int lmax = c->p.visc_order / 2;
  size_t sx = 1, sy = (size_t)c->nxg, sz = (size_t)c->nxg * c->nyg;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        size_t p = gi(c, i, j, k);
        double ux = 0, vx = 0, wx = 0, uy = 0, vy = 0, wy = 0, uz = 0, vz = 0, wz = 0;
        for (int l = 1; l <= lmax; l++) {
          double ccl = c->cd1[l][lmax];
          ux = ux + ccl * (WG(wa, p + l * sx, J_U) - WG(wa, p - l * sx, J_U));
          vx = vx + ccl * (WG(wa, p + l * sx, J_V) - WG(wa, p - l * sx, J_V));
          wx = wx + ccl * (WG(wa, p + l * sx, J_W) - WG(wa, p - l * sx, J_W));
          uy = uy + ccl * (WG(wa, p + l * sy, J_U) - WG(wa, p - l * sy, J_U));
          vy = vy + ccl * (WG(wa, p + l * sy, J_V) - WG(wa, p - l * sy, J_V));
          wy = wy + ccl * (WG(wa, p + l * sy, J_W) - WG(wa, p - l * sy, J_W));
          uz = uz + ccl * (WG(wa, p + l * sz, J_U) - WG(wa, p - l * sz, J_U));
          vz = vz + ccl * (WG(wa, p + l * sz, J_V) - WG(wa, p - l * sz, J_V));
          wz = wz + ccl * (WG(wa, p + l * sz, J_W) - WG(wa, p - l * sz, J_W));
        }
        ux = ux * c->g.dcsidx[i - 1]; vx = vx * c->g.dcsidx[i - 1]; wx = wx * c->g.dcsidx[i - 1];
        uy = uy * c->g.detady[j - 1]; vy = vy * c->g.detady[j - 1]; wy = wy * c->g.detady[j - 1];
        uz = uz * c->g.dzitdz[k - 1]; vz = vz * c->g.dzitdz[k - 1]; wz = wz * c->g.dzitdz[k - 1];
        double div = ux + vy + wz;
        double div3l = div / 3.0;
        double omegax = wy - vz, omegay = uz - wx, omegaz = vx - uy;
        double omod2 = omegax * omegax + omegay * omegay + omegaz * omegaz;
        double s = -div / sqrt(omod2 + div * div + c->p.eps_sensor);
        if (c->p.sensor_type == 0) WG(wa, p, J_DUC) = s * s;
        else { double t = dmax(s, 0.0); WG(wa, p, J_DUC) = t * t; }
        WG(wa, p, J_DIV) = div3l;
      }
}

/* ---------------------------------------------------------------- ghosts */
/* bcextr_var_cuf (kernels_gpu.F90:5147-5207) */
void ox_bcextr_var(ox_ctx *c, double *v) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz, ng = c->g.ng;
  for (int k = 1; k <= nz; k++) for (int j = 1; j <= ny; j++) for (int l = 1; l <= ng; l++) v[gi(c, 1 - l, j, k)] = v[gi(c, 1, j, k)];
  for (int k = 1; k <= nz; k++) for (int j = 1; j <= ny; j++) for (int l = 1; l <= ng; l++) v[gi(c, nx + l, j, k)] = v[gi(c, nx, j, k)];
  for (int k = 1; k <= nz; k++) for (int i = 1; i <= nx; i++) for (int l = 1; l <= ng; l++) v[gi(c, i, 1 - l, k)] = v[gi(c, i, 1, k)];
  for (int k = 1; k <= nz; k++) for (int i = 1; i <= nx; i++) for (int l = 1; l <= ng; l++) v[gi(c, i, ny + l, k)] = v[gi(c, i, ny, k)];
  for (int j = 1; j <= ny; j++) for (int i = 1; i <= nx; i++) for (int l = 1; l <= ng; l++) v[gi(c, i, j, 1 - l)] = v[gi(c, i, j, 1)];
  for (int j = 1; j <= ny; j++) for (int i = 1; i <= nx; i++) for (int l = 1; l <= ng; l++) v[gi(c, i, j, nz + l)] = v[gi(c, i, j, nz)];
}

/* base_gpu%bcswap on one rank (base_gpu.F90:1132-1196 with bcswap_step_1/3_cuf
 * :155-207, :297-383): pack every face buffer first, then unpack the periodic
 * directions (a non-periodic side has MPI_PROC_NULL as neighbour: no unpack). */
void ox_bcswap(ox_ctx *c, double *f, int nvar) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz, ng = c->g.ng;
  int per[3] = {c->p.bctags[0] == 0, c->p.bctags[2] == 0, c->p.bctags[4] == 0};
  size_t bx = (size_t)ng * ny * nz, by = (size_t)nx * ng * nz, bz = (size_t)nx * ny * ng;
  double *b1 = (double *)malloc(sizeof(double) * bx * nvar), *b2 = (double *)malloc(sizeof(double) * bx * nvar);
  double *b3 = (double *)malloc(sizeof(double) * by * nvar), *b4 = (double *)malloc(sizeof(double) * by * nvar);
  double *b5 = (double *)malloc(sizeof(double) * bz * nvar), *b6 = (double *)malloc(sizeof(double) * bz * nvar);
  for (int m = 1; m <= nvar; m++)
    for (int k = 1; k <= nz; k++) for (int j = 1; j <= ny; j++) for (int i = 1; i <= ng; i++) {
      size_t q = (size_t)(i - 1) + ng * ((size_t)(j - 1) + ny * ((size_t)(k - 1) + nz * (size_t)(m - 1)));
      b1[q] = WG(f, gi(c, i, j, k), m);
      b2[q] = WG(f, gi(c, nx - ng + i, j, k), m);
    }
  for (int m = 1; m <= nvar; m++)
    for (int k = 1; k <= nz; k++) for (int j = 1; j <= ng; j++) for (int i = 1; i <= nx; i++) {
      size_t q = (size_t)(i - 1) + nx * ((size_t)(j - 1) + ng * ((size_t)(k - 1) + nz * (size_t)(m - 1)));
      b3[q] = WG(f, gi(c, i, j, k), m);
      b4[q] = WG(f, gi(c, i, ny - ng + j, k), m);
    }
  for (int m = 1; m <= nvar; m++)
    for (int k = 1; k <= ng; k++) for (int j = 1; j <= ny; j++) for (int i = 1; i <= nx; i++) {
      size_t q = (size_t)(i - 1) + nx * ((size_t)(j - 1) + ny * ((size_t)(k - 1) + ng * (size_t)(m - 1)));
      b5[q] = WG(f, gi(c, i, j, k), m);
      b6[q] = WG(f, gi(c, i, j, nz - ng + k), m);
    }
  /* self-exchange: wbuf2r = wbuf1s, wbuf1r = wbuf2s (base_gpu.F90:1168-1170) */
  if (per[0])
    for (int m = 1; m <= nvar; m++)
      for (int k = 1; k <= nz; k++) for (int j = 1; j <= ny; j++) for (int i = 1; i <= ng; i++) {
        size_t q = (size_t)(i - 1) + ng * ((size_t)(j - 1) + ny * ((size_t)(k - 1) + nz * (size_t)(m - 1)));
        WG(f, gi(c, i - ng, j, k), m) = b2[q];
        WG(f, gi(c, nx + i, j, k), m) = b1[q];
      }
  if (per[1])
    for (int m = 1; m <= nvar; m++)
      for (int k = 1; k <= nz; k++) for (int j = 1; j <= ng; j++) for (int i = 1; i <= nx; i++) {
        size_t q = (size_t)(i - 1) + nx * ((size_t)(j - 1) + ng * ((size_t)(k - 1) + nz * (size_t)(m - 1)));
        WG(f, gi(c, i, j - ng, k), m) = b4[q];
        WG(f, gi(c, i, ny + j, k), m) = b3[q];
      }
  if (per[2])
    for (int m = 1; m <= nvar; m++)
      for (int k = 1; k <= ng; k++) for (int j = 1; j <= ny; j++) for (int i = 1; i <= nx; i++) {
        size_t q = (size_t)(i - 1) + nx * ((size_t)(j - 1) + ny * ((size_t)(k - 1) + ng * (size_t)(m - 1)));
        WG(f, gi(c, i, j, k - ng), m) = b6[q];
        WG(f, gi(c, i, j, nz + k), m) = b5[q];
      }
  free(b1); free(b2); free(b3); free(b4); free(b5); free(b6);
}

/* the ghost point l of face ilat (1..6) at tangential indices (a, b), and the
 * interior point at normal index n (1..nx etc.) on the same line */
static size_t face_pt(const ox_ctx *c, int ilat, int a, int b, int n) {
  int dir = (ilat - 1) / 2;
  if (dir == 0) return gi(c, n, a, b);
  if (dir == 1) return gi(c, a, n, b);
  return gi(c, a, b, n);
}

/* bcextr_sub_cuf (kernels_gpu.F90:4092-4327), every side: the boundary cell's
 * mass fractions into w_aux, then ng ghosts with its species and momentum and the
 * energy of T = p0 / (rho R_mix) */
static void bc_extr_sub(ox_ctx *c, int ilat, double *w, double *wa) {
  int dir = (ilat - 1) / 2, hi = (ilat - 1) % 2, ng = c->g.ng;
  int n = dir == 0 ? c->g.nx : (dir == 1 ? c->g.ny : c->g.nz);
  int na = dir == 0 ? c->g.ny : c->g.nx, nb = dir == 2 ? c->g.ny : c->g.nz;
  int ib = hi ? n : 1;
  for (int b = 1; b <= nb; b++)
    for (int a = 1; a <= na; a++) {
      size_t p = face_pt(c, ilat, a, b, ib);
      double rho = rho_from_w(c, w, p);
      for (int lsp = 1; lsp <= NS; lsp++) WG(wa, p, lsp) = WG(w, p, lsp) / rho;
    }
  for (int b = 1; b <= nb; b++)
    for (int a = 1; a <= na; a++)
      for (int l = 1; l <= ng; l++) {
        size_t p = face_pt(c, ilat, a, b, ib), q = face_pt(c, ilat, a, b, hi ? n + l : 1 - l);
        double rho = rho_from_w(c, w, p);
        double rhou = WG(w, p, I_U), rhov = WG(w, p, I_V), rhow = WG(w, p, I_W);
        double rmixtloc = rmix_wa(c, wa, p);
        double tt = c->p.p0 / rho / rmixtloc;
        double ee = mixture_e_wa(c, tt, wa, p);
        for (int lsp = 1; lsp <= NS; lsp++) WG(w, q, lsp) = WG(w, p, lsp);
        WG(w, q, I_U) = rhou;
        WG(w, q, I_V) = rhov;
        WG(w, q, I_W) = rhow;
        WG(w, q, I_E) = rho * ee + 0.5 * (rhou * rhou + rhov * rhov + rhow * rhow) / rho;
      }
}

/* bcwall_cuf (kernels_gpu.F90:5437-5545): isothermal wall on the y sides (the
 * x and z sides do nothing): the first ng interior layers' mass fractions into
 * w_aux, then ghost 1-l (ny+l) mirrors layer l (ny+1-l) with the velocity
 * reversed, the pressure kept and T' = max(2 T_wall - T, 200 K) */
static void bc_wall_iso(ox_ctx *c, int ilat, double *w, double *wa) {
  if (ilat != 3 && ilat != 4) return;
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz, ng = c->g.ng;
  for (int k = 1; k <= nz; k++)
    for (int i = 1; i <= nx; i++)
      for (int l = 1; l <= ng; l++) {
        size_t p = gi(c, i, ilat == 3 ? l : ny + 1 - l, k);
        double rho = rho_from_w(c, w, p);
        for (int lsp = 1; lsp <= NS; lsp++) WG(wa, p, lsp) = WG(w, p, lsp) / rho;
      }
  for (int k = 1; k <= nz; k++)
    for (int i = 1; i <= nx; i++)
      for (int l = 1; l <= ng; l++) {
        size_t p = gi(c, i, ilat == 3 ? l : ny + 1 - l, k), q = gi(c, i, ilat == 3 ? 1 - l : ny + l, k);
        double rho = rho_from_w(c, w, p);
        double uu = WG(w, p, I_U) / rho, vv = WG(w, p, I_V) / rho, ww = WG(w, p, I_W) / rho;
        double rhoe = WG(w, p, I_E);
        double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
        double ee = rhoe / rho - qq;
        double Y[MAXNS];
        for (int lsp = 1; lsp <= NS; lsp++) Y[lsp - 1] = WG(wa, p, lsp);
        double tt = temperature_from_poly(c, c->cv, ee, WG(wa, p, J_T), Y);
        double rmixtloc = rmix_wa(c, wa, p);
        double pp = rho * tt * rmixtloc;
        tt = 2.0 * c->p.T_wall - tt;
        if (tt < 200.0) tt = 200.0;
        ee = mixture_e_wa(c, tt, wa, p);
        rho = pp / tt / rmixtloc;
        for (int lsp = 1; lsp <= NS; lsp++) WG(w, q, lsp) = rho * WG(wa, p, lsp);
        WG(w, q, I_U) = -rho * uu;
        WG(w, q, I_V) = -rho * vv;
        WG(w, q, I_W) = -rho * ww;
        WG(w, q, I_E) = rho * (ee + qq);
      }
}

/* update_ghost (multideal_gpu.F90:1165-1238) for tags 0 (nothing), 1 (bcfree_cuf
 * :5073-5100, left side only), 2 (bcextr_cuf :5209-5288), 4 (bcextr_sub_cuf
 * :4092-4327), 5 (bcsym_cuf :5395-5435, y sides only), 6 (bcwall_cuf :5437-5545),
 * 7 (bcoutopenfoam_cuf :5290-5393), 8 (bcwall_ad_cuf :5749-5852).  Tags 4 and 6
 * need w_aux (the mass fractions they write back, the Newton guess of tag 6). */
void ox_update_ghost_aux(ox_ctx *c, double *w, double *wa, int do_swap) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz, ng = c->g.ng, nv = c->nv;
  for (int ilat = 1; ilat <= 6; ilat++) {
    int tag = c->p.bctags[ilat - 1];
    if (tag == 4) { bc_extr_sub(c, ilat, w, wa); continue; }
    if (tag == 6) { bc_wall_iso(c, ilat, w, wa); continue; }
    if (tag == 5) {
      /* symmetry about the first (last) row: the y velocity there is set to zero,
       * ghost 1-l mirrors row l on the lower side, ghost ny+l mirrors ny-l on the upper */
      if (ilat != 3 && ilat != 4) continue;
      for (int k = 1; k <= nz; k++)
        for (int i = 1; i <= nx; i++) {
          WG(w, gi(c, i, ilat == 3 ? 1 : ny, k), I_V) = 0.0;
          for (int l = 1; l <= ng; l++) {
            size_t q = gi(c, i, ilat == 3 ? 1 - l : ny + l, k), p = gi(c, i, ilat == 3 ? l : ny - l, k);
            for (int lsp = 1; lsp <= NS; lsp++) WG(w, q, lsp) = WG(w, p, lsp);
            WG(w, q, I_U) = WG(w, p, I_U);
            WG(w, q, I_V) = -WG(w, p, I_V);
            WG(w, q, I_W) = WG(w, p, I_W);
            WG(w, q, I_E) = WG(w, p, I_E);
          }
        }
      continue;
    }
    if (tag == 7) {
      /* zero-gradient outflow; the normal momentum's ghosts are zero where the
       * boundary cell's flow enters the domain.  The lower z side tests the x
       * momentum (as the reference does). */
      int dir = (ilat - 1) / 2, hi = (ilat - 1) % 2;
      int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
      int na = dir == 0 ? ny : nx, nb = dir == 2 ? ny : nz;
      int mn = I_U + dir, mtest = ilat == 5 ? I_U : mn;
      for (int b = 1; b <= nb; b++)
        for (int a = 1; a <= na; a++) {
          size_t p = face_pt(c, ilat, a, b, hi ? n : 1);
          int enter = hi ? WG(w, p, mtest) < 0.0 : WG(w, p, mtest) > 0.0;
          for (int l = 1; l <= ng; l++) {
            size_t q = face_pt(c, ilat, a, b, hi ? n + l : 1 - l);
            for (int m = 1; m <= nv; m++) WG(w, q, m) = (m == mn && enter) ? 0.0 : WG(w, p, m);
          }
        }
      continue;
    }
    if (tag == 1 && ilat == 1 && c->p.winf) {
      for (int k = 1; k <= nz; k++) for (int j = 1; j <= ny; j++) for (int l = 1; l <= ng; l++)
        for (int m = 1; m <= nv; m++) WG(w, gi(c, 1 - l, j, k), m) = c->p.winf[m - 1];
    } else if (tag == 2) {
      for (int m = 1; m <= nv; m++) {
        if (ilat == 1) { for (int k = 1; k <= nz; k++) for (int j = 1; j <= ny; j++) for (int l = 1; l <= ng; l++) WG(w, gi(c, 1 - l, j, k), m) = WG(w, gi(c, 1, j, k), m); }
        if (ilat == 2) { for (int k = 1; k <= nz; k++) for (int j = 1; j <= ny; j++) for (int l = 1; l <= ng; l++) WG(w, gi(c, nx + l, j, k), m) = WG(w, gi(c, nx, j, k), m); }
        if (ilat == 3) { for (int k = 1; k <= nz; k++) for (int i = 1; i <= nx; i++) for (int l = 1; l <= ng; l++) WG(w, gi(c, i, 1 - l, k), m) = WG(w, gi(c, i, 1, k), m); }
        if (ilat == 4) { for (int k = 1; k <= nz; k++) for (int i = 1; i <= nx; i++) for (int l = 1; l <= ng; l++) WG(w, gi(c, i, ny + l, k), m) = WG(w, gi(c, i, ny, k), m); }
        if (ilat == 5) { for (int j = 1; j <= ny; j++) for (int i = 1; i <= nx; i++) for (int l = 1; l <= ng; l++) WG(w, gi(c, i, j, 1 - l), m) = WG(w, gi(c, i, j, 1), m); }
        if (ilat == 6) { for (int j = 1; j <= ny; j++) for (int i = 1; i <= nx; i++) for (int l = 1; l <= ng; l++) WG(w, gi(c, i, j, nz + l), m) = WG(w, gi(c, i, j, nz), m); }
      }
    } else if (tag == 8) {
      for (int m = 1; m <= nv; m++) {
        double sg = (m == I_U || m == I_V || m == I_W) ? -1.0 : 1.0;
        if (ilat == 1) { for (int k = 1; k <= nz; k++) for (int j = 1; j <= ny; j++) for (int l = 1; l <= ng; l++) WG(w, gi(c, 1 - l, j, k), m) = sg * WG(w, gi(c, l, j, k), m); }
        if (ilat == 2) { for (int k = 1; k <= nz; k++) for (int j = 1; j <= ny; j++) for (int l = 1; l <= ng; l++) WG(w, gi(c, nx + l, j, k), m) = sg * WG(w, gi(c, nx + 1 - l, j, k), m); }
        if (ilat == 3) { for (int k = 1; k <= nz; k++) for (int l = 1; l <= ng; l++) for (int i = 1; i <= nx; i++) WG(w, gi(c, i, 1 - l, k), m) = sg * WG(w, gi(c, i, l, k), m); }
        if (ilat == 4) { for (int k = 1; k <= nz; k++) for (int l = 1; l <= ng; l++) for (int i = 1; i <= nx; i++) WG(w, gi(c, i, ny + l, k), m) = sg * WG(w, gi(c, i, ny + 1 - l, k), m); }
        if (ilat == 5) { for (int l = 1; l <= ng; l++) for (int j = 1; j <= ny; j++) for (int i = 1; i <= nx; i++) WG(w, gi(c, i, j, 1 - l), m) = sg * WG(w, gi(c, i, j, l), m); }
        if (ilat == 6) { for (int l = 1; l <= ng; l++) for (int j = 1; j <= ny; j++) for (int i = 1; i <= nx; i++) WG(w, gi(c, i, j, nz + l), m) = sg * WG(w, gi(c, i, j, nz + 1 - l), m); }
      }
    }
  }
  if (do_swap == 1) ox_bcswap(c, w, c->nv);
}
void ox_update_ghost(ox_ctx *c, double *w, int do_swap) { ox_update_ghost_aux(c, w, NULL, do_swap); }

/* ---------------------------------------------------------------- Euler fluxes */
/* Roe state, compute_roe_average (kernels_gpu.F90:2986-3295) between points p and q */
typedef struct { double b1, b2, b3, rho, c, ci, h, uu, vv, ww; double yy[MAXNS], prhoi[MAXNS]; } roe_t;

static void roe_average(ox_ctx *c, const double *wa, size_t p, size_t q, roe_t *R) {
  double rho = WG(wa, p, J_R), uu = WG(wa, p, J_U), vv = WG(wa, p, J_V), ww = WG(wa, p, J_W);
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double h = WG(wa, p, J_H), pp = WG(wa, p, J_P);
  double ee = h - pp / rho - qq;
  double rho_L = rho, ee_L = ee;
  double rhop = WG(wa, q, J_R), up = WG(wa, q, J_U), vp = WG(wa, q, J_V), wp = WG(wa, q, J_W);
  double qqp = 0.5 * (up * up + vp * vp + wp * wp);
  double hp = WG(wa, q, J_H), ppp = WG(wa, q, J_P);
  double eep = hp - ppp / rhop - qqp;
  double r = sqrt(rhop / rho);
  rho = r * rho_L;
  double rp1 = 1.0 / (r + 1.0);
  uu = (r * up + uu) * rp1;
  vv = (r * vp + vv) * rp1;
  ww = (r * wp + ww) * rp1;
  h = (r * hp + h) * rp1;
  qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  ee = (r * eep + ee) * rp1;
  double p_over_rho = h - ee - qq;
  double rmixtloc = 0.0;
  double drho_SLV[MAXNS];
  for (int lsp = 1; lsp <= NS; lsp++) {
    double yy = WG(wa, p, lsp), yyp = WG(wa, q, lsp);
    drho_SLV[lsp - 1] = rhop * yyp - rho_L * yy;
    yy = (r * yyp + yy) * rp1;
    rmixtloc = rmixtloc + c->rgas[lsp - 1] * yy;
    R->yy[lsp - 1] = yy;
  }
  double told = p_over_rho / rmixtloc;
  double tt = ox_temperature_from_e(c, ee, told, R->yy);
  double cploc = mix_cp(c, tt, R->yy);
  double gamloc = cploc / (cploc - rmixtloc);
  double gm1loc = gamloc - 1.0;
  double p_e = rho * gm1loc;
  for (int lsp = 1; lsp <= NS; lsp++) R->prhoi[lsp - 1] = species_poly_int(c, c->cv, tt, lsp);
  for (int lsp = 1; lsp <= NS; lsp++) {
    double eei = R->prhoi[lsp - 1];
    R->prhoi[lsp - 1] = c->rgas[lsp - 1] * tt + gm1loc * (ee - eei);
  }
  double etot = ee + qq;
  double dp_SLV = ppp - pp;
  double de_SLV = eep - ee_L;
  double pede = p_e * de_SLV;
  double dp_err = dp_SLV - pede;
  double den_correction = pede * pede;
  for (int lsp = 1; lsp <= NS; lsp++) {
    double prhoidrho = R->prhoi[lsp - 1] * drho_SLV[lsp - 1];
    dp_err = dp_err - prhoidrho;
    den_correction = den_correction + prhoidrho * prhoidrho;
  }
  double dpfact = dp_err / dmax(den_correction, 0.000001);
  p_e = p_e * (1.0 + pede * dpfact);
  for (int lsp = 1; lsp <= NS; lsp++)
    R->prhoi[lsp - 1] = R->prhoi[lsp - 1] * (1.0 + R->prhoi[lsp - 1] * drho_SLV[lsp - 1] * dpfact);
  double cc = p_over_rho / rho * p_e;
  for (int lsp = 1; lsp <= NS; lsp++) cc = cc + R->yy[lsp - 1] * R->prhoi[lsp - 1];
  R->c = sqrt(cc);
  R->ci = 1.0 / R->c;
  R->b3 = etot;
  R->b2 = p_e / (rho * cc);
  R->b1 = -R->b2 * (etot - 2.0 * qq);
  R->rho = rho; R->h = h; R->uu = uu; R->vv = vv; R->ww = ww;
}

/* eigenvectors_x/y/z (kernels_gpu.F90:2703-2984); dir 0,1,2.  el, er are (nv,nv)
 * column-major: el[(m-1)*nv + n-1] = el(n,m). */
static void eigenvectors(ox_ctx *c, int dir, const roe_t *R, double *el, double *er) {
  int nv = c->nv;
  double vel[3] = {R->uu, R->vv, R->ww};
  double un = vel[dir];
  int it1 = dir == 0 ? 1 : 0, it2 = dir == 2 ? 1 : 2;      /* tangential components */
  int In = I_U + dir, It1 = I_U + it1, It2 = I_U + it2;
  double cci = R->ci * R->ci;
#define EL(n, m) el[(size_t)((m) - 1) * nv + (n) - 1]
#define ER(n, m) er[(size_t)((m) - 1) * nv + (n) - 1]
  memset(el, 0, sizeof(double) * nv * nv);
  memset(er, 0, sizeof(double) * nv * nv);
  for (int lsp = 1; lsp <= NS; lsp++) {
    double b1i = R->b1 + R->prhoi[lsp - 1] * cci;
    EL(lsp, 1) = 0.5 * (b1i + un * R->ci);
    EL(lsp, NS + 2) = -vel[it1];
    EL(lsp, NS + 3) = -vel[it2];
    EL(lsp, NS + 4) = 0.5 * (b1i - un * R->ci);
    EL(lsp, lsp + 1) = 1.0;
    EL(I_U, 1 + lsp) = R->b2 * R->uu * R->yy[lsp - 1];
    EL(I_V, 1 + lsp) = R->b2 * R->vv * R->yy[lsp - 1];
    EL(I_W, 1 + lsp) = R->b2 * R->ww * R->yy[lsp - 1];
    EL(I_E, 1 + lsp) = -R->b2 * R->yy[lsp - 1];
    for (int msp = 1; msp <= NS; msp++) {
      double b1m = R->b1 + R->prhoi[msp - 1] * cci;
      EL(msp, 1 + lsp) = EL(msp, 1 + lsp) - b1m * R->yy[lsp - 1];
    }
  }
  EL(In, 1) = -0.5 * (R->b2 * un + R->ci);
  EL(It1, 1) = -0.5 * (R->b2 * vel[it1]);
  EL(It2, 1) = -0.5 * (R->b2 * vel[it2]);
  EL(I_E, 1) = 0.5 * R->b2;
  EL(It1, NS + 2) = 1.0;
  EL(It2, NS + 3) = 1.0;
  EL(In, NS + 4) = -0.5 * (R->b2 * un - R->ci);
  EL(It1, NS + 4) = -0.5 * (R->b2 * vel[it1]);
  EL(It2, NS + 4) = -0.5 * (R->b2 * vel[it2]);
  EL(I_E, NS + 4) = 0.5 * R->b2;
  for (int lsp = 1; lsp <= NS; lsp++) {
    double b3i = R->b3 - R->prhoi[lsp - 1] / R->b2 * cci;
    ER(1, lsp) = R->yy[lsp - 1];
    ER(1 + lsp, lsp) = 1.0;
    ER(4 + NS, lsp) = R->yy[lsp - 1];
    ER(1 + lsp, I_U) = R->uu;
    ER(1 + lsp, I_V) = R->vv;
    ER(1 + lsp, I_W) = R->ww;
    ER(1 + lsp, I_E) = b3i;
  }
  ER(1, In) = un - R->c;
  ER(1, It1) = vel[it1];
  ER(1, It2) = vel[it2];
  ER(1, I_E) = R->h - un * R->c;
  ER(NS + 2, It1) = 1.0;
  ER(NS + 3, It2) = 1.0;
  ER(NS + 4, In) = un + R->c;
  ER(NS + 4, It1) = vel[it1];
  ER(NS + 4, It2) = vel[it2];
  ER(NS + 2, I_E) = vel[it1];
  ER(NS + 3, I_E) = vel[it2];
  ER(NS + 4, I_E) = R->h + un * R->c;
#undef EL
#undef ER
}

/* wenorec_1d / wenorec_1d_rusanov (kernels_gpu.F90:2065-2637): vp, vm are
 * (nvar, 8) column-major with 1-based stencil slot; betascale per variable. */
static void wenorec(int nvar, const double *vp, const double *vm, double *vhat, int iweno, int ord,
                    int version, const double *bs) {
#define VP(m, i) vp[(size_t)((i) - 1) * nvar + (m) - 1]
#define VM(m, i) vm[(size_t)((i) - 1) * nvar + (m) - 1]
  double betap[4], betam[4], dwe[4];
  int i = iweno;
  if (ord == 1) {
    for (int m = 1; m <= nvar; m++) vhat[m - 1] = VP(m, i) + VM(m, i + 1);
  } else if (ord == 2) {
    dwe[1] = 2.0 / 3.0; dwe[0] = 1.0 / 3.0;
    for (int m = 1; m <= nvar; m++) {
      double t;
      t = VP(m, i) - VP(m, i - 1); betap[0] = t * t;
      t = VP(m, i + 1) - VP(m, i); betap[1] = t * t;
      betap[1] = bs[m - 1] * betap[1]; betap[0] = bs[m - 1] * betap[0];
      t = VM(m, i + 2) - VM(m, i + 1); betam[0] = t * t;
      t = VM(m, i + 1) - VM(m, i); betam[1] = t * t;
      betam[1] = bs[m - 1] * betam[1]; betam[0] = bs[m - 1] * betam[0];
      double sump = 0.0, summ = 0.0;
      for (int l = 0; l <= 1; l++) {
        t = 0.000001 + betap[l]; betap[l] = dwe[l] / (t * t);
        t = 0.000001 + betam[l]; betam[l] = dwe[l] / (t * t);
        sump = sump + betap[l]; summ = summ + betam[l];
      }
      for (int l = 0; l <= 1; l++) { betap[l] = betap[l] / sump; betam[l] = betam[l] / summ; }
      double vminus = betap[0] * (-VP(m, i - 1) + 3 * VP(m, i)) + betap[1] * (VP(m, i) + VP(m, i + 1));
      double vplus = betam[0] * (-VM(m, i + 2) + 3 * VM(m, i + 1)) + betam[1] * (VM(m, i) + VM(m, i + 1));
      vhat[m - 1] = 0.5 * (vminus + vplus);
    }
  } else if (ord == 3) {
    dwe[0] = 1.0 / 10.0; dwe[1] = 6.0 / 10.0; dwe[2] = 3.0 / 10.0;
    const double d0 = 13.0 / 12.0, d1 = 1.0 / 4.0;
    const double c0 = 1.0 / 3.0, c1 = 5.0 / 6.0, c2 = -1.0 / 6.0, c3 = -7.0 / 6.0, c4 = 11.0 / 6.0;
    for (int m = 1; m <= nvar; m++) {
      double a, b;
      a = VP(m, i) - 2.0 * VP(m, i + 1) + VP(m, i + 2); b = 3.0 * VP(m, i) - 4.0 * VP(m, i + 1) + VP(m, i + 2);
      betap[2] = d0 * (a * a) + d1 * (b * b);
      a = VP(m, i - 1) - 2.0 * VP(m, i) + VP(m, i + 1); b = VP(m, i - 1) - VP(m, i + 1);
      betap[1] = d0 * (a * a) + d1 * (b * b);
      a = VP(m, i) - 2.0 * VP(m, i - 1) + VP(m, i - 2); b = 3.0 * VP(m, i) - 4.0 * VP(m, i - 1) + VP(m, i - 2);
      betap[0] = d0 * (a * a) + d1 * (b * b);
      betap[2] = bs[m - 1] * betap[2]; betap[1] = bs[m - 1] * betap[1]; betap[0] = bs[m - 1] * betap[0];
      a = VM(m, i + 1) - 2.0 * VM(m, i) + VM(m, i - 1); b = 3.0 * VM(m, i + 1) - 4.0 * VM(m, i) + VM(m, i - 1);
      betam[2] = d0 * (a * a) + d1 * (b * b);
      a = VM(m, i + 2) - 2.0 * VM(m, i + 1) + VM(m, i); b = VM(m, i + 2) - VM(m, i);
      betam[1] = d0 * (a * a) + d1 * (b * b);
      a = VM(m, i + 1) - 2.0 * VM(m, i + 2) + VM(m, i + 3); b = 3.0 * VM(m, i + 1) - 4.0 * VM(m, i + 2) + VM(m, i + 3);
      betam[0] = d0 * (a * a) + d1 * (b * b);
      betam[2] = bs[m - 1] * betam[2]; betam[1] = bs[m - 1] * betam[1]; betam[0] = bs[m - 1] * betam[0];
      double sump = 0.0, summ = 0.0;
      if (version == 0) {
        for (int l = 0; l <= 2; l++) {
          double t = 0.000001 + betap[l]; betap[l] = dwe[l] / (t * t);
          t = 0.000001 + betam[l]; betam[l] = dwe[l] / (t * t);
          sump = sump + betap[l]; summ = summ + betam[l];
        }
      } else {
        const double eps40 = 1.0e-40;
        double tau5p = fabs(betap[0] - betap[2]) + eps40;
        double tau5m = fabs(betam[0] - betam[2]) + eps40;
        for (int l = 0; l <= 2; l++) {
          betap[l] = (betap[l] + eps40) / (betap[l] + tau5p);
          betam[l] = (betam[l] + eps40) / (betam[l] + tau5m);
        }
        for (int l = 0; l <= 2; l++) {
          betap[l] = dwe[l] / betap[l];
          betam[l] = dwe[l] / betam[l];
          sump = sump + betap[l]; summ = summ + betam[l];
        }
      }
      for (int l = 0; l <= 2; l++) { betap[l] = betap[l] / sump; betam[l] = betam[l] / summ; }
      double vminus = betap[2] * (c0 * VP(m, i) + c1 * VP(m, i + 1) + c2 * VP(m, i + 2)) +
                      betap[1] * (c2 * VP(m, i - 1) + c1 * VP(m, i) + c0 * VP(m, i + 1)) +
                      betap[0] * (c0 * VP(m, i - 2) + c3 * VP(m, i - 1) + c4 * VP(m, i));
      double vplus = betam[2] * (c0 * VM(m, i + 1) + c1 * VM(m, i) + c2 * VM(m, i - 1)) +
                     betam[1] * (c2 * VM(m, i + 2) + c1 * VM(m, i + 1) + c0 * VM(m, i)) +
                     betam[0] * (c0 * VM(m, i + 3) + c3 * VM(m, i + 2) + c4 * VM(m, i + 1));
      vhat[m - 1] = vminus + vplus;
    }
  } else if (ord == 4) {
    dwe[0] = 1.0 / 35.0; dwe[1] = 12.0 / 35.0; dwe[2] = 18.0 / 35.0; dwe[3] = 4.0 / 35.0;
    const double d1 = 1.0 / 36.0, d2 = 13.0 / 12.0, d3 = 781.0 / 720.0;
    for (int m = 1; m <= nvar; m++) {
      double a, b, e;
      a = -11 * VP(m, i) + 18 * VP(m, i + 1) - 9 * VP(m, i + 2) + 2 * VP(m, i + 3);
      b = 2 * VP(m, i) - 5 * VP(m, i + 1) + 4 * VP(m, i + 2) - VP(m, i + 3);
      e = -VP(m, i) + 3 * VP(m, i + 1) - 3 * VP(m, i + 2) + VP(m, i + 3);
      betap[3] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
      a = -2 * VP(m, i - 1) - 3 * VP(m, i) + 6 * VP(m, i + 1) - VP(m, i + 2);
      b = VP(m, i - 1) - 2 * VP(m, i) + VP(m, i + 1);
      e = -VP(m, i - 1) + 3 * VP(m, i) - 3 * VP(m, i + 1) + VP(m, i + 2);
      betap[2] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
      a = VP(m, i - 2) - 6 * VP(m, i - 1) + 3 * VP(m, i) + 2 * VP(m, i + 1);
      b = VP(m, i - 1) - 2 * VP(m, i) + VP(m, i + 1);
      e = -VP(m, i - 2) + 3 * VP(m, i - 1) - 3 * VP(m, i) + VP(m, i + 1);
      betap[1] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
      a = -2 * VP(m, i - 3) + 9 * VP(m, i - 2) - 18 * VP(m, i - 1) + 11 * VP(m, i);
      b = -VP(m, i - 3) + 4 * VP(m, i - 2) - 5 * VP(m, i - 1) + 2 * VP(m, i);
      e = -VP(m, i - 3) + 3 * VP(m, i - 2) - 3 * VP(m, i - 1) + VP(m, i);
      betap[0] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
      for (int l = 0; l <= 3; l++) betap[l] = bs[m - 1] * betap[l];
      a = -11 * VM(m, i + 1) + 18 * VM(m, i) - 9 * VM(m, i - 1) + 2 * VM(m, i - 2);
      b = 2 * VM(m, i + 1) - 5 * VM(m, i) + 4 * VM(m, i - 1) - VM(m, i - 2);
      e = -VM(m, i + 1) + 3 * VM(m, i) - 3 * VM(m, i - 1) + VM(m, i - 2);
      betam[3] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
      a = -2 * VM(m, i + 2) - 3 * VM(m, i + 1) + 6 * VM(m, i) - VM(m, i - 1);
      b = VM(m, i + 2) - 2 * VM(m, i + 1) + VM(m, i);
      e = -VM(m, i + 2) + 3 * VM(m, i + 1) - 3 * VM(m, i) + VM(m, i - 1);
      betam[2] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
      a = VM(m, i + 3) - 6 * VM(m, i + 2) + 3 * VM(m, i + 1) + 2 * VM(m, i);
      b = VM(m, i + 2) - 2 * VM(m, i + 1) + VM(m, i);
      e = -VM(m, i + 3) + 3 * VM(m, i + 2) - 3 * VM(m, i + 1) + VM(m, i);
      betam[1] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
      a = -2 * VM(m, i + 4) + 9 * VM(m, i + 3) - 18 * VM(m, i + 2) + 11 * VM(m, i + 1);
      b = -VM(m, i + 4) + 4 * VM(m, i + 3) - 5 * VM(m, i + 2) + 2 * VM(m, i + 1);
      e = -VM(m, i + 4) + 3 * VM(m, i + 3) - 3 * VM(m, i + 2) + VM(m, i + 1);
      betam[0] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
      for (int l = 0; l <= 3; l++) betam[l] = bs[m - 1] * betam[l];
      double sump = 0.0, summ = 0.0;
      for (int l = 0; l <= 3; l++) {
        double t = 0.000001 + betap[l]; betap[l] = dwe[l] / (t * t);
        t = 0.000001 + betam[l]; betam[l] = dwe[l] / (t * t);
        sump = sump + betap[l]; summ = summ + betam[l];
      }
      for (int l = 0; l <= 3; l++) { betap[l] = betap[l] / sump; betam[l] = betam[l] / summ; }
      double vminus = betap[3] * (6 * VP(m, i) + 26 * VP(m, i + 1) - 10 * VP(m, i + 2) + 2 * VP(m, i + 3)) +
                      betap[2] * (-2 * VP(m, i - 1) + 14 * VP(m, i) + 14 * VP(m, i + 1) - 2 * VP(m, i + 2)) +
                      betap[1] * (2 * VP(m, i - 2) - 10 * VP(m, i - 1) + 26 * VP(m, i) + 6 * VP(m, i + 1)) +
                      betap[0] * (-6 * VP(m, i - 3) + 26 * VP(m, i - 2) - 46 * VP(m, i - 1) + 50 * VP(m, i));
      double vplus = betam[3] * (6 * VM(m, i + 1) + 26 * VM(m, i) - 10 * VM(m, i - 1) + 2 * VM(m, i - 2)) +
                     betam[2] * (-2 * VM(m, i + 2) + 14 * VM(m, i + 1) + 14 * VM(m, i) - 2 * VM(m, i - 1)) +
                     betam[1] * (2 * VM(m, i + 3) - 10 * VM(m, i + 2) + 26 * VM(m, i + 1) + 6 * VM(m, i)) +
                     betam[0] * (-6 * VM(m, i + 4) + 26 * VM(m, i + 3) - 46 * VM(m, i + 2) + 50 * VM(m, i + 1));
      vhat[m - 1] = (vminus + vplus) / 24.0;
    }
  }
#undef VP
#undef VM
}

/* One face flux of euler_{x,y,z}_fluxes_hybrid[_rusanov]_kernel
 * (kernels_gpu.F90:88-730, 795-1425, 1427-2063).  p is the point left of the
 * face, st the stride along the sweep; face is the face index along the sweep
 * (for force_zero_flux) and nmax the number of cells along it. */
static void face_flux(ox_ctx *c, int dir, const double *wa, size_t p, long st, int face, int nmax, double *fh) {
  int nv = c->nv, ws = c->p.weno_scheme, wsz = 2 * ws;
  int In = I_U + dir, Jn = J_U + dir;
  int fz = (face == 0 && c->p.force_zero_flux[2 * dir] == 1) || (face == nmax && c->p.force_zero_flux[2 * dir + 1] == 1);
#define PT(s) ((size_t)((long)p + (long)(s) * st))
  /* the sensor window is ii = i-ws+1 .. i+ws, offsets -ws+1 .. ws from the face point */
  int ishk = 0;
  for (int s = -ws + 1; s <= ws; s++)
    if (WG(wa, PT(s), J_DUC) > c->p.sensor_threshold) ishk = 1;
  if (ishk == 0) {
    int lmax = c->p.ep_order / 2;
    if (lmax < 1) lmax = 1;
    int nkeep = c->p.nkeep;
    for (int lsp = 1; lsp <= NS; lsp++) {
      double ft1 = 0.0;
      for (int l = 1; l <= lmax; l++) {
        double uvs1 = 0.0;
        for (int m = 0; m <= l - 1; m++) {
          double rhoi = WG(wa, PT(-m), J_R), uui = WG(wa, PT(-m), Jn), yyi = WG(wa, PT(-m), lsp);
          double rhoip = WG(wa, PT(-m + l), J_R), uuip = WG(wa, PT(-m + l), Jn), yyip = WG(wa, PT(-m + l), lsp);
          double rhom = rhoi + rhoip, drhof;
          if (nkeep <= 0) {
            drhof = 1.0;
          } else {
            double drho = 2.0 * (rhoip - rhoi) / rhom;
            double t = (0.5 * drho) * (0.5 * drho), t2 = t;
            double sumden = 1.0 + t / 3.0;
            for (int n = 2; n <= nkeep; n++) { int n2 = 2 * n; t = t2 * t; sumden = sumden + t / (1.0 + n2); }
            drhof = 1.0 / sumden;
          }
          double uv_part = (uui + uuip) * rhom * drhof;
          uvs1 = uvs1 + uv_part * (yyi + yyip);
        }
        ft1 = ft1 + c->cd1[l][lmax] * uvs1;
      }
      double fh1 = 0.25 * ft1;
      if (fz) fh1 = 0.0;
      fh[lsp - 1] = fh1;
    }
    double ft2 = 0, ft3 = 0, ft4 = 0, ft5 = 0, ft6 = 0;
    for (int l = 1; l <= lmax; l++) {
      double uvs2 = 0, uvs3 = 0, uvs4 = 0, uvs5 = 0, uvs5_i = 0, uvs5_k = 0, uvs5_p = 0, uvs6 = 0;
      for (int m = 0; m <= l - 1; m++) {
        size_t a = PT(-m), b = PT(-m + l);
        double rhoi = WG(wa, a, J_R), uui = WG(wa, a, J_U), vvi = WG(wa, a, J_V), wwi = WG(wa, a, J_W);
        double enti = WG(wa, a, J_H), ppi = WG(wa, a, J_P);
        double rhoip = WG(wa, b, J_R), uuip = WG(wa, b, J_U), vvip = WG(wa, b, J_V), wwip = WG(wa, b, J_W);
        double entip = WG(wa, b, J_H), ppip = WG(wa, b, J_P);
        double uni = WG(wa, a, Jn), unip = WG(wa, b, Jn);
        double rhom = rhoi + rhoip;
        if (nkeep >= 0) {
          double eei = enti - ppi / rhoi - 0.5 * (uui * uui + vvi * vvi + wwi * wwi);
          double eeip = entip - ppip / rhoip - 0.5 * (uuip * uuip + vvip * vvip + wwip * wwip);
          double eem = eei + eeip, drhof, deef;
          if (nkeep == 0) {
            drhof = 1.0; deef = 1.0;
          } else {
            double drho = 2.0 * (rhoip - rhoi) / rhom;
            double dee = 2.0 * (eeip - eei) / eem;
            double tr = (0.5 * drho) * (0.5 * drho), te = (0.5 * dee) * (0.5 * dee);
            double tr2 = tr, te2 = te;
            double sumdenrho = 1.0 + tr / 3.0, sumdenee = 1.0 + te, sumnumee = 1.0 + te / 3.0;
            for (int n = 2; n <= nkeep; n++) {
              int n2 = 2 * n;
              tr = tr2 * tr; te = te2 * te;
              sumdenrho = sumdenrho + tr / (1.0 + n2);
              sumdenee = sumdenee + te;
              sumnumee = sumnumee + te / (1.0 + n2);
            }
            drhof = 1.0 / sumdenrho;
            deef = sumnumee / sumdenee;
          }
          double uv_part = (uni + unip) * rhom * drhof;
          uvs2 = uvs2 + uv_part * (uui + uuip);
          uvs3 = uvs3 + uv_part * (vvi + vvip);
          uvs4 = uvs4 + uv_part * (wwi + wwip);
          uvs5_i = uvs5_i + uv_part * eem * deef;
          uvs5_k = uvs5_k + uv_part * (uui * uuip + vvi * vvip + wwi * wwip);
          uvs5_p = uvs5_p + 4.0 * (uni * ppip + unip * ppi);
          uvs6 = uvs6 + (2.0) * (ppi + ppip);
        } else {
          double uv_part = (uni + unip) * rhom;
          uvs2 = uvs2 + uv_part * (uui + uuip);
          uvs3 = uvs3 + uv_part * (vvi + vvip);
          uvs4 = uvs4 + uv_part * (wwi + wwip);
          uvs5 = uvs5 + uv_part * (enti + entip);
          uvs6 = uvs6 + (2.0) * (ppi + ppip);
        }
      }
      double cl = c->cd1[l][lmax];
      ft2 = ft2 + cl * uvs2;
      ft3 = ft3 + cl * uvs3;
      ft4 = ft4 + cl * uvs4;
      ft5 = ft5 + cl * (nkeep >= 0 ? (uvs5_i + uvs5_k + uvs5_p) : uvs5);
      ft6 = ft6 + cl * uvs6;
    }
    double fm[3] = {0.25 * ft2, 0.25 * ft3, 0.25 * ft4};
    double fh5 = 0.25 * ft5;
    if (fz) { fm[0] = fm[1] = fm[2] = 0.0; fh5 = 0.0; }
    fm[dir] = fm[dir] + 0.5 * ft6;
    fh[I_U - 1] = fm[0]; fh[I_V - 1] = fm[1]; fh[I_W - 1] = fm[2]; fh[I_E - 1] = fh5;
    return;
  }
  /* upwind branch: stencil points ll = face + l - ws, l = 1..wsz */
  double gp[MAXNV * 8], gm[MAXNV * 8], fi_[MAXNV], bsc[MAXNV];
  double u0 = c->p.u0, rho0 = c->p.rho0;
  double u0_2 = u0 * u0, r2u2 = rho0 * rho0 * u0_2, r2u4 = r2u2 * u0_2;
  int ord = c->p.weno_scheme;   /* wenorec_ord = max(weno_scheme + ep_ord_change, 1) */
  if (ord < 1) ord = 1;
  if (c->p.flux_splitting == 1) {
    double r2u4i = 1.0 / r2u4;
    bsc[0] = 1.0 / r2u2;
    for (int lsp = 2; lsp <= NS; lsp++) bsc[lsp - 1] = bsc[0];
    bsc[I_U - 1] = r2u4i; bsc[I_V - 1] = r2u4i; bsc[I_W - 1] = r2u4i; bsc[I_E - 1] = r2u4i / u0_2;
    double evmax = -1.0;
    for (int l = 1; l <= wsz; l++) {
      size_t q = PT(l - ws);
      double un = WG(wa, q, Jn), cc = WG(wa, q, J_C);
      double evm = dmax(fabs(un - cc), fabs(un + cc));
      evmax = dmax(evm, evmax);
    }
    for (int l = 1; l <= wsz; l++) {
      size_t q = PT(l - ws);
      double rho = WG(wa, q, J_R), vel[3] = {WG(wa, q, J_U), WG(wa, q, J_V), WG(wa, q, J_W)};
      double h = WG(wa, q, J_H), pp = WG(wa, q, J_P);
      double rhou = rho * vel[dir];
      double rhoevm = rho * evmax;
      for (int lsp = 1; lsp <= NS; lsp++) {
        double yy = WG(wa, q, lsp);
        double evm = rhou * yy;
        double cc = 0.5 * (evm + rhoevm * yy);
        gp[(size_t)(l - 1) * nv + lsp - 1] = cc;
        gm[(size_t)(l - 1) * nv + lsp - 1] = evm - cc;
      }
      for (int d = 0; d < 3; d++) {
        double evm = (d == dir) ? vel[d] * rhou + pp : vel[d] * rhou;
        double cc = 0.5 * (evm + rhoevm * vel[d]);
        gp[(size_t)(l - 1) * nv + I_U + d - 1] = cc;
        gm[(size_t)(l - 1) * nv + I_U + d - 1] = evm - cc;
      }
      double evm = h * rhou;
      double cc = 0.5 * (evm + evmax * (rho * h - pp));
      gp[(size_t)(l - 1) * nv + I_E - 1] = cc;
      gm[(size_t)(l - 1) * nv + I_E - 1] = evm - cc;
    }
    wenorec(nv, gp, gm, fi_, ws, ord, c->p.weno_version, bsc);
    for (int m = 1; m <= nv; m++) fh[m - 1] = fi_[m - 1];
    return;
  }
  bsc[0] = 1.0 / r2u2;
  for (int lsp = 1; lsp <= NS + 1; lsp++) bsc[lsp - 1] = bsc[0];
  bsc[NS + 1] = 1.0 / r2u4;
  bsc[NS + 2] = bsc[NS + 1];
  bsc[NS + 3] = bsc[0];
  roe_t R;
  roe_average(c, wa, PT(0), PT(1), &R);
  double el[MAXNV * MAXNV], er[MAXNV * MAXNV], evmax[MAXNV];
  eigenvectors(c, dir, &R, el, er);
  for (int m = 1; m <= nv; m++) evmax[m - 1] = -1.0;
  for (int l = 1; l <= wsz; l++) {
    size_t q = PT(l - ws);
    double un = WG(wa, q, Jn), cc = WG(wa, q, J_C);
    evmax[0] = dmax(fabs(un - cc), evmax[0]);
    evmax[1] = dmax(fabs(un), evmax[1]);
    for (int lsp = 3; lsp <= NS + 3; lsp++) evmax[lsp - 1] = evmax[1];
    evmax[NS + 3] = dmax(fabs(un + cc), evmax[NS + 3]);
  }
  for (int l = 1; l <= wsz; l++) {
    size_t q = PT(l - ws);
    double rho = WG(wa, q, J_R), vel[3] = {WG(wa, q, J_U), WG(wa, q, J_V), WG(wa, q, J_W)};
    double h = WG(wa, q, J_H), pp = WG(wa, q, J_P);
    double rhou = rho * vel[dir];
    for (int lsp = 1; lsp <= NS; lsp++) fi_[lsp - 1] = rhou * WG(wa, q, lsp);
    fi_[I_U - 1] = vel[0] * rhou;
    fi_[I_V - 1] = vel[1] * rhou;
    fi_[I_W - 1] = vel[2] * rhou;
    fi_[In - 1] = fi_[In - 1] + pp;
    fi_[I_E - 1] = h * rhou;
    for (int m = 1; m <= nv; m++) {
      const double *e = el + (size_t)(m - 1) * nv;
      double wc = 0.0, gc = 0.0;
      for (int lsp = 1; lsp <= NS; lsp++) {
        wc = wc + e[lsp - 1] * rho * WG(wa, q, lsp);
        gc = gc + e[lsp - 1] * fi_[lsp - 1];
      }
      wc = wc + e[I_U - 1] * rho * vel[0]; gc = gc + e[I_U - 1] * fi_[I_U - 1];
      wc = wc + e[I_V - 1] * rho * vel[1]; gc = gc + e[I_V - 1] * fi_[I_V - 1];
      wc = wc + e[I_W - 1] * rho * vel[2]; gc = gc + e[I_W - 1] * fi_[I_W - 1];
      wc = wc + e[I_E - 1] * (rho * h - pp); gc = gc + e[I_E - 1] * fi_[I_E - 1];
      double cc = 0.5 * (gc + evmax[m - 1] * wc);
      gp[(size_t)(l - 1) * nv + m - 1] = cc;
      gm[(size_t)(l - 1) * nv + m - 1] = gc - cc;
    }
  }
  wenorec(nv, gp, gm, fi_, ws, ord, c->p.weno_version, bsc);
  for (int m = 1; m <= nv; m++) {
    double s = 0.0;
    for (int mm = 1; mm <= nv; mm++) s = s + er[(size_t)(m - 1) * nv + mm - 1] * fi_[mm - 1];
    fh[m - 1] = s;
  }
#undef PT
}

/* euler_x/y/z (multideal_gpu.F90:877-1044): faces nmin-1..nmax, then the update */
void ox_euler(ox_ctx *c, int dir, const double *wa, double *fhat, double *fl, int nmin, int nmax) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz, nv = c->nv;
  int n[3] = {nx, ny, nz};
  long st = dir == 0 ? 1 : (dir == 1 ? (long)c->nxg : (long)c->nxg * c->nyg);
  if (nmax - nmin < 0) return;
  int lo[3] = {1, 1, 1}, hi[3] = {nx, ny, nz};
  lo[dir] = nmin - 1; hi[dir] = nmax;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
  for (int k = lo[2]; k <= hi[2]; k++)
    for (int j = lo[1]; j <= hi[1]; j++)
      for (int i = lo[0]; i <= hi[0]; i++) {
        double fh[MAXNV];
        int idx[3] = {i, j, k};
        size_t p = gi(c, i, j, k);
        face_flux(c, dir, wa, p, st, idx[dir], n[dir], fh);
        for (int m = 1; m <= nv; m++) WG(fhat, p, m) = fh[m - 1];
      }
  const double *met = dir == 0 ? c->g.dcsidx : (dir == 1 ? c->g.detady : c->g.dzitdz);
  int ulo[3] = {1, 1, 1};
  ulo[dir] = nmin; hi[dir] = nmax;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = ulo[2]; k <= hi[2]; k++)
    for (int j = ulo[1]; j <= hi[1]; j++)
      for (int i = ulo[0]; i <= hi[0]; i++) {
        int idx[3] = {i, j, k};
        size_t p = gi(c, i, j, k), q = fi(c, i, j, k);
        for (int m = 1; m <= nv; m++)
          WF(fl, q, m) = WF(fl, q, m) + (WG(fhat, p, m) - WG(fhat, (size_t)((long)p - st), m)) * met[idx[dir] - 1];
      }
}

/* ---------------------------------------------------------------- viscous */
/* visflx_x/y/z_cuf (kernels_gpu.F90:3658-4031), mode 1, one direction */
static void visflx_dir(ox_ctx *c, int dir, const double *wa, double *fl, double *fhat) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz, nv = c->nv;
  long st = dir == 0 ? 1 : (dir == 1 ? (long)c->nxg : (long)c->nxg * c->nyg);
  const double *xc = dir == 0 ? c->g.x : (dir == 1 ? c->g.y : c->g.z);
  int ng = c->g.ng;
#define XC(i) xc[(i) + ng - 1]
  int lo[3] = {1, 1, 1}, hi[3] = {nx, ny, nz};
  lo[dir] = 0;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = lo[2]; k <= hi[2]; k++)
    for (int j = lo[1]; j <= hi[1]; j++)
      for (int i = lo[0]; i <= hi[0]; i++) {
        int idx[3] = {i, j, k};
        int ii = idx[dir];
        size_t p = gi(c, i, j, k), q = (size_t)((long)p + st);
        double uu = WG(wa, p, J_U), uup = WG(wa, q, J_U), vv = WG(wa, p, J_V), vvp = WG(wa, q, J_V);
        double ww = WG(wa, p, J_W), wwp = WG(wa, q, J_W), tt = WG(wa, p, J_T), ttp = WG(wa, q, J_T);
        double mu = WG(wa, p, J_MU), mup = WG(wa, q, J_MU);
        double k_cond = WG(wa, p, J_K_COND), k_cond_p = WG(wa, q, J_K_COND);
        double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
        double qqp = 0.5 * (uup * uup + vvp * vvp + wwp * wwp);
        double sigx = uup - uu, sigy = vvp - vv, sigz = wwp - ww;
        double sigq_tt = ttp - tt, sigq_qq = qqp - qq;
        double dxf = XC(ii + 1) - XC(ii);
        double muf = mu + mup;
        muf = 0.5 * muf / dxf;
        double k_cond_f = k_cond + k_cond_p;
        k_cond_f = 0.5 * k_cond_f / dxf;
        sigx = sigx * muf; sigy = sigy * muf; sigz = sigz * muf;
        double sigq = sigq_tt * k_cond_f + sigq_qq * muf;
        double rm = c->rgas[0] * WG(wa, p, 1);
        for (int lsp = 2; lsp <= NS; lsp++) rm = rm + c->rgas[lsp - 1] * WG(wa, p, lsp);
        double mwm = c->t.R_univ / rm;
        rm = c->rgas[0] * WG(wa, q, 1);
        for (int lsp = 2; lsp <= NS; lsp++) rm = rm + c->rgas[lsp - 1] * WG(wa, q, lsp);
        double mwmp = c->t.R_univ / rm;
        double mwmif = 0.5 * (mwmp + mwm) / (mwmp * mwm);
        mwmif = mwmif / dxf;
        double fhat_tmp = 0.0;
        for (int msp = 1; msp <= NS; msp++) {
          double rhodiff = 0.5 * (WG(wa, p, J_D_START + msp) + WG(wa, q, J_D_START + msp));
          double xxp = WG(wa, q, msp) * mwmp, xx = WG(wa, p, msp) * mwm;
          fhat_tmp = fhat_tmp + (xxp - xx) * rhodiff;
        }
        fhat_tmp = fhat_tmp * mwmif;
        double fhat_tmp_et = 0.0;
        for (int lsp = 1; lsp <= NS; lsp++) {
          double rhodiff = 0.5 * (WG(wa, p, J_D_START + lsp) + WG(wa, q, J_D_START + lsp));
          double yyp = WG(wa, q, lsp), yy = WG(wa, p, lsp);
          double yyf = 0.5 * (yyp + yy);
          double xxp = yyp * mwmp, xx = yy * mwm;
          double siglsp = -rhodiff * (xxp - xx) * mwmif + fhat_tmp * yyf;
          WG(fhat, p, lsp) = siglsp;
          double hh = species_poly_int(c, c->cp, tt, lsp);
          double hhp = species_poly_int(c, c->cp, ttp, lsp);
          double hhf = 0.5 * (hh + hhp);
          fhat_tmp_et = fhat_tmp_et + siglsp * hhf;
        }
        WG(fhat, p, I_U) = -sigx;
        WG(fhat, p, I_V) = -sigy;
        WG(fhat, p, I_W) = -sigz;
        WG(fhat, p, I_E) = -sigq + fhat_tmp_et;
      }
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        int idx[3] = {i, j, k};
        int ii = idx[dir];
        double dxhl = 2.0 / (XC(ii + 1) - XC(ii - 1));
        size_t p = gi(c, i, j, k), q = fi(c, i, j, k);
        for (int iv = 1; iv <= nv; iv++)
          WF(fl, q, iv) = WF(fl, q, iv) + dxhl * (WG(fhat, p, iv) - WG(fhat, (size_t)((long)p - st), iv));
      }
#undef XC
}

/* visflx_reduced_cuf (kernels_gpu.F90:3539-3656) */
static void visflx_reduced(ox_ctx *c, const double *wa, double *fl) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz;
  int lmax = c->p.visc_order / 2;
  size_t sx = 1, sy = (size_t)c->nxg, sz = (size_t)c->nxg * c->nyg;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        size_t p = gi(c, i, j, k), q = fi(c, i, j, k);
        double uu = WG(wa, p, J_U), vv = WG(wa, p, J_V), ww = WG(wa, p, J_W);
        double mu = WG(wa, p, J_MU), div3l = WG(wa, p, J_DIV);
        double ux = 0, vx = 0, wx = 0, mux = 0, divx3l = 0, uy = 0, vy = 0, wy = 0, muy = 0, divy3l = 0;
        double uz = 0, vz = 0, wz = 0, muz = 0, divz3l = 0;
        for (int l = 1; l <= lmax; l++) {
          double ccl = c->cd1[l][lmax];
#define D(s, J) (WG(wa, p + l * (s), J) - WG(wa, p - l * (s), J))
          ux = ux + ccl * D(sx, J_U); vx = vx + ccl * D(sx, J_V); wx = wx + ccl * D(sx, J_W);
          mux = mux + ccl * D(sx, J_MU); divx3l = divx3l + ccl * D(sx, J_DIV);
          uy = uy + ccl * D(sy, J_U); vy = vy + ccl * D(sy, J_V); wy = wy + ccl * D(sy, J_W);
          muy = muy + ccl * D(sy, J_MU); divy3l = divy3l + ccl * D(sy, J_DIV);
          uz = uz + ccl * D(sz, J_U); vz = vz + ccl * D(sz, J_V); wz = wz + ccl * D(sz, J_W);
          muz = muz + ccl * D(sz, J_MU); divz3l = divz3l + ccl * D(sz, J_DIV);
#undef D
        }
        double dx = c->g.dcsidx[i - 1], dy = c->g.detady[j - 1], dz = c->g.dzitdz[k - 1];
        ux = ux * dx; vx = vx * dx; wx = wx * dx; mux = mux * dx; divx3l = divx3l * dx;
        uy = uy * dy; vy = vy * dy; wy = wy * dy; muy = muy * dy; divy3l = divy3l * dy;
        uz = uz * dz; vz = vz * dz; wz = wz * dz; muz = muz * dz; divz3l = divz3l * dz;
        double sig11 = ux - 2.0 * div3l, sig12 = vx, sig13 = wx;
        double sig21 = uy, sig22 = vy - 2.0 * div3l, sig23 = wy;
        double sig31 = uz, sig32 = vz, sig33 = wz - 2.0 * div3l;
        double sigx = mux * sig11 + muy * sig12 + muz * sig13 + mu * divx3l;
        double sigy = mux * sig21 + muy * sig22 + muz * sig23 + mu * divy3l;
        double sigz = mux * sig31 + muy * sig32 + muz * sig33 + mu * divz3l;
        double sigah = (sig11 * ux + sig12 * uy + sig13 * uz + sig21 * vx + sig22 * vy + sig23 * vz +
                        sig31 * wx + sig32 * wy + sig33 * wz) * mu;
        double sigq = sigx * uu + sigy * vv + sigz * ww + sigah;
        WF(fl, q, I_U) = WF(fl, q, I_U) - sigx;
        WF(fl, q, I_V) = WF(fl, q, I_V) - sigy;
        WF(fl, q, I_W) = WF(fl, q, I_W) - sigz;
        WF(fl, q, I_E) = WF(fl, q, I_E) - sigq;
      }
}

/* visflx (multideal_gpu.F90:300-359) modes 1 and 2 */
void ox_visflx(ox_ctx *c, const double *wa, double *fl, double *fhat, int mode) {
  if (mode == 1) {
    if (c->g.nx > 1) visflx_dir(c, 0, wa, fl, fhat);
    if (c->g.ny > 1) visflx_dir(c, 1, wa, fl, fhat);
    if (c->g.nz > 1) visflx_dir(c, 2, wa, fl, fhat);
  } else if (mode == 2) {
    visflx_reduced(c, wa, fl);
  }
}

/* ---------------------------------------------------------------- RK bookkeeping */
/* bc_nr (multideal_gpu.F90:1116-1163) with bc_nr_lat_{x,y,z}_kernel
 * (kernels_gpu.F90:4330-4793): the characteristic boundary treatment of the
 * boundary cells of every face with bctags_nr > 0.  The one-sided derivative of
 * the conservative variables, projected on the left eigenvectors of the cell's
 * state, has its wave amplitudes modified (1: incoming acoustic waves killed;
 * 2 / 3: incoming waves from the difference to the outer ghost / to winf; 6: a
 * reflecting wall, entropy and shear waves zero and the incoming acoustic wave
 * equal to the outgoing one), and the projection back adds to fl. */
void ox_bc_nr(ox_ctx *c, const double *wa, const double *w, double *fl) {
  int nv = c->nv;
  double *el = (double *)malloc(sizeof(double) * nv * nv), *er = (double *)malloc(sizeof(double) * nv * nv);
  const double c_one[3] = {-1.5, 2.0, -0.5};
  for (int ilat = 1; ilat <= 6; ilat++) {
    int nr_type = c->p.bctags_nr[ilat - 1];
    if (nr_type <= 0) continue;
    int dir = (ilat - 1) / 2, se = (ilat - 1) % 2 + 1;
    int n = dir == 0 ? c->g.nx : (dir == 1 ? c->g.ny : c->g.nz);
    int na = dir == 0 ? c->g.ny : c->g.nx, nb = dir == 2 ? c->g.ny : c->g.nz;
    int ib = se == 1 ? 1 : n, sgn = se == 1 ? 1 : -1;
    const double *met = dir == 0 ? c->g.dcsidx : (dir == 1 ? c->g.detady : c->g.dzitdz);
    for (int b = 1; b <= nb; b++)
      for (int a = 1; a <= na; a++) {
        double dw[MAXNS + 4], dwo[MAXNS + 4], dwc[MAXNS + 4], dwco[MAXNS + 4], ev[MAXNS + 4];
        size_t p = face_pt(c, ilat, a, b, ib);
        for (int m = 1; m <= nv; m++) {
          dw[m - 1] = 0.0;
          for (int l = 1; l <= 3; l++) dw[m - 1] = dw[m - 1] + sgn * c_one[l - 1] * WG(w, face_pt(c, ilat, a, b, ib + sgn * (l - 1)), m);
          double w_target = 0.0;
          if (nr_type == 2) w_target = WG(w, face_pt(c, ilat, a, b, ib - sgn), m);
          else if (nr_type == 3) w_target = c->p.winf ? c->p.winf[m - 1] : 0.0;
          dwo[m - 1] = sgn * (WG(w, p, m) - w_target);
        }
        roe_t R;
        for (int lsp = 1; lsp <= NS; lsp++) R.yy[lsp - 1] = WG(wa, p, lsp);
        double rho = WG(wa, p, J_R), uu = WG(wa, p, J_U), vv = WG(wa, p, J_V), ww = WG(wa, p, J_W);
        double h = WG(wa, p, J_H), tt = WG(wa, p, J_T), pp = WG(wa, p, J_P), cs = WG(wa, p, J_C);
        double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
        double cc = cs * cs, rmix_tt = pp / rho, gamloc = cc / rmix_tt, gm1loc = gamloc - 1.0;
        double p_e = rho * gm1loc, etot = h - rmix_tt;
        R.b3 = etot;
        R.b2 = p_e / (rho * cc);
        R.b1 = -R.b2 * (etot - 2.0 * qq);
        for (int lsp = 1; lsp <= NS; lsp++) {
          double eei = species_poly_int(c, c->cv, tt, lsp);
          R.prhoi[lsp - 1] = c->rgas[lsp - 1] * tt + gm1loc * (etot - qq - eei);
        }
        R.rho = rho; R.uu = uu; R.vv = vv; R.ww = ww; R.c = cs; R.ci = 1.0 / cs; R.h = h;
        eigenvectors(c, dir, &R, el, er);
        for (int m = 1; m <= nv; m++) {
          dwc[m - 1] = 0.0;
          dwco[m - 1] = 0.0;
          for (int mm = 1; mm <= nv; mm++) {
            dwc[m - 1] = dwc[m - 1] + el[(size_t)(m - 1) * nv + mm - 1] * dw[mm - 1];
            dwco[m - 1] = dwco[m - 1] + el[(size_t)(m - 1) * nv + mm - 1] * dwo[mm - 1];
          }
        }
        double un = dir == 0 ? uu : (dir == 1 ? vv : ww);
        ev[0] = un - cs;
        for (int lsp = 2; lsp <= NS + 3; lsp++) ev[lsp - 1] = un;
        ev[NS + 3] = un + cs;
        if (nr_type == 1)
          for (int l = 1; l <= nv; l++) ev[l - 1] = sgn * dmin(sgn * ev[l - 1], 0.0);
        if (nr_type == 2 || nr_type == 3)
          for (int m = 1; m <= nv; m++)
            if (sgn * ev[m - 1] > 0.0) dwc[m - 1] = dwco[m - 1];
        for (int m = 1; m <= nv; m++) dwc[m - 1] = ev[m - 1] * dwc[m - 1];
        if (nr_type == 6) {
          for (int lsp = 2; lsp <= NS + 3; lsp++) dwc[lsp - 1] = 0.0;
          if (se == 1) dwc[NS + 3] = dwc[0];
          else dwc[0] = dwc[NS + 3];
        }
        int ii = dir == 0 ? ib : a, jj = dir == 1 ? ib : (dir == 0 ? a : b), kk = dir == 2 ? ib : b;
        size_t q = fi(c, ii, jj, kk);
        for (int m = 1; m <= nv; m++) {
          double df = 0.0;
          for (int mm = 1; mm <= nv; mm++) df = df + er[(size_t)(m - 1) * nv + mm - 1] * dwc[mm - 1];
          fl[q + (size_t)(m - 1) * c->npi] = fl[q + (size_t)(m - 1) * c->npi] + df * met[ib - 1];
        }
      }
  }
  free(el);
  free(er);
}

void ox_init_flux(ox_ctx *c, double *fl, double *fln, double rhodt) {
  size_t n = c->npi * c->nv;
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < n; q++) { fln[q] = -rhodt * fl[q]; fl[q] = 0.0; }
}
void ox_init_flux_simpler(ox_ctx *c, double *fl, double *fln, const double *fl_sav, double rhodt) {
  size_t n = c->npi * c->nv;
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < n; q++) { fln[q] = -rhodt * (fl[q] - fl_sav[q]); fl[q] = 0.0; }
}
void ox_sav_flx(ox_ctx *c, const double *fl, double *fl_sav) {
  memcpy(fl_sav, fl, sizeof(double) * c->npi * c->nv);
}
void ox_update_flux(ox_ctx *c, const double *fl, double *fln, double gamdt) {
  size_t n = c->npi * c->nv;
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < n; q++) fln[q] = fln[q] - gamdt * fl[q];
}
void ox_update_simpler_flux(ox_ctx *c, const double *fl, double *fln, const double *fl_sav, double gamdt) {
  size_t n = c->npi * c->nv;
#pragma omp parallel for schedule(static)
  for (size_t q = 0; q < n; q++) fln[q] = fln[q] - gamdt * (fl[q] - fl_sav[q]);
}
void ox_update_field(ox_ctx *c, double *w, const double *fln, const int32_t *mask) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        size_t p = gi(c, i, j, k), q = fi(c, i, j, k);
        if (mask == NULL || mask[p] == 0)
          for (int m = 1; m <= c->nv; m++) WG(w, p, m) = WG(w, p, m) + WF(fln, q, m);
      }
}

/* compute_dt_cuf (kernels_gpu.F90:6075-6152) */
void ox_compute_dt(ox_ctx *c, const double *wa, const int32_t *mask, double out9[9]) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz;
  double mx[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        size_t p = gi(c, i, j, k);
        if (mask != NULL && mask[p] != 0) continue;
        double Y[MAXNS];
        for (int lsp = 1; lsp <= NS; lsp++) Y[lsp - 1] = WG(wa, p, lsp);
        double rho = WG(wa, p, J_R), ri = 1.0 / rho;
        double uu = WG(wa, p, J_U), vv = WG(wa, p, J_V), ww = WG(wa, p, J_W), tt = WG(wa, p, J_T);
        double mu = WG(wa, p, J_MU), cc = WG(wa, p, J_C), k_cond = WG(wa, p, J_K_COND);
        double cploc = mix_cp(c, tt, Y);
        double nu = ri * mu;
        double kr = k_cond * ri / cploc;
        double v[9] = {(fabs(uu) + cc) * c->g.dcsidx[i - 1], (fabs(vv) + cc) * c->g.detady[j - 1],
                       (fabs(ww) + cc) * c->g.dzitdz[k - 1], nu * c->g.dcsidxs[i - 1], nu * c->g.detadys[j - 1],
                       nu * c->g.dzitdzs[k - 1], kr * c->g.dcsidxs[i - 1], kr * c->g.detadys[j - 1],
                       kr * c->g.dzitdzs[k - 1]};
        for (int q = 0; q < 9; q++) mx[q] = dmax(mx[q], v[q]);
      }
  for (int q = 0; q < 9; q++) out9[q] = mx[q];
}

/* compute_residual_cuf + compute_rho_t_p_minmax_cuf (kernels_gpu.F90:5991-6011,
 * 6038-6073) and the residual's normalisation (multideal_gpu.F90:1603-1606):
 * out7 = {residual_rhou, rhomin, rhomax, tmin, tmax, pmin, pmax}. */
void ox_compute_residual(ox_ctx *c, const double *fln, const double *wa, const int32_t *mask, double dt,
                         double out7[7]) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz;
  double res = 0.0;
  double mn[3] = {HUGE_VAL, HUGE_VAL, HUGE_VAL}, mx[3] = {-100.0, -100.0, -100.0};
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        size_t p = gi(c, i, j, k);
        if (mask != NULL && mask[p] != 0) continue;
        size_t q = (size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)ny * (size_t)(k - 1));
        double f = fln[q + (size_t)(I_U - 1) * (size_t)nx * ny * nz] / dt;
        res = res + f * f;
        double v[3] = {WG(wa, p, J_R), WG(wa, p, J_T), WG(wa, p, J_P)};
        for (int l = 0; l < 3; l++) { mn[l] = fmin(mn[l], v[l]); mx[l] = dmax(mx[l], v[l]); }
      }
  out7[0] = sqrt(res / ((double)nx * (double)ny * (double)nz));
  for (int l = 0; l < 3; l++) { out7[1 + 2 * l] = mn[l]; out7[2 + 2 * l] = mx[l]; }
}

/* ---------------------------------------------------------------- chemistry */
/* Production rates of rosenbrock_rhs / rosenbrock_krylov_rhs / compute_chemistry_cuf
 * (kernels_gpu.F90:9251-9357, :10854-10955, :9557-9650): rhs_k = W_k sum_r nu_kr q_r
 * for the concentrations conc and temperature tt.  qlr returns q_r. */
static void reaction_rates(const ox_ctx *c, double tt, const double *conc, double *qlr_out) {
  int nr = c->t.nr;
  double Rtti = 1.0 / (c->t.R_univ * tt);
  int itt = (int)((tt - c->t.t_min_tab) / c->t.dt_tab) + 1;
  if (itt < 1) itt = 1;
  if (itt > c->t.num_t_tab) itt = c->t.num_t_tab;
  double ttleft = (itt - 1) * c->t.dt_tab + c->t.t_min_tab;
  double dtt = (tt - ttleft) / c->t.dt_tab;
  for (int lr = 1; lr <= nr; lr++) {
    double kf = 0.0, k0, kinf, tb, rpres;
    int ty = c->t.reac_ty[lr - 1];
    const double *A = c->t.arr_a, *B = c->t.arr_b, *E = c->t.arr_ea, *F = c->t.falloff;
    switch (ty) {
      case 0: case 1:
        kf = RX(A, lr, 1);
        if (RX(B, lr, 1) != 0.0) kf = kf * pow(tt, RX(B, lr, 1));
        if (RX(E, lr, 1) != 0.0) kf = kf * exp(-RX(E, lr, 1) * Rtti);
        break;
      case 2:
        k0 = RX(A, lr, 1) * pow(tt, RX(B, lr, 1)) * exp(-RX(E, lr, 1) * Rtti);
        kinf = RX(A, lr, 2) * pow(tt, RX(B, lr, 2)) * exp(-RX(E, lr, 2) * Rtti);
        tb = 0.0;
        for (int lsp = 1; lsp <= NS; lsp++) tb = tb + RX(c->t.tb_eff, lr, lsp) * conc[lsp - 1];
        rpres = k0 * tb / kinf;
        kf = kinf * (rpres / (1.0 + rpres));
        break;
      case 3:
        k0 = RX(A, lr, 1) * pow(tt, RX(B, lr, 1)) * exp(-RX(E, lr, 1) * Rtti);
        kinf = RX(A, lr, 2) * pow(tt, RX(B, lr, 2)) * exp(-RX(E, lr, 2) * Rtti);
        tb = 0.0;
        for (int lsp = 1; lsp <= NS; lsp++) tb = tb + RX(c->t.tb_eff, lr, lsp) * conc[lsp - 1];
        rpres = k0 * tb / kinf;
        if (rpres < 1e-30) {
          kf = k0 * tb;
        } else {
          double fcent = (1.0 - RX(F, lr, 1)) * exp(-tt / RX(F, lr, 2)) + RX(F, lr, 1) * exp(-tt / RX(F, lr, 3));
          if (RX(F, lr, 4) != -3.14) fcent = fcent + exp(-RX(F, lr, 4) / tt);
          fcent = log10(fcent);
          double coff = -0.4 - 0.67 * fcent;
          double noff = 0.75 - 1.27 * fcent;
          double doff = 0.14;
          double lp = log10(rpres);
          double foff = pow(10.0, pow(1.0 + pow((lp + coff) / (noff - doff * (lp + coff)), 2.0), -1.0) * fcent);
          kf = kinf * (rpres / (1.0 + rpres)) * foff;
        }
        break;
      case 4: {
        k0 = RX(A, lr, 1) * pow(tt, RX(B, lr, 1)) * exp(-RX(E, lr, 1) * Rtti);
        kinf = RX(A, lr, 2) * pow(tt, RX(B, lr, 2)) * exp(-RX(E, lr, 2) * Rtti);
        tb = 0.0;
        for (int lsp = 1; lsp <= NS; lsp++) tb = tb + RX(c->t.tb_eff, lr, lsp) * conc[lsp - 1];
        rpres = k0 * tb / kinf;
        double xoff = 1.0 / (1.0 + pow(log10(rpres), 2.0));
        double foff = RX(F, lr, 4) * pow(RX(F, lr, 1) * exp(-RX(F, lr, 2) / tt) + exp(-tt / RX(F, lr, 3)), xoff) *
                      pow(tt, RX(F, lr, 5));
        kf = kinf * (rpres / (1.0 + rpres)) * foff;
        break;
      }
      default: kf = 0.0;
    }
    double kb;
    if (c->t.is_rev[lr - 1] == 1) {
      double dkc = KC(itt + 1, lr) - KC(itt, lr);
      double kc = KC(itt, lr) + dkc * dtt;
      kb = kf / kc;
    } else {
      kb = 0.0;
    }
    double q1 = 1.0, q2 = 1.0;
    for (int lsp = 1; lsp <= NS; lsp++) {
      double rr = RX(c->t.r_coeffs, lr, lsp), pp = RX(c->t.p_coeffs, lr, lsp);
      if (rr == 1.0) q1 = q1 * conc[lsp - 1];
      else if (rr != 0.0) q1 = q1 * pow(conc[lsp - 1], rr);
      if (pp == 1.0) q2 = q2 * conc[lsp - 1];
      else if (pp != 0.0) q2 = q2 * pow(conc[lsp - 1], pp);
    }
    tb = 1.0;
    if (ty == 1) {
      tb = 0.0;
      for (int lsp = 1; lsp <= NS; lsp++) tb = tb + RX(c->t.tb_eff, lr, lsp) * conc[lsp - 1];
    }
    qlr_out[lr - 1] = tb * (kf * q1 - kb * q2);
  }
}

static void species_rhs(const ox_ctx *c, const double *qlr, double *rhs) {
  for (int lr = 1; lr <= c->t.nr; lr++) {
    for (int lsp = 1; lsp <= NS; lsp++) {
      double rr = RX(c->t.r_coeffs, lr, lsp), pp = RX(c->t.p_coeffs, lr, lsp);
      if (rr != 0.0 || pp != 0.0) {
        double wdtkj = (pp - rr) * qlr[lr - 1];
        rhs[lsp - 1] = rhs[lsp - 1] + wdtkj * c->mw[lsp - 1];
      }
    }
  }
}

/* rosenbrock_krylov_rhs (kernels_gpu.F90:10794-10976), PaSR off */
static void krylov_rhs(ox_ctx *c, const double *w_sav, double T_iter, double *rhs) {
  double wl[MAXNS], Y[MAXNS], conc[MAXNS], qlr[512];
  for (int n = 1; n <= NS; n++) wl[n - 1] = dmax(w_sav[n - 1], 0.0);
  double rho = wl[0];
  for (int lsp = 2; lsp <= NS; lsp++) rho = rho + wl[lsp - 1];
  double ri = 1.0 / rho;
  for (int lsp = 1; lsp <= NS; lsp++) {
    Y[lsp - 1] = wl[lsp - 1] * ri;
    conc[lsp - 1] = rho * Y[lsp - 1] / c->mw[lsp - 1];
  }
  double uu = w_sav[I_U - 1] * ri, vv = w_sav[I_V - 1] * ri, ww = w_sav[I_W - 1] * ri;
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double ee = (w_sav[I_E - 1] * ri) - qq;
  double tt = ox_temperature_from_e(c, ee, T_iter, Y);
  for (int m = 0; m < c->nv; m++) rhs[m] = 0.0;
  reaction_rates(c, tt, conc, qlr);
  species_rhs(c, qlr, rhs);
}

static double norm2(const double *v, int n) {
  double s = 0.0;
  for (int q = 0; q < n; q++) s = s + v[q] * v[q];
  return sqrt(s);
}

/* ludcmp_krylov / lubksb_krylov / inv_matrix_krylov (kernels_gpu.F90:11061-11205) on
 * the leading d x d block of a column-major MMAX x MMAX matrix */
#define AK(r, s) a[((s) - 1) * MMAX + (r) - 1]
static void ludcmp_k(double *a, int *indx, int d) {
  const double tiny = 1.5e-16;
  double vv[MMAX];
  for (int i = 1; i <= d; i++) {
    double amax = 0.0;
    for (int j = 1; j <= d; j++) if (fabs(AK(i, j)) > amax) amax = fabs(AK(i, j));
    if (amax < tiny) return;
    vv[i - 1] = 1.0 / amax;
  }
  for (int j = 1; j <= d; j++) {
    for (int i = 1; i <= j - 1; i++) {
      double summ = AK(i, j);
      for (int k = 1; k <= i - 1; k++) summ = summ - AK(i, k) * AK(k, j);
      AK(i, j) = summ;
    }
    double amax = 0.0;
    int imax = j;
    for (int i = j; i <= d; i++) {
      double summ = AK(i, j);
      for (int k = 1; k <= j - 1; k++) summ = summ - AK(i, k) * AK(k, j);
      AK(i, j) = summ;
      double dum = vv[i - 1] * fabs(summ);
      if (dum >= amax) { imax = i; amax = dum; }
    }
    if (j != imax) {
      for (int k = 1; k <= d; k++) { double dum = AK(imax, k); AK(imax, k) = AK(j, k); AK(j, k) = dum; }
      vv[imax - 1] = vv[j - 1];
    }
    indx[j - 1] = imax;
    if (fabs(AK(j, j)) < tiny) AK(j, j) = tiny;
    if (j != d) {
      double dum = 1.0 / AK(j, j);
      for (int i = j + 1; i <= d; i++) AK(i, j) = AK(i, j) * dum;
    }
  }
}
static void lubksb_k(const double *a, const int *indx, double *b, int d) {
  int ii = 0;
  for (int i = 1; i <= d; i++) {
    int ll = indx[i - 1];
    double summ = b[ll - 1];
    b[ll - 1] = b[i - 1];
    if (ii != 0) { for (int j = ii; j <= i - 1; j++) summ = summ - AK(i, j) * b[j - 1]; }
    else if (summ != 0.0) ii = i;
    b[i - 1] = summ;
  }
  for (int i = d; i >= 1; i--) {
    double summ = b[i - 1];
    if (i < d) for (int j = i + 1; j <= d; j++) summ = summ - AK(i, j) * b[j - 1];
    b[i - 1] = summ / AK(i, i);
  }
}
static void inv_matrix_k(double *a, int d) {
  if (d == 1) { AK(1, 1) = 1.0 / AK(1, 1); return; }
  int indx[MMAX];
  for (int q = 0; q < MMAX; q++) indx[q] = q + 1;   /* defined pivots if ludcmp returns early */
  double y[MMAX * MMAX];
  for (int r = 1; r <= d; r++) for (int s = 1; s <= d; s++) y[(s - 1) * MMAX + r - 1] = 0.0;
  for (int r = 1; r <= d; r++) y[(r - 1) * MMAX + r - 1] = 1.0;
  ludcmp_k(a, indx, d);
  for (int s = 1; s <= d; s++) lubksb_k(a, indx, y + (s - 1) * MMAX, d);
  for (int r = 1; r <= d; r++) for (int s = 1; s <= d; s++) AK(r, s) = y[(s - 1) * MMAX + r - 1];
}
#undef AK

/* The system a ROK4 integration advances: nv components, the right-hand side,
 * and what happens after an accepted step (the temperature guess is updated;
 * the 0-D reactor may also move the end time at ignition). */
typedef struct ox_sys ox_sys;
struct ox_sys {
  ox_ctx *c;
  int nv;
  void (*rhs)(ox_sys *s, const double *y, double T_iter, double *out);
  void (*accept)(ox_sys *s, const double *y, double time, double *T_iter, double *time_end);
  /* constant-pressure reactor */
  double p, h, T0, t_max, ign_factor, end_factor, t_ign;
  int max_steps, nsteps;
  double time_reached, T_final;
};

/* arnoldi (kernels_gpu.F90:10664-10792) */
static void arnoldi(ox_sys *S, const double *w_sav, double dt, double *Vb, double *inv, double T_iter,
                    double *rhs_sav, const double *fl_sav_cell, int simpler) {
  const double gam = 0.572816062482135, TOL = 1e-6;
  int nv = S->nv;
  double HH[(MMAX + 1) * MMAX], V[MAXNV * (MMAX + 1)], Vt[MMAX * MAXNV], HH_inv[MMAX * MMAX];
  double rhs_sav_pr[MMAX], lambda[MMAX], jac[MAXNV], wl[MAXNV], rhsp[MAXNV];
  memset(HH, 0, sizeof(HH)); memset(V, 0, sizeof(V)); memset(Vt, 0, sizeof(Vt));
  memset(lambda, 0, sizeof(lambda)); memset(HH_inv, 0, sizeof(HH_inv));
  for (int q = 0; q < nv * MMAX; q++) Vb[q] = 0.0;
#define HHm(r, s) HH[((s) - 1) * (MMAX + 1) + (r) - 1]
#define Vm(r, s) V[((s) - 1) * nv + (r) - 1]
#define VTm(r, s) Vt[((s) - 1) * MMAX + (r) - 1]
#define HI(r, s) HH_inv[((s) - 1) * MMAX + (r) - 1]
  S->rhs(S, w_sav, T_iter, rhs_sav);
  if (simpler == 1) for (int m = 0; m < nv; m++) rhs_sav[m] = rhs_sav[m] - fl_sav_cell[m];
  double nrm = norm2(rhs_sav, nv);
  for (int m = 1; m <= nv; m++) Vm(m, 1) = rhs_sav[m - 1] / nrm;
  const double eps = 1.0e-08;
  for (int kk = 1; kk <= MMAX; kk++) {
    /* rosenbrock_krylov_jacobian (:10613-10662) */
    for (int m = 1; m <= nv; m++) wl[m - 1] = w_sav[m - 1] + (eps * Vm(m, kk));
    S->rhs(S, wl, T_iter, rhsp);
    if (simpler == 1) for (int m = 0; m < nv; m++) rhsp[m] = rhsp[m] - fl_sav_cell[m];
    for (int m = 0; m < nv; m++) jac[m] = (rhsp[m] - rhs_sav[m]) / eps;
    for (int jj = 1; jj <= kk; jj++) {
      double dot = 0.0;
      for (int m = 1; m <= nv; m++) dot = dot + Vm(m, jj) * jac[m - 1];
      HHm(jj, kk) = dot;
      for (int m = 1; m <= nv; m++) jac[m - 1] = jac[m - 1] - (HHm(jj, kk) * Vm(m, jj));
    }
    HHm(kk + 1, kk) = norm2(jac, nv);
    for (int m = 1; m <= nv; m++) Vm(m, kk + 1) = jac[m - 1] / HHm(kk + 1, kk);
    int lim_min = kk < MMAX ? kk : MMAX;
    for (int ll = 1; ll <= lim_min; ll++) for (int jj = 1; jj <= nv; jj++) VTm(ll, jj) = Vm(jj, ll);
    for (int ll = 1; ll <= MMAX; ll++) {
      rhs_sav_pr[ll - 1] = 0.0;
      for (int jj = 1; jj <= nv; jj++) rhs_sav_pr[ll - 1] = rhs_sav_pr[ll - 1] + VTm(ll, jj) * rhs_sav[jj - 1];
    }
    for (int n = 1; n <= lim_min; n++)
      for (int nn = 1; nn <= lim_min; nn++) {
        HI(n, nn) = -(dt * gam * HHm(n, nn));
        if (n == nn) HI(n, nn) = HI(n, nn) + 1.0;
      }
    if (kk < MMAX) for (int n = kk + 1; n <= MMAX; n++) HI(n, n) = 1.0;
    inv_matrix_k(HH_inv, kk);
    for (int ll = 1; ll <= MMAX; ll++) {
      lambda[ll - 1] = 0.0;
      for (int jj = 1; jj <= MMAX; jj++) lambda[ll - 1] = lambda[ll - 1] + HI(ll, jj) * rhs_sav_pr[jj - 1];
    }
    if (fabs(dt * gam * HHm(kk + 1, kk)) * fabs(lambda[kk - 1]) < TOL) {
      for (int s = 1; s <= kk; s++) for (int r = 1; r <= nv; r++) Vb[(s - 1) * nv + r - 1] = Vm(r, s);
      for (int q = 0; q < MMAX * MMAX; q++) inv[q] = HH_inv[q];
      break;
    }
  }
#undef HHm
#undef Vm
#undef VTm
#undef HI
}

/* The flow cell of the reacting step: state (rho Y_k, rho u, rho v, rho w, rho E) at
 * constant volume; after an accepted step T follows from e (:10597-10606). */
static void flow_rhs(ox_sys *S, const double *y, double T_iter, double *out) { krylov_rhs(S->c, y, T_iter, out); }
static void flow_accept(ox_sys *S, const double *VEC, double time, double *T_iter, double *time_end) {
  (void)time; (void)time_end;
  ox_ctx *c = S->c;
  double rho = VEC[0];
  for (int n = 2; n <= NS; n++) rho = rho + VEC[n - 1];
  double ri = 1.0 / rho, Y[MAXNS];
  for (int n = 1; n <= NS; n++) Y[n - 1] = VEC[n - 1] * ri;
  double uu = VEC[NS] * ri, vv = VEC[NS + 1] * ri, ww = VEC[NS + 2] * ri;
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double ee = VEC[NS + 3] * ri - qq;
  *T_iter = ox_temperature_from_e(c, ee, *T_iter, Y);
}

static void rok4_core(ox_sys *S, double *VEC, double T_iter, const double *fl_sav_cell, double dttry,
                      double time_start, double time_end, int simpler);

/* rosenbrock_krylov_kernel per cell (kernels_gpu.F90:10360-10611), PaSR off.
 * The Z gate (:10464-10465) is applied by the caller. */
void ox_krylov_cell(ox_ctx *c, double *VEC, double T_iter, double Z, const double *fl_sav_cell,
                    double dttry, double time_start, double time_end, int simpler) {
  const double eps_Z = 5e-4;
  if (!(Z > eps_Z && Z < 1.0 - eps_Z)) return;
  ox_sys S;
  memset(&S, 0, sizeof(S));
  S.c = c; S.nv = c->nv; S.rhs = flow_rhs; S.accept = flow_accept; S.max_steps = c->p.ros_maxsteps;
  rok4_core(&S, VEC, T_iter, fl_sav_cell, dttry, time_start, time_end, simpler);
}

/* The ROK4 integration of one state (the body of rosenbrock_krylov_kernel,
 * kernels_gpu.F90:10463-10610) for the system S. */
static void rok4_core(ox_sys *S, double *VEC, double T_iter, const double *fl_sav_cell, double dttry,
                      double time_start, double time_end, int simpler) {
  ox_ctx *c = S->c;
  int nv = S->nv;
  const double gam = 0.572816062482135;
  double alpha[5][4] = {{0}}, gamma_c[5][4] = {{0}}, bs[5], bt[5];
  alpha[2][1] = 0.432364435748567;
  alpha[3][1] = -0.514211316876170; alpha[3][2] = 1.382271144617360;
  alpha[4][1] = -0.514211316876170; alpha[4][2] = 1.382271144617360; alpha[4][3] = 0.0;
  bs[1] = 0.194335256262729; bs[2] = 0.483167813989227; bs[3] = 0.0; bs[4] = 0.322496929748044;
  gamma_c[2][1] = -0.602765307997356;
  gamma_c[3][1] = -1.389195789724843; gamma_c[3][2] = 1.072950969011413;
  gamma_c[4][1] = 0.992356412977094; gamma_c[4][2] = -1.390032613873701; gamma_c[4][3] = -0.440875890223325;
  bt[1] = -0.217819895945721; bt[2] = 1.03130847478467; bt[3] = 0.186511421161047; bt[4] = 0.0;
  double Vb[MAXNV * MMAX], inv[MMAX * MMAX], IDIFF[MMAX * MMAX], A[MAXNV * MMAX], B[MAXNV * MAXNV];
  double rhs_sav[MAXNV], ys[MAXNV], yt[MAXNV], F[MAXNV], GK[MAXNV], Cv[MAXNV], Ks[MAXNV * NSTAGE], errv[MAXNV];
  memset(inv, 0, sizeof(inv));
  double time = time_start, dt = dttry, errn = 1.0;
  int it = 0;
  while (time < (time_end - 1.0e-12)) {
    dt = dmin(dt, time_end - time);
    it = it + 1;
    arnoldi(S, VEC, dt, Vb, inv, T_iter, rhs_sav, fl_sav_cell, simpler);
    for (int r = 1; r <= MMAX; r++)
      for (int s = 1; s <= MMAX; s++)
        IDIFF[(s - 1) * MMAX + r - 1] = (r == s ? 1.0 : 0.0) - inv[(s - 1) * MMAX + r - 1];
    for (int kk = 1; kk <= MMAX; kk++)
      for (int ll = 1; ll <= nv; ll++) {
        double a = Vb[ll - 1] * IDIFF[(kk - 1) * MMAX + 0];
        for (int jj = 2; jj <= MMAX; jj++) a = a + Vb[(jj - 1) * nv + ll - 1] * IDIFF[(kk - 1) * MMAX + jj - 1];
        A[(kk - 1) * nv + ll - 1] = a;
      }
    for (int kk = 1; kk <= nv; kk++)
      for (int ll = 1; ll <= nv; ll++) {
        double b = A[ll - 1] * Vb[kk - 1];   /* E(1,kk) = Vb(kk,1) */
        for (int jj = 2; jj <= MMAX; jj++) b = b + A[(jj - 1) * nv + ll - 1] * Vb[(jj - 1) * nv + kk - 1];
        B[(kk - 1) * nv + ll - 1] = b;
      }
    for (int ii = 1; ii <= NSTAGE; ii++) {
      for (int m = 0; m < nv; m++) ys[m] = VEC[m];
      for (int jj = 1; jj <= ii - 1; jj++)
        for (int m = 0; m < nv; m++) ys[m] = ys[m] + dt * alpha[ii][jj] * Ks[(jj - 1) * nv + m];
      S->rhs(S, ys, T_iter, F);
      for (int m = 0; m < nv; m++) GK[m] = 0.0;
      for (int jj = 1; jj <= ii - 1; jj++)
        for (int m = 0; m < nv; m++) GK[m] = GK[m] + gamma_c[ii][jj] / gam * Ks[(jj - 1) * nv + m];
      for (int m = 0; m < nv; m++) F[m] = F[m] + GK[m];
      if (simpler == 1) for (int m = 0; m < nv; m++) F[m] = F[m] - fl_sav_cell[m];
      for (int ll = 1; ll <= nv; ll++) {
        double s = B[ll - 1] * F[0];
        for (int jj = 2; jj <= nv; jj++) s = s + B[(jj - 1) * nv + ll - 1] * F[jj - 1];
        Cv[ll - 1] = s;
      }
      for (int m = 0; m < nv; m++) Ks[(ii - 1) * nv + m] = F[m] - Cv[m] - GK[m];
    }
    for (int ll = 1; ll <= nv; ll++) {
      ys[ll - 1] = VEC[ll - 1];
      yt[ll - 1] = VEC[ll - 1];
      for (int ii = 1; ii <= NSTAGE; ii++) {
        ys[ll - 1] = ys[ll - 1] + dt * bs[ii] * Ks[(ii - 1) * nv + ll - 1];
        yt[ll - 1] = yt[ll - 1] + dt * bt[ii] * Ks[(ii - 1) * nv + ll - 1];
      }
      errv[ll - 1] = (yt[ll - 1] - ys[ll - 1]) / ((1.0e-4) * ys[ll - 1] + 1.0e-8);
    }
    double errmax = norm2(errv, nv);
    double fac = 0.625 * pow(errn, 0.1) / pow(errmax, 0.175);
    double dtnext = dt * dmin(5.0, dmax(0.2, fac));
    if (errmax < 1.0) {
      time = time + dt;
      for (int m = 0; m < nv; m++) VEC[m] = ys[m];
      S->accept(S, VEC, time, &T_iter, &time_end);
      dt = dtnext;
      errn = errmax;
    } else {
      dt = dtnext;
      errn = errmax;
    }
    if (it > S->max_steps) { c->status |= STX_ST_ROS_STEPS_CAP; break; }
  }
  S->nsteps = it;
  S->time_reached = time;
  S->T_final = T_iter;
}

void ox_rosenbrock_krylov(ox_ctx *c, double *w, const double *wa, const double *fl_sav, double dttry,
                          double time_start, double time_end, int simpler) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz, nv = c->nv;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        size_t p = gi(c, i, j, k), q = fi(c, i, j, k);
        double VEC[MAXNV], fs[MAXNV];
        for (int m = 1; m <= nv; m++) {
          VEC[m - 1] = WG(w, p, m);
          fs[m - 1] = (simpler == 1 && fl_sav) ? WF(fl_sav, q, m) : 0.0;
        }
        double Z = WG(wa, p, J_Z);
        if (Z > 5e-4 && Z < 1.0 - 5e-4) {
          ox_krylov_cell(c, VEC, WG(wa, p, J_T), Z, fs, dttry, time_start, time_end, simpler);
          for (int m = 1; m <= nv; m++) WG(w, p, m) = VEC[m - 1];
        }
      }
}

/* ---- 0-D adiabatic constant-pressure reactors.  The reference's batch reactor
 * (examples/batch_reactor) is constant-volume; the constant-pressure form has no
 * counterpart there.  State Y_k (clipped at 0 where evaluated); h = sum Y_k h_k(T0)
 * and p stay fixed; T follows from h by the Newton iteration of
 * get_mixture_temperature_from_h_roe_dev (kernels_gpu.F90:6810-6900); rho = p/(R T);
 * dY_k/dt = W_k omega_k / rho with the production rates of rosenbrock_krylov_rhs
 * (:10794-10976), integrated by the same ROK4 scheme.  After the first accepted
 * step with T > ign_factor T0 (the ignition time t_ign, as mech_comp.py's
 * T > 1.05 T0 test) the end time becomes min(t_max, end_factor t_ign). */
static void cp_rhs(ox_sys *S, const double *y, double T_iter, double *out) {
  ox_ctx *c = S->c;
  double Yc[MAXNS], conc[MAXNS], qlr[512];
  for (int k = 0; k < NS; k++) Yc[k] = dmax(y[k], 0.0);
  double tt = temperature_from_poly(c, c->cp, S->h, T_iter, Yc);
  double rm = 0.0;
  for (int k = 0; k < NS; k++) rm = rm + c->rgas[k] * Yc[k];
  double rho = S->p / (rm * tt);
  for (int k = 0; k < NS; k++) conc[k] = rho * Yc[k] / c->mw[k];
  for (int k = 0; k < NS; k++) out[k] = 0.0;
  reaction_rates(c, tt, conc, qlr);
  species_rhs(c, qlr, out);
  for (int k = 0; k < NS; k++) out[k] = out[k] / rho;
}

static void cp_accept(ox_sys *S, const double *y, double time, double *T_iter, double *time_end) {
  ox_ctx *c = S->c;
  double Yc[MAXNS];
  for (int k = 0; k < NS; k++) Yc[k] = dmax(y[k], 0.0);
  *T_iter = temperature_from_poly(c, c->cp, S->h, *T_iter, Yc);
  if (S->t_ign < 0.0 && *T_iter > S->ign_factor * S->T0) {
    S->t_ign = time;
    double te = S->end_factor * time;
    if (te < *time_end) *time_end = te;
  }
}

void ox_batch0d_cp(ox_ctx *c, int n, const double *T0, const double *p0, const double *Y0, double t_max,
                   double dttry, double ign_factor, double end_factor, int max_steps, double *Y, double *T,
                   double *t_ign, double *t_end, int32_t *nsteps) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int r = 0; r < n; r++) {
    ox_sys S;
    memset(&S, 0, sizeof(S));
    S.c = c; S.nv = NS; S.rhs = cp_rhs; S.accept = cp_accept; S.max_steps = max_steps;
    double VEC[MAXNS];
    for (int k = 0; k < NS; k++) VEC[k] = Y0[(size_t)k * n + r];
    double h = 0.0;
    for (int k = 0; k < NS; k++) h = h + VEC[k] * species_poly_int(c, c->cp, T0[r], k + 1);
    S.h = h; S.p = p0[r]; S.T0 = T0[r]; S.t_max = t_max;
    S.ign_factor = ign_factor; S.end_factor = end_factor; S.t_ign = -1.0;
    rok4_core(&S, VEC, T0[r], NULL, dttry, 0.0, t_max, 0);
    for (int k = 0; k < NS; k++) Y[(size_t)k * n + r] = VEC[k];
    T[r] = S.T_final;
    t_ign[r] = S.t_ign;
    t_end[r] = S.time_reached;
    nsteps[r] = S.nsteps;
  }
}

/* ---- full-Jacobian Rosenbrock (kernels_gpu.F90:8928-9501), one cell.  The cell
 * state (w, Y = w_aux(1:ns), T = w_aux(J_T)) is updated in place exactly as the
 * reference updates w_gpu / w_aux_gpu inside rosenbrock_rhs. */
static void ros_rhs(ox_ctx *c, double *wc, double *Y, double *T, double *rhs) {
  double conc[MAXNS], qlr[512];
  for (int lsp = 1; lsp <= NS; lsp++) wc[lsp - 1] = dmax(wc[lsp - 1], 0.0);
  double rho = wc[0];
  for (int lsp = 2; lsp <= NS; lsp++) rho = rho + wc[lsp - 1];
  double ri = 1.0 / rho;
  for (int lsp = 1; lsp <= NS; lsp++) {
    Y[lsp - 1] = wc[lsp - 1] * ri;
    conc[lsp - 1] = rho * Y[lsp - 1] / c->mw[lsp - 1];
  }
  double uu = wc[I_U - 1] * ri, vv = wc[I_V - 1] * ri, ww = wc[I_W - 1] * ri;
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double ee = wc[I_E - 1] * ri - qq;
  double tt = ox_temperature_from_e(c, ee, *T, Y);
  *T = tt;
  for (int m = 0; m < c->nv; m++) rhs[m] = 0.0;
  reaction_rates(c, tt, conc, qlr);
  species_rhs(c, qlr, rhs);
}

#define AM(r, s) a[((s) - 1) * nv + (r) - 1]
static void ludcmp_full(double *a, int *indx, int nv) {
  const double tiny = 1.5e-16;
  double vv[MAXNV];
  for (int i = 1; i <= nv; i++) {
    double amax = 0.0;
    for (int j = 1; j <= nv; j++) if (fabs(AM(i, j)) > amax) amax = fabs(AM(i, j));
    if (amax < tiny) return;
    vv[i - 1] = 1.0 / amax;
  }
  for (int j = 1; j <= nv; j++) {
    for (int i = 1; i <= j - 1; i++) {
      double summ = AM(i, j);
      for (int k = 1; k <= i - 1; k++) summ = summ - AM(i, k) * AM(k, j);
      AM(i, j) = summ;
    }
    double amax = 0.0;
    int imax = j;
    for (int i = j; i <= nv; i++) {
      double summ = AM(i, j);
      for (int k = 1; k <= j - 1; k++) summ = summ - AM(i, k) * AM(k, j);
      AM(i, j) = summ;
      double dum = vv[i - 1] * fabs(summ);
      if (dum >= amax) { imax = i; amax = dum; }
    }
    if (j != imax) {
      for (int k = 1; k <= nv; k++) { double dum = AM(imax, k); AM(imax, k) = AM(j, k); AM(j, k) = dum; }
      vv[imax - 1] = vv[j - 1];
    }
    indx[j - 1] = imax;
    if (fabs(AM(j, j)) < tiny) AM(j, j) = tiny;
    if (j != nv) {
      double dum = 1.0 / AM(j, j);
      for (int i = j + 1; i <= nv; i++) AM(i, j) = AM(i, j) * dum;
    }
  }
}
static void lubksb_full(const double *a, const int *indx, double *b, int nv) {
  int ii = 0;
  for (int i = 1; i <= nv; i++) {
    int ll = indx[i - 1];
    double summ = b[ll - 1];
    b[ll - 1] = b[i - 1];
    if (ii != 0) { for (int j = ii; j <= i - 1; j++) summ = summ - AM(i, j) * b[j - 1]; }
    else if (summ != 0.0) ii = i;
    b[i - 1] = summ;
  }
  for (int i = nv; i >= 1; i--) {
    double summ = b[i - 1];
    if (i < nv) for (int j = i + 1; j <= nv; j++) summ = summ - AM(i, j) * b[j - 1];
    b[i - 1] = summ / AM(i, i);
  }
}
#undef AM

void ox_rosenbrock_cell(ox_ctx *c, double *wc, double *Y, double *T, double dttry, double time_start, double time_end) {
  int nv = c->nv;
  const double safety = 0.9, grow = 1.5, pgrow = -0.25, shrnk = 0.5, pshrnk = -1.0 / 3.0, errcon = 0.1296;
  const double gam = 1.0 / 2.0, a21 = 2.0, a31 = 48.0 / 25.0, a32 = 6.0 / 25.0;
  const double c21 = -8.0, c31 = 372.0 / 25.0, c32 = 12.0 / 5.0;
  const double c41 = -112.0 / 125.0, c42 = -54.0 / 125.0, c43 = -2.0 / 5.0;
  const double b1 = 19.0 / 9.0, b2 = 1.0 / 2.0, b3 = 25.0 / 108.0, b4 = 125.0 / 108.0;
  const double e1 = 17.0 / 54.0, e2 = 7.0 / 36.0, e3 = 0.0, e4 = 125.0 / 108.0;
  const double a2x = 1.0, a3x = 3.0 / 5.0;
  double jac[MAXNV * MAXNV], amat[MAXNV * MAXNV], w_sav[MAXNV], rhs_sav[MAXNV], yscal[MAXNV], err[MAXNV];
  double rhs[MAXNV], rhsp[MAXNV], rhsm[MAXNV], g1[MAXNV], g2[MAXNV], g3[MAXNV], g4[MAXNV];
  int indx[MAXNV];
  int finish = 0;
  double time = time_start, dt = dttry, itol = 1.0 / c->p.ros_eps, dtnext = dt;
  int steps_done = 0;
  for (int iter = 1; iter <= c->p.ros_maxsteps; iter++) {
    double t0 = time;
    /* rosenbrock_jacobian (:9141-9193) */
    for (int n = 1; n <= nv; n++) {
      double wtmp = wc[n - 1];
      double h = wtmp * 1.0e-06 + 1.0e-14;
      wc[n - 1] = wtmp + h;
      ros_rhs(c, wc, Y, T, rhsp);
      wc[n - 1] = wtmp - h;
      ros_rhs(c, wc, Y, T, rhsm);
      wc[n - 1] = wtmp;
      for (int m = 1; m <= nv; m++) jac[(n - 1) * nv + m - 1] = (rhsp[m - 1] - rhsm[m - 1]) / (2.0 * h);
    }
    ros_rhs(c, wc, Y, T, rhs_sav);
    for (int m = 1; m <= nv; m++) { w_sav[m - 1] = wc[m - 1]; yscal[m - 1] = dmax(1.0, fabs(w_sav[m - 1])); }
    int accepted = 0;
    for (int jtry = 1; jtry <= c->p.ros_maxtry; jtry++) {
      /* rosenbrock_step (:9046-9139) */
      for (int n = 1; n <= nv; n++) {
        for (int m = 1; m <= nv; m++) amat[(n - 1) * nv + m - 1] = -jac[(n - 1) * nv + m - 1];
        amat[(n - 1) * nv + n - 1] = amat[(n - 1) * nv + n - 1] + 1.0 / (gam * dt);
      }
      for (int q = 0; q < nv; q++) indx[q] = q + 1;
      ludcmp_full(amat, indx, nv);
      for (int m = 0; m < nv; m++) g1[m] = rhs_sav[m];
      lubksb_full(amat, indx, g1, nv);
      for (int m = 0; m < nv; m++) wc[m] = w_sav[m] + a21 * g1[m];
      time = t0 + a2x * dt;
      ros_rhs(c, wc, Y, T, rhs);
      for (int m = 0; m < nv; m++) g2[m] = rhs[m] + c21 * g1[m] / dt;
      lubksb_full(amat, indx, g2, nv);
      for (int m = 0; m < nv; m++) wc[m] = w_sav[m] + a31 * g1[m] + a32 * g2[m];
      time = t0 + a3x * dt;
      ros_rhs(c, wc, Y, T, rhs);
      for (int m = 0; m < nv; m++) g3[m] = rhs[m] + (c31 * g1[m] + c32 * g2[m]) / dt;
      lubksb_full(amat, indx, g3, nv);
      for (int m = 0; m < nv; m++) g4[m] = rhs[m] + (c41 * g1[m] + c42 * g2[m] + c43 * g3[m]) / dt;
      lubksb_full(amat, indx, g4, nv);
      for (int m = 0; m < nv; m++) {
        wc[m] = w_sav[m] + b1 * g1[m] + b2 * g2[m] + b3 * g3[m] + b4 * g4[m];
        err[m] = e1 * g1[m] + e2 * g2[m] + e3 * g3[m] + e4 * g4[m];
      }
      time = t0 + dt;
      double errmax = 0.0;
      for (int m = 0; m < nv; m++) errmax = dmax(errmax, fabs(err[m] / yscal[m]));
      errmax = errmax * itol;
      if (errmax < 1.0 || finish == 1) {
        if (errmax > errcon) dtnext = safety * dt * pow(errmax, pgrow);
        else dtnext = grow * dt;
        accepted = 1;
        break;
      } else {
        dtnext = safety * dt * pow(errmax, pshrnk);
        double mag = dmax(fabs(dtnext), shrnk * fabs(dt));
        dt = dt >= 0 ? mag : -mag;
      }
    }
    if (!accepted) c->status |= STX_ST_ROS_TRY_CAP;
    steps_done = iter;
    double remaining = time_end - time;
    if (finish == 1 || remaining < 1.0e-012 * time_end) {
      break;
    } else {
      if (dtnext * 1.5 > remaining) { dt = remaining; finish = 1; }
      else { dt = dtnext; finish = 0; }
    }
    if (iter == c->p.ros_maxsteps) c->status |= STX_ST_ROS_STEPS_CAP;
  }
  (void)steps_done;
}

void ox_rosenbrock(ox_ctx *c, double *w, double *wa, double dttry, double time_start, double time_end) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz, nv = c->nv;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        size_t p = gi(c, i, j, k);
        double wc[MAXNV], Y[MAXNS], T;
        for (int m = 1; m <= nv; m++) wc[m - 1] = WG(w, p, m);
        for (int l = 1; l <= NS; l++) Y[l - 1] = WG(wa, p, l);
        T = WG(wa, p, J_T);
        ox_rosenbrock_cell(c, wc, Y, &T, dttry, time_start, time_end);
        for (int m = 1; m <= nv; m++) WG(w, p, m) = wc[m - 1];
        for (int l = 1; l <= NS; l++) WG(wa, p, l) = Y[l - 1];
        WG(wa, p, J_T) = T;
      }
}

/* compute_chemistry_cuf (kernels_gpu.F90:9503-9674): explicit source into fl */
void ox_compute_chemistry(ox_ctx *c, double *w, double *wa, double *fl) {
  int nx = c->g.nx, ny = c->g.ny, nz = c->g.nz;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        size_t p = gi(c, i, j, k), q = fi(c, i, j, k);
        double Y[MAXNS], conc[MAXNS], qlr[512];
        for (int lsp = 1; lsp <= NS; lsp++) WG(w, p, lsp) = dmax(WG(w, p, lsp), 0.0);
        double rho = WG(w, p, 1);
        for (int lsp = 2; lsp <= NS; lsp++) rho = rho + WG(w, p, lsp);
        double ri = 1.0 / rho;
        for (int lsp = 1; lsp <= NS; lsp++) {
          Y[lsp - 1] = WG(w, p, lsp) * ri;
          WG(wa, p, lsp) = Y[lsp - 1];
          conc[lsp - 1] = rho * Y[lsp - 1] / c->mw[lsp - 1];
        }
        double uu = WG(w, p, I_U) * ri, vv = WG(w, p, I_V) * ri, ww = WG(w, p, I_W) * ri;
        double rhoe = WG(w, p, I_E);
        double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
        double ee = rhoe * ri - qq;
        double tt = ox_temperature_from_e(c, ee, WG(wa, p, J_T), Y);
        WG(wa, p, J_T) = tt;
        reaction_rates(c, tt, conc, qlr);
        for (int lr = 1; lr <= c->t.nr; lr++)
          for (int lsp = 1; lsp <= NS; lsp++) {
            double wdtkj = (RX(c->t.p_coeffs, lr, lsp) - RX(c->t.r_coeffs, lr, lsp)) * qlr[lr - 1] * c->mw[lsp - 1];
            WF(fl, q, lsp) = WF(fl, q, lsp) - wdtkj;
          }
      }
}

/* ---------------------------------------------------------------- step drivers */
/* rk_sync (multideal_gpu.F90:536-621), no IBM / LES / NR / limiter / tripping */
void ox_rk_sync(ox_ctx *c, const stx_fields *f, double *fhat, double dt, int simpler) {
  for (int istep = 1; istep <= c->p.nrk; istep++) {
    double rhodt = c->p.rhork[istep - 1] * dt;
    double gamdt = c->p.gamrk[istep - 1] * dt;
    if (simpler == 1) ox_init_flux_simpler(c, f->fl, f->fln, f->fl_sav, rhodt);
    else ox_init_flux(c, f->fl, f->fln, rhodt);
    ox_bcswap(c, f->w, c->nv);
    ox_compute_aux(c, f->w, f->w_aux, 1, 1);
    ox_bcextr_var(c, f->w_aux + (size_t)(J_DIV - 1) * c->npg);
    ox_bcswap(c, f->w_aux + (size_t)(J_DUC - 1) * c->npg, 1);
    ox_bcswap(c, f->w_aux + (size_t)(J_DIV - 1) * c->npg, 1);
    ox_euler(c, 0, f->w_aux, fhat, f->fl, c->p.eul_imin, c->p.eul_imax);
    if (c->g.ny > 1) ox_euler(c, 1, f->w_aux, fhat, f->fl, c->p.eul_jmin, c->p.eul_jmax);
    if (c->g.nz > 1) ox_euler(c, 2, f->w_aux, fhat, f->fl, c->p.eul_kmin, c->p.eul_kmax);
    if (c->p.conservative_viscous == 1) {
      ox_visflx(c, f->w_aux, f->fl, fhat, 1);
      ox_visflx(c, f->w_aux, f->fl, fhat, 2);
    }
    ox_bc_nr(c, f->w_aux, f->w, f->fl);
    if (c->p.enable_chemistry == 1) ox_compute_chemistry(c, f->w, f->w_aux, f->fl);
    if (simpler == 1) ox_update_simpler_flux(c, f->fl, f->fln, f->fl_sav, gamdt);
    else ox_update_flux(c, f->fl, f->fln, gamdt);
    ox_update_field(c, f->w, f->fln, f->fluid_mask);
    ox_update_ghost_aux(c, f->w, f->w_aux, 0);
  }
}

/* sav_flx (multideal_gpu.F90:623-692): one RK3 right-hand side at t^n into fl_sav */
static void ox_sav_flx_step(ox_ctx *c, const stx_fields *f, double *fhat) {
  ox_bcswap(c, f->w, c->nv);
  ox_compute_aux(c, f->w, f->w_aux, 1, 1);
  ox_bcextr_var(c, f->w_aux + (size_t)(J_DIV - 1) * c->npg);
  ox_bcswap(c, f->w_aux + (size_t)(J_DUC - 1) * c->npg, 1);
  ox_bcswap(c, f->w_aux + (size_t)(J_DIV - 1) * c->npg, 1);
  memset(f->fl, 0, sizeof(double) * c->npi * c->nv);
  ox_euler(c, 0, f->w_aux, fhat, f->fl, c->p.eul_imin, c->p.eul_imax);
  if (c->g.ny > 1) ox_euler(c, 1, f->w_aux, fhat, f->fl, c->p.eul_jmin, c->p.eul_jmax);
  if (c->g.nz > 1) ox_euler(c, 2, f->w_aux, fhat, f->fl, c->p.eul_kmin, c->p.eul_kmax);
  if (c->p.conservative_viscous == 1) {
    ox_visflx(c, f->w_aux, f->fl, fhat, 1);
    ox_visflx(c, f->w_aux, f->fl, fhat, 2);
  }
  ox_bc_nr(c, f->w_aux, f->w, f->fl);
  if (c->p.enable_chemistry == 1) ox_compute_chemistry(c, f->w, f->w_aux, f->fl);
  ox_update_ghost_aux(c, f->w, f->w_aux, 0);
  ox_sav_flx(c, f->fl, f->fl_sav);
}

/* advance_solution (multideal_gpu.F90:1853-1931) */
void ox_advance_solution(ox_ctx *c, const stx_fields *f, double *fhat, double dt, double time) {
  if (c->p.enable_chemistry == 2) {
    if (c->p.operator_splitting == 1) {
      double dt_chem = dt;
      double dth = 0.5 * dt;
      ox_sav_flx_step(c, f, fhat);
      ox_compute_aux(c, f->w, f->w_aux, 1, 0);
      ox_rosenbrock_krylov(c, f->w, f->w_aux, f->fl_sav, dt_chem, time, time + dt_chem, 1);
      ox_rk_sync(c, f, fhat, dth, 1);
    } else {
      double dt_chem = 0.5 * dt;
      if (c->p.rosenbrock_version == 1) ox_rosenbrock(c, f->w, f->w_aux, dt_chem, time, time + dt_chem);
      else ox_rosenbrock_krylov(c, f->w, f->w_aux, NULL, dt_chem, time, time + dt_chem, 0);
      ox_rk_sync(c, f, fhat, dt, 0);
      ox_compute_aux(c, f->w, f->w_aux, 1, 0);
      if (c->p.rosenbrock_version == 1) ox_rosenbrock(c, f->w, f->w_aux, dt_chem, time, time + dt_chem);
      else ox_rosenbrock_krylov(c, f->w, f->w_aux, NULL, dt_chem, time, time + dt_chem, 0);
    }
  } else {
    ox_rk_sync(c, f, fhat, dt, 0);
  }
}
