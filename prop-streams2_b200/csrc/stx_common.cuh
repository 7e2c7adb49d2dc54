// stx_common.cuh -- device-side context, indexing and thermodynamics shared by
// the sm_100a kernels of libstx.so.
//
// Layouts are the reference's (src/multideal/multideal_gpu.F90:1481-1502):
// ghosted SoA fields w(1-ng:nx+ng,1-ng:ny+ng,1-ng:nz+ng,m), i fastest.  The
// species count is a template parameter so that per-species vectors live in
// registers; the host dispatches on the runtime value (STX_FOR_NS below).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/stx.h"

#define STX_MMAX 4     // Krylov dimension M_max (index_define.h:27)
#define STX_NSTAGE 4   // ROK4 stages (index_define.h:4)
#define STX_SPR 6      // most reactant (or product) species of one reaction
#define STX_SPW (4 * STX_SPR)   // sparse row: reactants, products, union (2 STX_SPR)

// species counts compiled into the library
#ifndef STX_FOR_NS
#define STX_FOR_NS(X) X(9) X(11) X(13) X(14) X(53)
#endif

// CTA sizes of the kernels that keep NS-long per-thread rows (chemistry) or
// (NS+4)-long per-face rows (the x sweeps) in shared memory: smaller CTAs for
// large mechanisms keep the static shared memory under 48 KB.
__host__ __device__ constexpr int chem_block(int ns) { return ns > 20 ? 32 : 128; }
__host__ __device__ constexpr int xsweep_block(int ns) { return ns > 20 ? 64 : 128; }

struct DevTab {
  int ns, nr, icl, icr, nset, ntab, ncp;
  double tmin, dtab, Ru;
  const double *mw, *mwinv, *rgas;
  const double *trange;           // (ns, nset+1)
  const double *cp, *cv;          // (ncp, ns, nset)
  const double *cpi, *cvi;        // the same with coef_l / (l + 1) for l >= 0 (species_poly_int)
  const double *visc_r, *lam_r;   // repacked [it][lsp]
  const double *diff_r;           // repacked [it][lsp][msp] (msp fastest)
  const int *reac_ty, *is_rev;
  const double *arr_a, *arr_b, *arr_ea, *falloff;   // (nr,2) / (nr,5)
  const double *tb_eff, *r_coeffs, *p_coeffs;       // (nr, ns)
  const double *kc_r;             // repacked [it][lr]
  // sparse stoichiometry, per reaction lr (built from r_coeffs / p_coeffs):
  // sp_cnt = nR | nP << 8 | nU << 16; sp_idx / sp_coef [lr][STX_SPW] hold the
  // reactant species (nu' != 0), the product species (nu'' != 0) and their
  // union, each in ascending species order, with nu', nu'' and nu'' - nu'.
  const int *sp_cnt;
  const unsigned char *sp_idx;
  const double *sp_coef;
  // the same stoichiometry by species (CSR): for species k the reactions
  // sk_r[sk_ptr[k] .. sk_ptr[k+1]) with nu'' - nu' != 0 or a nonzero term, in
  // ascending order, and their coefficients sk_c = nu'' - nu'
  const int *sk_ptr;
  const int *sk_r;
  const double *sk_c;
  const double *wk_a, *wk_b;      // Wilke pair factors [l][m]
  int n_eoi;
  const double *aw_eoi, *coeff_eoi, *beta0;
  const int *nainsp;
};

struct DevGrid {
  int nx, ny, nz, ng, nxg, nyg, nzg;
  long long npg, npi;
  const double *x, *y, *z;
  const double *dcsidx, *detady, *dzitdz, *dcsidxs, *detadys, *dzitdzs;
};

struct DevPar {
  double p0, rho0, u0, eps_sensor, tol, sensor_threshold, ros_eps;
  int ep_order, nkeep, weno_scheme, weno_version, flux_splitting, sensor_type, visc_order, nv_aux;
  int fzf[6];
  int ros_maxsteps, ros_maxtry;
  double cd1[5][5];               // coeff_deriv1(l, lmax) -> cd1[l][lmax]
  unsigned int *status;           // device status word
  // Simulation time in device memory, set only while a step is captured into a
  // CUDA graph: the chemistry kernels then take their window [time, time + dttry]
  // from it (the same double operations the host performs) instead of their
  // t0 / t1 arguments, so a replayed step sees the current time.
  const double *time_d;
  // Step size in device memory, set only while a CFL-driven step is captured
  // (stx_graph_create_cfl; its last computation in the step, from the CFL
  // maxima): a kernel that takes a dt-derived scalar by value (rhodt, gamdt,
  // the chemistry's dttry) then receives its coefficient in that argument and
  // forms coefficient * (scale * dt), the double operations the host performs
  // on its own dt (scale: the factor of the splitting, 1 or 0.5).
  const double *dt_d;
  // precision form: 0 plain FP64; 1 mixed -- central face fluxes, viscous and
  // diffusive fluxes and the transport properties in FP32 (RK residual still
  // accumulated in FP64; T(e) Newton, rates, K_c and the chemistry in FP64)
  int mixed;
  // convective sweep kernel per direction: 0 staged shared-memory tiles (where
  // they apply), 1 one face per thread; chosen by the autotuner or by
  // STX_EULER_KERNEL=face
  int sweep_kind[3];
  // persistent CTAs per SM of the cell chemistry kernels (0: occupancy limit)
  int chem_ctas_per_sm;
  // most CTAs of a batched-reactor launch (0: no cap), so that several
  // concurrent launches leave the SMs room for other work
  int batch_ctas_max;
  // wall temperature of the isothermal-wall ghost fill (bc tag 6)
  double T_wall;
};

struct DevCtx {
  DevTab t;
  DevGrid g;
  DevPar p;
};

// ---------------------------------------------------------------- indexing
__device__ __forceinline__ long long gidx(const DevGrid &g, int i, int j, int k) {
  return (long long)(i + g.ng - 1) + (long long)g.nxg * ((long long)(j + g.ng - 1) + (long long)g.nyg * (long long)(k + g.ng - 1));
}
__device__ __forceinline__ long long fidx(const DevGrid &g, int i, int j, int k) {
  return (long long)(i - 1) + (long long)g.nx * ((long long)(j - 1) + (long long)g.ny * (long long)(k - 1));
}
// field m (1-based) of a ghosted array
#define FG(a, p, m) ((a)[(p) + (long long)((m) - 1) * g.npg])
#define FI(a, q, m) ((a)[(q) + (long long)((m) - 1) * g.npi])

__device__ __forceinline__ double ldg(const double *p) { return __ldg(p); }

// Fortran real**integer (the same repeated product as the oracle)
__device__ __forceinline__ double ipow(double x, int n) {
  double r = 1.0;
  int u = n < 0 ? -n : n;
  for (int q = 0; q < u; q++) r *= x;
  return n < 0 ? 1.0 / r : r;
}
__device__ __forceinline__ double dmax_(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmin_(double a, double b) { return a < b ? a : b; }

__device__ __forceinline__ void set_status(const DevPar &p, unsigned bits) {
  if (p.status) atomicOr(p.status, bits);
}

// ---------------------------------------------------------------- thermo
__device__ __forceinline__ double trange_(const DevTab &t, int lsp, int jm) {
  return ldg(t.trange + (long long)(jm - 1) * t.ns + lsp - 1);
}
__device__ __forceinline__ double cpc(const DevTab &t, const double *arr, int l, int lsp, int m) {
  return ldg(arr + ((long long)(m - 1) * t.ns + lsp - 1) * t.ncp + (l - t.icl));
}

// Numerical-Recipes locate (kernels_gpu.F90:6397-6415)
__device__ __forceinline__ int locate_range(const DevTab &t, double T, int lsp) {
  int jl = 0, ju = t.nset + 2;
  while (ju - jl > 1) {
    int jm = (ju + jl) / 2;
    if (T >= trange_(t, lsp, jm)) jl = jm; else ju = jm;
  }
  if (jl < 1) jl = 1;
  if (jl > t.nset) jl = t.nset;
  return jl;
}

// get_cp_dev (kernels_gpu.F90:6384-6432)
template <int NS>
__device__ double mix_cp(const DevTab &t, double tt, const double *Y) {
  int nrange[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) nrange[k] = 1;
  if (t.nset > 1) {
#pragma unroll
    for (int k = 0; k < NS; k++) nrange[k] = locate_range(t, tt, k + 1);
  }
  double cploc = 0.0;
  double pw = 1.0;                       // tt^pe: ipow's partial products, formed once
  int pe = 0;
  for (int l = t.icl; l <= t.icr; l++) {
    double tpow;
    if (l >= 0) {
      while (pe < l) { pw = pw * tt; pe++; }
      tpow = pw;
    } else {
      tpow = ipow(tt, l);
    }
    double cp_l = 0.0;
#pragma unroll
    for (int k = 0; k < NS; k++) cp_l = cp_l + cpc(t, t.cp, l, k + 1, nrange[k]) * Y[k];
    cploc = cploc + cp_l * tpow;
  }
  return cploc;
}

// get_mixture_temperature_from_e_dev (kernels_gpu.F90:6532-6622) with coef = the
// cv table; with the cp table it is get_mixture_temperature_from_h_roe_dev
// (:6810-6900), T from the mixture enthalpy.
template <int NS>
__device__ double temp_from_poly(const DevTab &t, const double *coef, const DevPar &p, double ee, double T_start,
                                 const double *Y);
template <int NS>
__device__ __forceinline__ double temp_from_e(const DevTab &t, const DevPar &p, double ee, double T_start,
                                              const double *Y) {
  return temp_from_poly<NS>(t, t.cv, p, ee, T_start, Y);
}
template <int NS>
__device__ double temp_from_poly(const DevTab &t, const double *coef, const DevPar &p, double ee, double T_start,
                                 const double *Y) {
  int nrange[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) nrange[k] = 1;
  if (t.nset > 1) {
#pragma unroll
    for (int k = 0; k < NS; k++) nrange[k] = locate_range(t, T_start, k + 1);
  }
  double T_old = T_start, tt = T_start;
  bool conv = false;
  for (int iter = 1; iter <= 10; iter++) {
    if (t.nset > 1) {
#pragma unroll
      for (int k = 0; k < NS; k++) {
        int nl = nrange[k];
        if (T_old < trange_(t, k + 1, nl)) nrange[k] = nrange[k] - 1;
        else if (T_old > trange_(t, k + 1, nl + 1)) nrange[k] = nrange[k] + 1;
        if (nrange[k] < 1) nrange[k] = 1;
        if (nrange[k] > t.nset) nrange[k] = t.nset;
      }
    }
    double sumb = 0.0;
#pragma unroll
    for (int k = 0; k < NS; k++) sumb = sumb + cpc(t, coef, t.icr + 1, k + 1, nrange[k]) * Y[k];
    double ebar = ee - sumb;
    double den = 0.0, num = 0.0;
    double pw = 1.0;                     // T_old^pe: ipow's partial products, formed once
    int pe = 0;
    for (int l = t.icl; l <= t.icr; l++) {
      double T_pow;
      if (l >= 0) {
        while (pe < l) { pw = pw * T_old; pe++; }
        T_pow = pw;
      } else {
        T_pow = ipow(T_old, l);
      }
      double tden = T_pow, tnum;
      if (l == -1) {
        tnum = log(T_old);
      } else {
        double T_powp = T_old * T_pow;
        // T_powp / (l + 1): a division by 1, 2 or 4 is an exact scaling (the
        // same result as the division), the others are divisions
        const int d = l + 1;
        tnum = d == 1 ? T_powp : (d == 2 ? T_powp * 0.5 : (d == 4 ? T_powp * 0.25 : T_powp / (l + 1.0)));
      }
      double cv_l = 0.0;
#pragma unroll
      for (int k = 0; k < NS; k++) cv_l = cv_l + cpc(t, coef, l, k + 1, nrange[k]) * Y[k];
      num = num + cv_l * tnum;
      den = den + cv_l * tden;
    }
    tt = T_old + (ebar - num) / den;
    if (fabs(tt - T_old) < p.tol) { conv = true; break; }
    T_old = tt;
  }
  if (!conv) set_status(p, STX_ST_NEWTON_CAP);
  return tt;
}

// get_species_h/e_from_temperature_dev (kernels_gpu.F90:7104-7183).  ai is the
// integrated table (DevTab::cpi / cvi): entry l holds coef_l / (l + 1), the
// quotient the reference forms for every term, formed once at context creation
// (the same correctly rounded division, so the same bits).  The powers T^(l+1)
// for l + 1 >= 1 are formed incrementally, T^(n+1) = T^n * T, the very products
// of the repeated multiplication ipow performs.
__device__ __forceinline__ double species_poly_int(const DevTab &t, const double *ai, double tt, int isp) {
  int nr = 1;
  if (t.nset > 1) nr = locate_range(t, tt, isp);
  double hh = cpc(t, ai, t.icr + 1, isp, nr);
  double tp = 1.0;                       // tt^tpe, ipow's partial products
  int tpe = 0;
  for (int l = t.icl; l <= t.icr; l++) {
    if (l == -1) {
      hh = hh + cpc(t, ai, l, isp, nr) * log(tt);
    } else if (l + 1 >= 1) {
      while (tpe < l + 1) { tp = tp * tt; tpe++; }
      hh = hh + cpc(t, ai, l, isp, nr) * tp;
    } else {
      hh = hh + cpc(t, ai, l, isp, nr) * ipow(tt, l + 1);
    }
  }
  return hh;
}

// table row index and fraction (kernels_gpu.F90:6245-6249)
__device__ __forceinline__ void table_pos(const DevTab &t, double tt, int &itt, double &dtt) {
  itt = (int)((tt - t.tmin) / t.dtab) + 1;
  if (itt < 1) itt = 1;
  if (itt > t.ntab) itt = t.ntab;
  double tloc = t.tmin + (itt - 1) * t.dtab;
  dtt = (tt - tloc) / t.dtab;
}

// ---------------------------------------------------------------- launch helpers
#define STX_CUDA_TRY(x)                          \
  do {                                           \
    cudaError_t e_ = (x);                        \
    if (e_ != cudaSuccess) return STX_E_CUDA;    \
  } while (0)

inline int grid1d(long long n, int block) {
  long long b = (n + block - 1) / block;
  return (int)(b < 1 ? 1 : b);
}
