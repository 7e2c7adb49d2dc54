// stx_chem.cuh -- device functions of the stiff chemistry cell updates, shared
// by the kernels of stx_chem.cu: production rates, the ROK4 Krylov cell update
// (kernels_gpu.F90:10360-11205) and the work-stealing cell claim.
#pragma once
#include <type_traits>
#include "stx_kernels.cuh"

// Linkage of the ROK4 right-hand side: one out-of-line copy (default).  Inlined
// at its three call sites it halves the local-memory frame (2.2 KB instead of
// 3.9 KB per thread) and is 10 % faster on a fresh field, but on a developed
// 256^3 reacting field the cells take more sub-steps and the three inlined
// copies overflow the instruction cache: 306 ms against 178 ms per launch
// (bit-identical results).
#ifndef STX_RHS_LINKAGE
#define STX_RHS_LINKAGE __noinline__
#endif


// x^e for a stoichiometric exponent: the square as one product (the reference's
// x**2.0 through pow costs a logarithm and an exponential), any other
// exponent through pow.
__device__ __forceinline__ double stoich_pow(double x, double e) { return e == 2.0 ? x * x : pow(x, e); }

// Temperature-table position of T for K_c (kernels_gpu.F90:9259-9264).
__device__ __forceinline__ void kc_pos(const DevTab &t, double tt, int &itt, double &dtt) {
  itt = (int)((tt - t.tmin) / t.dtab) + 1;
  if (itt < 1) itt = 1;
  if (itt > t.ntab) itt = t.ntab;
  double ttleft = (itt - 1) * t.dtab + t.tmin;
  dtt = (tt - ttleft) / t.dtab;
}

// Rate constants of reaction lr at T (kernels_gpu.F90:9266-9330): kf from the
// Arrhenius, Lindemann, Troe or SRI form (tbs is the third-body concentration
// sum the fall-off forms use), kb = kf / K_c with K_c interpolated in the 1-K
// table.  KCF selects where K_c is read: false -> t.kc_r, the context's
// temperature-major repacking; true -> t.kc_r in the reference's own layout
// kc_tab(num_t_tab+1, nr).
template <bool KCF>
__device__ __forceinline__ void rate_consts(const DevTab &t, int lr, int ty, double tt, double Rtti, int itt,
                                            double dtt, double tbs, double &kf, double &kb) {
  const int nr = t.nr;
  double A1 = ldg(t.arr_a + lr), B1 = ldg(t.arr_b + lr), E1 = ldg(t.arr_ea + lr);
  if (ty == 0 || ty == 1) {
    kf = A1;
    if (B1 != 0.0) kf = kf * pow(tt, B1);
    if (E1 != 0.0) kf = kf * exp(-E1 * Rtti);
  } else {
    double A2 = ldg(t.arr_a + nr + lr), B2 = ldg(t.arr_b + nr + lr), E2 = ldg(t.arr_ea + nr + lr);
    double k0 = A1 * pow(tt, B1) * exp(-E1 * Rtti);
    double kinf = A2 * pow(tt, B2) * exp(-E2 * Rtti);
    double rpres = k0 * tbs / kinf;
    if (ty == 2) {
      kf = kinf * (rpres / (1.0 + rpres));
    } else if (ty == 3) {
      if (rpres < 1e-30) {
        kf = k0 * tbs;
      } else {
        double F1 = ldg(t.falloff + lr), F2 = ldg(t.falloff + nr + lr), F3 = ldg(t.falloff + 2 * nr + lr),
               F4 = ldg(t.falloff + 3 * nr + lr);
        double fcent = (1.0 - F1) * exp(-tt / F2) + F1 * exp(-tt / F3);
        if (F4 != -3.14) fcent = fcent + exp(-F4 / tt);
        fcent = log10(fcent);
        double coff = -0.4 - 0.67 * fcent;
        double noff = 0.75 - 1.27 * fcent;
        double doff = 0.14;
        double lp = log10(rpres);
        const double tr = (lp + coff) / (noff - doff * (lp + coff));
        double foff = pow(10.0, (1.0 / (1.0 + tr * tr)) * fcent);   // (1 + tr^2)^-1 as a product and a division
        kf = kinf * (rpres / (1.0 + rpres)) * foff;
      }
    } else if (ty == 4) {
      double F1 = ldg(t.falloff + lr), F2 = ldg(t.falloff + nr + lr), F3 = ldg(t.falloff + 2 * nr + lr),
             F4 = ldg(t.falloff + 3 * nr + lr), F5 = ldg(t.falloff + 4 * nr + lr);
      double xoff = 1.0 / (1.0 + pow(log10(rpres), 2.0));
      double foff = F4 * pow(F1 * exp(-F2 / tt) + exp(-tt / F3), xoff) * pow(tt, F5);
      kf = kinf * (rpres / (1.0 + rpres)) * foff;
    } else {
      kf = 0.0;
    }
  }
  if (__ldg(t.is_rev + lr) == 1) {
    double a, dkc;
    if (KCF) {
      const double *kcol = t.kc_r + (long long)lr * (t.ntab + 1) + (itt - 1);
      a = ldg(kcol);
      dkc = ldg(kcol + 1) - a;
    } else {
      const double *kcrow = t.kc_r + (long long)(itt - 1) * nr;
      a = ldg(kcrow + lr);
      dkc = ldg(kcrow + nr + lr) - a;
    }
    double kc = a + dkc * dtt;
    kb = kf / kc;
  } else {
    kb = 0.0;
  }
}

// Production terms of rosenbrock_rhs / rosenbrock_krylov_rhs / compute_chemistry_cuf
// (kernels_gpu.F90:9251-9357): rhs_k += W_k sum_r (nu''_kr - nu'_kr) q_r, summed
// over reactions in order for every species, with dense species loops.
// explicit_form selects the explicit kernel's form (every species term,
// :9654-9661) instead of the Rosenbrock one.  The third-body sum is the sum
// the reference forms in its fall-off branch and again for three-body
// reactions; it is formed once here (same terms, same order, same value).
template <int NS, bool KCF = false>
__device__ void chem_source(const DevTab &t, double tt, const double *conc, double *rhs, bool explicit_form) {
  const int nr = t.nr;
  double Rtti = 1.0 / (t.Ru * tt);
  int itt;
  double dtt;
  kc_pos(t, tt, itt, dtt);
#pragma unroll 1
  for (int lr = 0; lr < nr; lr++) {
    int ty = __ldg(t.reac_ty + lr);
    double tbs = 1.0;
    if (ty != 0) {
      tbs = 0.0;
#pragma unroll
      for (int k = 0; k < NS; k++) tbs = tbs + ldg(t.tb_eff + (long long)k * nr + lr) * conc[k];
    }
    double kf, kb;
    rate_consts<KCF>(t, lr, ty, tt, Rtti, itt, dtt, tbs, kf, kb);
    double q1 = 1.0, q2 = 1.0;
#pragma unroll
    for (int k = 0; k < NS; k++) {
      double rr = ldg(t.r_coeffs + (long long)k * nr + lr), pp = ldg(t.p_coeffs + (long long)k * nr + lr);
      if (rr == 1.0) q1 = q1 * conc[k];
      else if (rr != 0.0) q1 = q1 * stoich_pow(conc[k], rr);
      if (pp == 1.0) q2 = q2 * conc[k];
      else if (pp != 0.0) q2 = q2 * stoich_pow(conc[k], pp);
    }
    double tb = (ty == 1) ? tbs : 1.0;
    double qlr = tb * (kf * q1 - kb * q2);
#pragma unroll
    for (int k = 0; k < NS; k++) {
      double rr = ldg(t.r_coeffs + (long long)k * nr + lr), pp = ldg(t.p_coeffs + (long long)k * nr + lr);
      if (explicit_form) {
        rhs[k] = rhs[k] - (pp - rr) * qlr * ldg(t.mw + k);
      } else if (rr != 0.0 || pp != 0.0) {
        double wdtkj = (pp - rr) * qlr;
        rhs[k] = rhs[k] + wdtkj * ldg(t.mw + k);
      }
    }
  }
}

// The Rosenbrock-form production terms of chem_source over the sparse
// stoichiometry lists (t.sp_*): the same terms in the same order, with compact
// rolled loops.  conc and rhs are per-thread rows with stride S (shared memory).
template <int NS, int S>
__device__ void chem_source_sp(const DevTab &t, double tt, const double *conc, double *rhs) {
  const int nr = t.nr;
  double Rtti = 1.0 / (t.Ru * tt);
  int itt;
  double dtt;
  kc_pos(t, tt, itt, dtt);
#pragma unroll 1
  for (int lr = 0; lr < nr; lr++) {
    int ty = __ldg(t.reac_ty + lr);
    double tbs = 1.0;
    if (ty != 0) {
      tbs = 0.0;
#pragma unroll 1
      for (int k = 0; k < NS; k++) tbs = tbs + ldg(t.tb_eff + (long long)k * nr + lr) * conc[k * S];
    }
    double kf, kb;
    rate_consts<false>(t, lr, ty, tt, Rtti, itt, dtt, tbs, kf, kb);
    const int cnt = __ldg(t.sp_cnt + lr);
    const unsigned char *ix = t.sp_idx + (long long)lr * STX_SPW;
    const double *cf = t.sp_coef + (long long)lr * STX_SPW;
    double q1 = 1.0, q2 = 1.0;
#pragma unroll 1
    for (int n = 0; n < (cnt & 255); n++) {
      double x = conc[__ldg(ix + n) * S], e = ldg(cf + n);
      if (e == 1.0) q1 = q1 * x;
      else q1 = q1 * stoich_pow(x, e);
    }
#pragma unroll 1
    for (int n = 0; n < ((cnt >> 8) & 255); n++) {
      double x = conc[__ldg(ix + STX_SPR + n) * S], e = ldg(cf + STX_SPR + n);
      if (e == 1.0) q2 = q2 * x;
      else q2 = q2 * stoich_pow(x, e);
    }
    double tb = (ty == 1) ? tbs : 1.0;
    double qlr = tb * (kf * q1 - kb * q2);
#pragma unroll 1
    for (int n = 0; n < (cnt >> 16); n++) {
      int k = __ldg(ix + 2 * STX_SPR + n);
      double wdtkj = ldg(cf + 2 * STX_SPR + n) * qlr;
      rhs[k * S] = rhs[k * S] + wdtkj * ldg(t.mw + k);
    }
  }
}

// rosenbrock_krylov_rhs (kernels_gpu.F90:10794-10976), PaSR off.  With the
// context's tables (KCF false) the production terms run over the sparse
// stoichiometry with per-thread rows in shared memory (launch with
// chem_block(NS) threads); with the reference's raw tables (KCF true) over the
// dense species loops.
template <int NS, bool KCF = false>
__device__ STX_RHS_LINKAGE void krylov_rhs(const DevCtx &c, const double *w_sav, const double *w_mom, double T_iter,
                                           double *rhs) {
  const DevTab &t = c.t;
  double Y[NS], conc[NS], wl[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) wl[k] = w_sav[k] > 0.0 ? w_sav[k] : 0.0;
  double rho = wl[0];
#pragma unroll
  for (int k = 1; k < NS; k++) rho = rho + wl[k];
  double ri = 1.0 / rho;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    Y[k] = wl[k] * ri;
    conc[k] = rho * Y[k] / ldg(t.mw + k);
  }
  double uu = w_mom[0] * ri, vv = w_mom[1] * ri, ww = w_mom[2] * ri;
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double ee = (w_mom[3] * ri) - qq;
  double tt = temp_from_e<NS>(t, c.p, ee, T_iter, Y);
  if (KCF) {
#pragma unroll
    for (int m = 0; m < NS; m++) rhs[m] = 0.0;
    chem_source<NS, KCF>(t, tt, conc, rhs, false);
  } else {
    constexpr int CB = chem_block(NS);
    __shared__ double s_conc[NS * CB], s_rhs[NS * CB];
    double *cs = s_conc + threadIdx.x, *rs = s_rhs + threadIdx.x;
#pragma unroll
    for (int k = 0; k < NS; k++) {
      cs[k * CB] = conc[k];
      rs[k * CB] = 0.0;
    }
    chem_source_sp<NS, CB>(t, tt, cs, rs);
#pragma unroll
    for (int k = 0; k < NS; k++) rhs[k] = rs[k * CB];
  }
}

template <int NV>
__device__ __forceinline__ double norm2v(const double *v) {
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < NV; q++) s = s + v[q] * v[q];
  return sqrt(s);
}

// inv_matrix_krylov with ludcmp_krylov / lubksb_krylov (kernels_gpu.F90:11061-11205)
// on the leading d x d block of a column-major 4x4 matrix.
static __device__ void inv_matrix_k(double *a, int d) {
#define AK(r, s) a[((s) - 1) * STX_MMAX + (r) - 1]
  if (d == 1) { AK(1, 1) = 1.0 / AK(1, 1); return; }
  int indx[STX_MMAX] = {1, 2, 3, 4};
  const double tiny = 1.5e-16;
  double vv[STX_MMAX];
  bool early = false;
  for (int i = 1; i <= d && !early; i++) {
    double amax = 0.0;
    for (int j = 1; j <= d; j++) if (fabs(AK(i, j)) > amax) amax = fabs(AK(i, j));
    if (amax < tiny) early = true;
    else vv[i - 1] = 1.0 / amax;
  }
  if (!early) {
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
  double y[STX_MMAX * STX_MMAX];
  for (int r = 1; r <= d; r++) for (int s = 1; s <= d; s++) y[(s - 1) * STX_MMAX + r - 1] = (r == s) ? 1.0 : 0.0;
  for (int s = 1; s <= d; s++) {
    double *b = y + (s - 1) * STX_MMAX;
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
  for (int r = 1; r <= d; r++) for (int s = 1; s <= d; s++) AK(r, s) = y[(s - 1) * STX_MMAX + r - 1];
#undef AK
}

// The ROK4 method's coefficients (rosenbrock_krylov_kernel, kernels_gpu.F90:10463-10480),
// in constant memory: indexed by the rolled stage loops, a per-thread copy
// takes 256 bytes of every thread's local frame.
__constant__ double c_rok4_alpha[STX_NSTAGE][3] = {{0.0, 0.0, 0.0},
                                                   {0.432364435748567, 0.0, 0.0},
                                                   {-0.514211316876170, 1.382271144617360, 0.0},
                                                   {-0.514211316876170, 1.382271144617360, 0.0}};
__constant__ double c_rok4_gmc[STX_NSTAGE][3] = {{0.0, 0.0, 0.0},
                                                 {-0.602765307997356, 0.0, 0.0},
                                                 {-1.389195789724843, 1.072950969011413, 0.0},
                                                 {0.992356412977094, -1.390032613873701, -0.440875890223325}};
__constant__ double c_rok4_bs[STX_NSTAGE] = {0.194335256262729, 0.483167813989227, 0.0, 0.322496929748044};
__constant__ double c_rok4_bt[STX_NSTAGE] = {-0.217819895945721, 1.03130847478467, 0.186511421161047, 0.0};

// The ROK4 integration of one state vector of NV components
// (rosenbrock_krylov_kernel body, kernels_gpu.F90:10463-10610).  V holds the
// Krylov basis; the basis handed back (Vb) is its first mA columns.  The
// system is the functor f:
//   f.rhs(y, T_iter, out)               the right-hand side at y;
//   f.accept(y, time, T_iter, time_end) after an accepted step: updates the
//                                       temperature guess, may move time_end;
//   f.done(time, T_iter, steps)         at the end: time reached, last T, steps.
// fls (simpler == 1 only) is the cell's saved residual fl_sav, component m at
// fls[m * fstride]; maxsteps caps the steps (ros_maxsteps).
//
// Per-thread working set, kept small because it lives in local memory for
// every resident thread: V (Krylov basis), inv, the stage vectors Ks and one
// 3 x NV scratch that serves the Arnoldi temporaries (jac, wl), the stage
// temporaries (ys, F, GK) and the new state.  The right-hand side at the
// start of a step, f(VEC), is formed once: the Arnoldi iteration uses it (less
// fl_sav: rhs_sav), and the first stage, whose state is VEC itself and whose
// temperature guess is the same, reuses it with the operations the reference
// applies to a fresh evaluation (f(VEC) + 0 - fl_sav), so the result is the
// same bit for bit with one right-hand side fewer per step.
//
// A: the storage of the Krylov basis V and the stage vectors Ks -- double (the
// reference method), or float for the FP32/FP64-split form of the batched
// reactors, where the state, every right-hand side (T from h, rates, K_c), the
// finite-difference Jacobian products, the small Krylov matrices and the error
// norm stay FP64 and only those two arrays are rounded to FP32.  f(VEC), which
// the finite differences subtract, is then kept in the FP64 scratch S2.
template <int NV, class F, typename A = double>
__device__ void rok4_core(const DevCtx &c, F &f, double *VEC, double T_iter, const double *fls, long long fstride,
                          double dttry, double time_start, double time_end, int simpler, int maxsteps) {
  const double gam = 0.572816062482135;
  constexpr bool AD = std::is_same<A, double>::value;
  // the Arnoldi matrices live in the stage vectors 2..4 (dead until the
  // stages; Ks is lengthened where they need more room), in arrays of their
  // own with FP32 stage vectors
  constexpr int NH = (STX_MMAX + 1) * STX_MMAX, NI = STX_MMAX * STX_MMAX;
  constexpr bool HK = AD;
  constexpr int NKS = HK && NV + NH + NI > NV * STX_NSTAGE ? NV + NH + NI : NV * STX_NSTAGE;
  A V[NV * (STX_MMAX + 1)];
  double inv[STX_MMAX * STX_MMAX];
  A Ks[NKS];                                 // Ks[0..NV) holds f(VEC) until stage 1 replaces it (A = double)
  double S0[NV], S1[NV], S2[NV];             // scratch: jac / wl, then ys / F / GK, then the new state
  double *raw;
  if constexpr (AD) raw = Ks;
  else raw = S2;
  auto fsav = [&](int m) -> double { return fls[(long long)m * fstride]; };
  // rhs_sav of the reference: f(VEC), less fl_sav with the simpler splitting
  auto rhs_sav = [&](int m) -> double { return simpler == 1 ? raw[m] - fsav(m) : raw[m]; };
  int mA = 0;
#pragma unroll
  for (int q = 0; q < STX_MMAX * STX_MMAX; q++) inv[q] = 0.0;
  double time = time_start, dt = dttry, errn = 1.0;
  int it = 0;
  while (time < (time_end - 1.0e-12)) {
    dt = dmin_(dt, time_end - time);
    it = it + 1;
    // ---- arnoldi (:10664-10792)
    {
      const double TOL = 1e-6, eps = 1.0e-08;
      double HHo[HK ? 1 : NH], HIo[HK ? 1 : NI];
      double *HH, *HI;
      if constexpr (HK) {
        HH = Ks + NV;
        HI = Ks + NV + NH;
      } else {
        HH = HHo;
        HI = HIo;
      }
      double prj[STX_MMAX], lam[STX_MMAX];
#pragma unroll
      for (int q = 0; q < (STX_MMAX + 1) * STX_MMAX; q++) HH[q] = 0.0;
#pragma unroll
      for (int q = 0; q < STX_MMAX * STX_MMAX; q++) HI[q] = 0.0;
#pragma unroll
      for (int q = 0; q < NV * (STX_MMAX + 1); q++) V[q] = 0.0;
      mA = 0;
      f.rhs(VEC, T_iter, raw);
      double nrm;
      {
        double sq = 0.0;
        for (int m = 0; m < NV; m++) { const double r = rhs_sav(m); sq = sq + r * r; }
        nrm = sqrt(sq);
      }
      for (int m = 0; m < NV; m++) V[m] = rhs_sav(m) / nrm;
      // the outer loops stay rolled (unroll 1): unrolled, the Krylov algebra
      // is straight-line code far larger than the instruction cache
#pragma unroll 1
      for (int kk = 1; kk <= STX_MMAX; kk++) {
        double *jac = S0, *wl = S1;
        for (int m = 0; m < NV; m++) wl[m] = VEC[m] + (eps * V[(kk - 1) * NV + m]);
        f.rhs(wl, T_iter, jac);
        if (simpler == 1)
          for (int m = 0; m < NV; m++) jac[m] = jac[m] - fsav(m);
        for (int m = 0; m < NV; m++) jac[m] = (jac[m] - rhs_sav(m)) / eps;
#pragma unroll 1
        for (int jj = 1; jj <= kk; jj++) {
          double dot = 0.0;
          for (int m = 0; m < NV; m++) dot = dot + V[(jj - 1) * NV + m] * jac[m];
          HH[(kk - 1) * (STX_MMAX + 1) + jj - 1] = dot;
          for (int m = 0; m < NV; m++) jac[m] = jac[m] - (dot * V[(jj - 1) * NV + m]);
        }
        double hn = norm2v<NV>(jac);
        HH[(kk - 1) * (STX_MMAX + 1) + kk] = hn;
        for (int m = 0; m < NV; m++) V[kk * NV + m] = jac[m] / hn;
        // projections of rhs_sav on the first kk basis vectors (the rest are zero)
#pragma unroll 1
        for (int ll = 1; ll <= STX_MMAX; ll++) {
          double s = 0.0;
          if (ll <= kk)
            for (int m = 0; m < NV; m++) s = s + V[(ll - 1) * NV + m] * rhs_sav(m);
          prj[ll - 1] = s;
        }
#pragma unroll 1
        for (int n = 1; n <= kk; n++)
#pragma unroll 1
          for (int nn = 1; nn <= kk; nn++) {
            double h = -(dt * gam * HH[(nn - 1) * (STX_MMAX + 1) + n - 1]);
            if (n == nn) h = h + 1.0;
            HI[(nn - 1) * STX_MMAX + n - 1] = h;
          }
        for (int n = kk + 1; n <= STX_MMAX; n++) HI[(n - 1) * STX_MMAX + n - 1] = 1.0;
        inv_matrix_k(HI, kk);
        for (int ll = 1; ll <= STX_MMAX; ll++) {
          double s = 0.0;
          for (int jj = 1; jj <= STX_MMAX; jj++) s = s + HI[(jj - 1) * STX_MMAX + ll - 1] * prj[jj - 1];
          lam[ll - 1] = s;
        }
        if (fabs(dt * gam * hn) * fabs(lam[kk - 1]) < TOL) {
          mA = kk;
#pragma unroll
          for (int q = 0; q < STX_MMAX * STX_MMAX; q++) inv[q] = HI[q];
          break;
        }
      }
    }
    // ---- stages.  The reference forms A = Vb (I - inv) and B = A Vb^T (nv x nv)
    // and applies B to F (:10540-10566).  Here B F = A (Vb^T F): the mA
    // projections of F on the basis first, then per row the 4 entries of A,
    // formed in registers from V and inv.  O(4 nv) instead of O(4 nv^2) per
    // stage; the sums are regrouped (rounding-level difference).
#pragma unroll 1
    for (int ii = 1; ii <= STX_NSTAGE; ii++) {
      double *ys = S0, *Fv = S1, *GK = S2;
      if (ii == 1) {
        for (int m = 0; m < NV; m++) Fv[m] = raw[m];            // f(VEC), formed for the Arnoldi iteration
      } else {
        for (int m = 0; m < NV; m++) ys[m] = VEC[m];
#pragma unroll 1
        for (int jj = 1; jj <= ii - 1; jj++)
          for (int m = 0; m < NV; m++) ys[m] = ys[m] + dt * c_rok4_alpha[ii - 1][jj - 1] * Ks[(jj - 1) * NV + m];
        f.rhs(ys, T_iter, Fv);
      }
      for (int m = 0; m < NV; m++) GK[m] = 0.0;
#pragma unroll 1
      for (int jj = 1; jj <= ii - 1; jj++)
        for (int m = 0; m < NV; m++) GK[m] = GK[m] + c_rok4_gmc[ii - 1][jj - 1] / gam * Ks[(jj - 1) * NV + m];
      for (int m = 0; m < NV; m++) Fv[m] = Fv[m] + GK[m];
      if (simpler == 1)
        for (int m = 0; m < NV; m++) Fv[m] = Fv[m] - fsav(m);
      double pf[STX_MMAX];
#pragma unroll
      for (int q = 0; q < STX_MMAX; q++) {
        double s = 0.0;
        if (q < mA)
          for (int jj = 0; jj < NV; jj++) s = s + V[q * NV + jj] * Fv[jj];
        pf[q] = s;
      }
#pragma unroll 1
      for (int ll = 0; ll < NV; ll++) {
        double vb[STX_MMAX];
#pragma unroll
        for (int q = 0; q < STX_MMAX; q++) vb[q] = (q < mA) ? V[q * NV + ll] : 0.0;
        double s = 0.0;
#pragma unroll
        for (int kk = 0; kk < STX_MMAX; kk++) {
          double a = vb[0] * ((kk == 0 ? 1.0 : 0.0) - inv[kk * STX_MMAX + 0]);
#pragma unroll
          for (int jj = 1; jj < STX_MMAX; jj++) a = a + vb[jj] * ((jj == kk ? 1.0 : 0.0) - inv[kk * STX_MMAX + jj]);
          s = s + a * pf[kk];
        }
        Ks[(ii - 1) * NV + ll] = Fv[ll] - s - GK[ll];
      }
    }
    // the new state and its error norm (the norm's sum in component order)
    double *ys = S0;
    double esq = 0.0;
    for (int ll = 0; ll < NV; ll++) {
      double a = VEC[ll], b = VEC[ll];
      for (int ii = 0; ii < STX_NSTAGE; ii++) {
        a = a + dt * c_rok4_bs[ii] * Ks[ii * NV + ll];
        b = b + dt * c_rok4_bt[ii] * Ks[ii * NV + ll];
      }
      ys[ll] = a;
      const double ev = (b - a) / ((1.0e-4) * a + 1.0e-8);
      esq = esq + ev * ev;
    }
    double errmax = sqrt(esq);
    double fac = 0.625 * pow(errn, 0.1) / pow(errmax, 0.175);
    double dtnext = dt * dmin_(5.0, dmax_(0.2, fac));
    if (errmax < 1.0) {
      time = time + dt;
      for (int m = 0; m < NV; m++) VEC[m] = ys[m];
      f.accept(VEC, time, T_iter, time_end);
    }
    dt = dtnext;
    errn = errmax;
    if (it > maxsteps) { set_status(c.p, STX_ST_ROS_STEPS_CAP); break; }
  }
  f.done(time, T_iter, it);
}

// The flow cell: state (rho Y_k, rho u, rho v, rho w, rho E), constant volume
// (rosenbrock_krylov_rhs, :10794-10976); after an accepted step T follows from
// e by the Newton inversion (:10597-10606).
template <int NS, bool KCF>
struct Rok4Flow {
  const DevCtx &c;
  __device__ __forceinline__ void rhs(const double *y, double T_iter, double *out) const {
    krylov_rhs<NS, KCF>(c, y, y + NS, T_iter, out);
#pragma unroll
    for (int m = NS; m < NS + 4; m++) out[m] = 0.0;
  }
  __device__ __forceinline__ void accept(const double *VEC, double, double &T_iter, double &) const {
    double rho = VEC[0];
    for (int n = 1; n < NS; n++) rho = rho + VEC[n];
    double ri = 1.0 / rho, Y[NS];
#pragma unroll
    for (int n = 0; n < NS; n++) Y[n] = VEC[n] * ri;
    double uu = VEC[NS] * ri, vv = VEC[NS + 1] * ri, ww = VEC[NS + 2] * ri;
    double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
    double ee = VEC[NS + 3] * ri - qq;
    T_iter = temp_from_e<NS>(c.t, c.p, ee, T_iter, Y);
  }
  __device__ __forceinline__ void done(double, double, int) const {}
};

// The flow cell without the simpler splitting's residual: the chemistry
// leaves rho u, rho v, rho w and rho E unchanged (their right-hand side is 0),
// so every Krylov vector, stage vector and error term of those four
// components is exactly zero and the integration runs over the NS species
// densities alone, the other four read from mom (the cell's state, fixed over
// the window).  Dropping exact zeros from the sums leaves every species
// component, step size and step count as the full NS + 4 component form gives
// them, bit for bit (measured: the same fields after a Strang half at 256^3,
// in 113 ms instead of 122 ms).  The forms part only where the full form
// breaks down: a momentum component of exactly -1e-4 makes its error term
// (b - a) / (1e-4 a + 1e-8) 0/0 there.
template <int NS, bool KCF>
struct Rok4FlowSpecies : Rok4Flow<NS, KCF> {
  const double *mom;
  __device__ __forceinline__ void rhs(const double *y, double T_iter, double *out) const {
    krylov_rhs<NS, KCF>(this->c, y, mom, T_iter, out);
  }
};

// The adiabatic constant-pressure 0-D reactor (no counterpart in the reference,
// whose batch reactor is constant-volume): state Y_k, clipped at 0 where
// evaluated; h and p fixed; T from h by the Newton iteration of
// get_mixture_temperature_from_h_roe_dev (kernels_gpu.F90:6810-6900);
// rho = p / (R T); dY_k/dt = W_k omega_k / rho.  Per-thread shared-memory rows
// as in krylov_rhs (launch with chem_block(NS) threads).
template <int NS>
__device__ __noinline__ void cp_rhs(const DevCtx &c, const double *y, double T_iter, double h, double p,
                                    double *out) {
  const DevTab &t = c.t;
  double Yc[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) Yc[k] = y[k] > 0.0 ? y[k] : 0.0;
  double tt = temp_from_poly<NS>(t, t.cp, c.p, h, T_iter, Yc);
  double rm = 0.0;
#pragma unroll
  for (int k = 0; k < NS; k++) rm = rm + ldg(t.rgas + k) * Yc[k];
  double rho = p / (rm * tt);
  constexpr int CB = chem_block(NS);
  __shared__ double s_conc[NS * CB], s_rhs[NS * CB];
  double *cs = s_conc + threadIdx.x, *rs = s_rhs + threadIdx.x;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    cs[k * CB] = rho * Yc[k] / ldg(t.mw + k);
    rs[k * CB] = 0.0;
  }
  chem_source_sp<NS, CB>(t, tt, cs, rs);
#pragma unroll
  for (int k = 0; k < NS; k++) out[k] = rs[k * CB] / rho;
}

template <int NS>
struct Rok4ConstP {
  const DevCtx &c;
  double h, p, T0, ign_factor, end_factor;
  double t_ign, time_reached, T_final;
  int steps;
  __device__ __forceinline__ void rhs(const double *y, double T_iter, double *out) const {
    cp_rhs<NS>(c, y, T_iter, h, p, out);
  }
  __device__ __forceinline__ void accept(const double *y, double time, double &T_iter, double &time_end) {
    double Yc[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) Yc[k] = y[k] > 0.0 ? y[k] : 0.0;
    T_iter = temp_from_poly<NS>(c.t, c.t.cp, c.p, h, T_iter, Yc);
    if (t_ign < 0.0 && T_iter > ign_factor * T0) {
      t_ign = time;
      double te = end_factor * time;
      if (te < time_end) time_end = te;
    }
  }
  __device__ __forceinline__ void done(double time, double T_iter, int it) {
    time_reached = time;
    T_final = T_iter;
    steps = it;
  }
};

// One ROK4 flow cell; fls: the cell's fl_sav components at stride fstride (simpler == 1).
template <int NS, bool KCF = false>
__device__ __forceinline__ void rok4_cell(const DevCtx &c, double *VEC, double T_iter, const double *fls,
                                          long long fstride, double dttry, double time_start, double time_end,
                                          int simpler) {
  if (simpler != 1) {
    Rok4FlowSpecies<NS, KCF> f{{c}, VEC + NS};
    rok4_core<NS>(c, f, VEC, T_iter, nullptr, 0, dttry, time_start, time_end, 0, c.p.ros_maxsteps);
  } else {
    Rok4Flow<NS, KCF> f{c};
    rok4_core<NS + 4>(c, f, VEC, T_iter, fls, fstride, dttry, time_start, time_end, simpler, c.p.ros_maxsteps);
  }
}

// claim the next cell: warp-aggregated atomicAdd over the currently active lanes
__device__ __forceinline__ long long claim(unsigned int *counter) {
  unsigned mask = __activemask();
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  int rank = __popc(mask & ((1u << lane) - 1u));
  unsigned base = 0;
  if (lane == leader) base = atomicAdd(counter, (unsigned)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  return (long long)base + rank;
}

