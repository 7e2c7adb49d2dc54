// stx_euler.cu -- hybrid central-KEEP / WENO convective fluxes fused with their
// divergence (euler_{x,y,z} of src/multideal/multideal_gpu.F90:877-1044 and the
// kernels of src/multideal/kernels_gpu.F90:88-2063, 2065-3295).
//
// B200 design:
//  * x sweep: one CTA of 128 threads per pencil segment; thread t computes face
//    f0+t, the faces go through shared memory and threads 1..127 apply
//    fl(i) += (fhat_i - fhat_{i-1}) * dxi/dx -- no fhat round trip through HBM.
//  * y/z sweeps: tiles of 32 contiguous i (coalesced) x 8 faces along the
//    sweep, one face per thread, differenced through shared memory; one
//    redundant face per 7 cells.
//  * WENO faces use the structure of the multi-species eigenvectors
//    (kernels_gpu.F90:2703-2984): the species block of L is identity + rank one,
//    so every characteristic variable follows from two per-point scalars
//    (Q = sum_k b1i_k W_k - b2 u.W_mom + b2 W_E and sigma = sum_k W_k): O(ns)
//    per stencil point instead of O(ns^2).  The back projection keeps the
//    reference's summation order.  Results equal the reference's dense
//    products up to rounding.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <tuple>
#include <utility>

#include "stx_kernels.cuh"

// wenorec_1d / wenorec_1d_rusanov (kernels_gpu.F90:2065-2637) for one variable;
// vp/vm indexed by stencil slot 1..2*ws (slot 0 unused).
__device__ __forceinline__ double weno_rec(const double *vp, const double *vm, int i, int ord, int version, double bs) {
  if (ord == 1) return vp[i] + vm[i + 1];
  if (ord == 2) {
    double t, bp0, bp1, bm0, bm1;
    t = vp[i] - vp[i - 1]; bp0 = bs * (t * t);
    t = vp[i + 1] - vp[i]; bp1 = bs * (t * t);
    t = vm[i + 2] - vm[i + 1]; bm0 = bs * (t * t);
    t = vm[i + 1] - vm[i]; bm1 = bs * (t * t);
    t = 0.000001 + bp0; bp0 = (1.0 / 3.0) / (t * t);
    t = 0.000001 + bm0; bm0 = (1.0 / 3.0) / (t * t);
    t = 0.000001 + bp1; bp1 = (2.0 / 3.0) / (t * t);
    t = 0.000001 + bm1; bm1 = (2.0 / 3.0) / (t * t);
    double sp = bp0 + bp1, sm = bm0 + bm1;
    bp0 = bp0 / sp; bp1 = bp1 / sp; bm0 = bm0 / sm; bm1 = bm1 / sm;
    double vminus = bp0 * (-vp[i - 1] + 3 * vp[i]) + bp1 * (vp[i] + vp[i + 1]);
    double vplus = bm0 * (-vm[i + 2] + 3 * vm[i + 1]) + bm1 * (vm[i] + vm[i + 1]);
    return 0.5 * (vminus + vplus);
  }
  if (ord == 3) {
    const double dwe0 = 1.0 / 10.0, dwe1 = 6.0 / 10.0, dwe2 = 3.0 / 10.0;
    const double d0 = 13.0 / 12.0, d1 = 1.0 / 4.0;
    const double c0 = 1.0 / 3.0, c1 = 5.0 / 6.0, c2 = -1.0 / 6.0, c3 = -7.0 / 6.0, c4 = 11.0 / 6.0;
    double a, b, bp0, bp1, bp2, bm0, bm1, bm2;
    a = vp[i] - 2.0 * vp[i + 1] + vp[i + 2]; b = 3.0 * vp[i] - 4.0 * vp[i + 1] + vp[i + 2];
    bp2 = bs * (d0 * (a * a) + d1 * (b * b));
    a = vp[i - 1] - 2.0 * vp[i] + vp[i + 1]; b = vp[i - 1] - vp[i + 1];
    bp1 = bs * (d0 * (a * a) + d1 * (b * b));
    a = vp[i] - 2.0 * vp[i - 1] + vp[i - 2]; b = 3.0 * vp[i] - 4.0 * vp[i - 1] + vp[i - 2];
    bp0 = bs * (d0 * (a * a) + d1 * (b * b));
    a = vm[i + 1] - 2.0 * vm[i] + vm[i - 1]; b = 3.0 * vm[i + 1] - 4.0 * vm[i] + vm[i - 1];
    bm2 = bs * (d0 * (a * a) + d1 * (b * b));
    a = vm[i + 2] - 2.0 * vm[i + 1] + vm[i]; b = vm[i + 2] - vm[i];
    bm1 = bs * (d0 * (a * a) + d1 * (b * b));
    a = vm[i + 1] - 2.0 * vm[i + 2] + vm[i + 3]; b = 3.0 * vm[i + 1] - 4.0 * vm[i + 2] + vm[i + 3];
    bm0 = bs * (d0 * (a * a) + d1 * (b * b));
    double sp, sm;
    if (version == 0) {
      double t;
      t = 0.000001 + bp0; bp0 = dwe0 / (t * t);
      t = 0.000001 + bm0; bm0 = dwe0 / (t * t);
      t = 0.000001 + bp1; bp1 = dwe1 / (t * t);
      t = 0.000001 + bm1; bm1 = dwe1 / (t * t);
      t = 0.000001 + bp2; bp2 = dwe2 / (t * t);
      t = 0.000001 + bm2; bm2 = dwe2 / (t * t);
    } else {
      const double eps40 = 1.0e-40;
      double tp = fabs(bp0 - bp2) + eps40, tm = fabs(bm0 - bm2) + eps40;
      bp0 = (bp0 + eps40) / (bp0 + tp); bm0 = (bm0 + eps40) / (bm0 + tm);
      bp1 = (bp1 + eps40) / (bp1 + tp); bm1 = (bm1 + eps40) / (bm1 + tm);
      bp2 = (bp2 + eps40) / (bp2 + tp); bm2 = (bm2 + eps40) / (bm2 + tm);
      bp0 = dwe0 / bp0; bm0 = dwe0 / bm0;
      bp1 = dwe1 / bp1; bm1 = dwe1 / bm1;
      bp2 = dwe2 / bp2; bm2 = dwe2 / bm2;
    }
    sp = bp0 + bp1 + bp2;
    sm = bm0 + bm1 + bm2;
    bp0 = bp0 / sp; bp1 = bp1 / sp; bp2 = bp2 / sp;
    bm0 = bm0 / sm; bm1 = bm1 / sm; bm2 = bm2 / sm;
    double vminus = bp2 * (c0 * vp[i] + c1 * vp[i + 1] + c2 * vp[i + 2]) +
                    bp1 * (c2 * vp[i - 1] + c1 * vp[i] + c0 * vp[i + 1]) +
                    bp0 * (c0 * vp[i - 2] + c3 * vp[i - 1] + c4 * vp[i]);
    double vplus = bm2 * (c0 * vm[i + 1] + c1 * vm[i] + c2 * vm[i - 1]) +
                   bm1 * (c2 * vm[i + 2] + c1 * vm[i + 1] + c0 * vm[i]) +
                   bm0 * (c0 * vm[i + 3] + c3 * vm[i + 2] + c4 * vm[i + 1]);
    return vminus + vplus;
  }
  // ord == 4: WENO-7
  const double d1 = 1.0 / 36.0, d2 = 13.0 / 12.0, d3 = 781.0 / 720.0;
  const double dwe[4] = {1.0 / 35.0, 12.0 / 35.0, 18.0 / 35.0, 4.0 / 35.0};
  double bp[4], bm[4], a, b, e;
  a = -11 * vp[i] + 18 * vp[i + 1] - 9 * vp[i + 2] + 2 * vp[i + 3];
  b = 2 * vp[i] - 5 * vp[i + 1] + 4 * vp[i + 2] - vp[i + 3];
  e = -vp[i] + 3 * vp[i + 1] - 3 * vp[i + 2] + vp[i + 3];
  bp[3] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
  a = -2 * vp[i - 1] - 3 * vp[i] + 6 * vp[i + 1] - vp[i + 2];
  b = vp[i - 1] - 2 * vp[i] + vp[i + 1];
  e = -vp[i - 1] + 3 * vp[i] - 3 * vp[i + 1] + vp[i + 2];
  bp[2] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
  a = vp[i - 2] - 6 * vp[i - 1] + 3 * vp[i] + 2 * vp[i + 1];
  b = vp[i - 1] - 2 * vp[i] + vp[i + 1];
  e = -vp[i - 2] + 3 * vp[i - 1] - 3 * vp[i] + vp[i + 1];
  bp[1] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
  a = -2 * vp[i - 3] + 9 * vp[i - 2] - 18 * vp[i - 1] + 11 * vp[i];
  b = -vp[i - 3] + 4 * vp[i - 2] - 5 * vp[i - 1] + 2 * vp[i];
  e = -vp[i - 3] + 3 * vp[i - 2] - 3 * vp[i - 1] + vp[i];
  bp[0] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
  a = -11 * vm[i + 1] + 18 * vm[i] - 9 * vm[i - 1] + 2 * vm[i - 2];
  b = 2 * vm[i + 1] - 5 * vm[i] + 4 * vm[i - 1] - vm[i - 2];
  e = -vm[i + 1] + 3 * vm[i] - 3 * vm[i - 1] + vm[i - 2];
  bm[3] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
  a = -2 * vm[i + 2] - 3 * vm[i + 1] + 6 * vm[i] - vm[i - 1];
  b = vm[i + 2] - 2 * vm[i + 1] + vm[i];
  e = -vm[i + 2] + 3 * vm[i + 1] - 3 * vm[i] + vm[i - 1];
  bm[2] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
  a = vm[i + 3] - 6 * vm[i + 2] + 3 * vm[i + 1] + 2 * vm[i];
  b = vm[i + 2] - 2 * vm[i + 1] + vm[i];
  e = -vm[i + 3] + 3 * vm[i + 2] - 3 * vm[i + 1] + vm[i];
  bm[1] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
  a = -2 * vm[i + 4] + 9 * vm[i + 3] - 18 * vm[i + 2] + 11 * vm[i + 1];
  b = -vm[i + 4] + 4 * vm[i + 3] - 5 * vm[i + 2] + 2 * vm[i + 1];
  e = -vm[i + 4] + 3 * vm[i + 3] - 3 * vm[i + 2] + vm[i + 1];
  bm[0] = d1 * (a * a) + d2 * (b * b) + d3 * (e * e);
  double sp = 0.0, sm = 0.0;
#pragma unroll
  for (int l = 0; l < 4; l++) {
    double t = 0.000001 + bs * bp[l]; bp[l] = dwe[l] / (t * t);
    t = 0.000001 + bs * bm[l]; bm[l] = dwe[l] / (t * t);
    sp = sp + bp[l]; sm = sm + bm[l];
  }
#pragma unroll
  for (int l = 0; l < 4; l++) { bp[l] = bp[l] / sp; bm[l] = bm[l] / sm; }
  double vminus = bp[3] * (6 * vp[i] + 26 * vp[i + 1] - 10 * vp[i + 2] + 2 * vp[i + 3]) +
                  bp[2] * (-2 * vp[i - 1] + 14 * vp[i] + 14 * vp[i + 1] - 2 * vp[i + 2]) +
                  bp[1] * (2 * vp[i - 2] - 10 * vp[i - 1] + 26 * vp[i] + 6 * vp[i + 1]) +
                  bp[0] * (-6 * vp[i - 3] + 26 * vp[i - 2] - 46 * vp[i - 1] + 50 * vp[i]);
  double vplus = bm[3] * (6 * vm[i + 1] + 26 * vm[i] - 10 * vm[i - 1] + 2 * vm[i - 2]) +
                 bm[2] * (-2 * vm[i + 2] + 14 * vm[i + 1] + 14 * vm[i] - 2 * vm[i - 1]) +
                 bm[1] * (2 * vm[i + 3] - 10 * vm[i + 2] + 26 * vm[i + 1] + 6 * vm[i]) +
                 bm[0] * (-6 * vm[i + 4] + 26 * vm[i + 3] - 46 * vm[i + 2] + 50 * vm[i + 1]);
  return (vminus + vplus) / 24.0;
}

#define WMAX 8   // 2 * max weno_scheme
#define CF_LMAX 4                            // largest ep_order / 2 (coeff_deriv1 is 4 x 4)
#define CF_NPAIR (CF_LMAX * (CF_LMAX + 1) / 2)   // stencil pairs (l, m), m < l <= CF_LMAX

// Central KEEP(n) face flux (kernels_gpu.F90:145-337 and the y/z copies), computed
// in R: double for the plain form, float for the mixed form (the fields are
// read in FP64 and rounded once).
template <int NS, int DIR, typename R>
__device__ __forceinline__ void central_flux(const DevCtx &c, const double *__restrict__ wa, long long p, long long st,
                                             bool fz, R *fh) {
  const DevGrid &g = c.g;
  auto ld = [&](long long q, int m) -> R { return (R)FG(wa, q, m); };
  const int J_U = NS + 1, J_V = NS + 2, J_W = NS + 3, J_H = NS + 4, J_P = NS + 6, J_R = NS + 11;
  const int Jn = J_U + DIR;
  int lmax = c.p.ep_order / 2;
  if (lmax < 1) lmax = 1;
  if (lmax > CF_LMAX) lmax = CF_LMAX;
  const int nkeep = c.p.nkeep;
  // Per stencil pair (l, m), a = p - m st, b = p + (l - m) st: the mass-flux
  // factor (un_a + un_b) (rho_a + rho_b) drhof that the species and the
  // momentum/energy fluxes share.  The reference forms it inside its species
  // loop (the KEEP density factor drhof depends on rho_a, rho_b only); it is
  // formed once per pair here, with the same operations.
  R up[CF_NPAIR];
#pragma unroll
  for (int l = 1; l <= CF_LMAX; l++)
#pragma unroll
    for (int m = 0; m < l; m++) {
      const int q = l * (l - 1) / 2 + m;
      up[q] = R(0.0);
      if (l <= lmax) {
        long long a = p - m * st, b = p + (l - m) * st;
        R rhoi = ld(a, J_R), uni = ld(a, Jn);
        R rhoip = ld(b, J_R), unip = ld(b, Jn);
        R rhom = rhoi + rhoip, drhof;
        if (nkeep <= 0) {
          drhof = R(1.0);
        } else {
          R drho = R(2.0) * (rhoip - rhoi) / rhom;
          R t = (R(0.5) * drho) * (R(0.5) * drho), t2 = t;
          R sumden = R(1.0) + t / R(3.0);
          for (int n = 2; n <= nkeep; n++) { int n2 = 2 * n; t = t2 * t; sumden = sumden + t / (R(1.0) + n2); }
          drhof = R(1.0) / sumden;
        }
        up[q] = (uni + unip) * rhom * drhof;
      }
    }
#pragma unroll 1
  for (int lsp = 1; lsp <= NS; lsp++) {
    R ft1 = R(0.0);
#pragma unroll
    for (int l = 1; l <= CF_LMAX; l++) {
      if (l <= lmax) {
        R uvs1 = R(0.0);
#pragma unroll
        for (int m = 0; m < l; m++) {
          long long a = p - m * st, b = p + (l - m) * st;
          uvs1 = uvs1 + up[l * (l - 1) / 2 + m] * (ld(a, lsp) + ld(b, lsp));
        }
        ft1 = ft1 + R(c.p.cd1[l][lmax]) * uvs1;
      }
    }
    R fh1 = R(0.25) * ft1;
    fh[lsp - 1] = fz ? R(0.0) : fh1;
  }
  R ft2 = 0, ft3 = 0, ft4 = 0, ft5 = 0, ft6 = 0;
#pragma unroll
  for (int l = 1; l <= CF_LMAX; l++) {
    if (l > lmax) break;
    R uvs2 = 0, uvs3 = 0, uvs4 = 0, uvs5 = 0, uvs6 = 0, uvs5_i = 0, uvs5_k = 0, uvs5_p = 0;
#pragma unroll
    for (int m = 0; m < l; m++) {
      const int q = l * (l - 1) / 2 + m;
      long long a = p - m * st, b = p + (l - m) * st;
      R rhoi = ld(a, J_R), uui = ld(a, J_U), vvi = ld(a, J_V), wwi = ld(a, J_W);
      R enti = ld(a, J_H), ppi = ld(a, J_P);
      R rhoip = ld(b, J_R), uuip = ld(b, J_U), vvip = ld(b, J_V), wwip = ld(b, J_W);
      R entip = ld(b, J_H), ppip = ld(b, J_P);
      R uni = DIR == 0 ? uui : (DIR == 1 ? vvi : wwi);
      R unip = DIR == 0 ? uuip : (DIR == 1 ? vvip : wwip);
      R uv_part = up[q];
      if (nkeep >= 0) {
        R eei = enti - ppi / rhoi - R(0.5) * (uui * uui + vvi * vvi + wwi * wwi);
        R eeip = entip - ppip / rhoip - R(0.5) * (uuip * uuip + vvip * vvip + wwip * wwip);
        R eem = eei + eeip, deef;
        if (nkeep == 0) {
          deef = R(1.0);
        } else {
          R dee = R(2.0) * (eeip - eei) / eem;
          R te = (R(0.5) * dee) * (R(0.5) * dee);
          R te2 = te;
          R sde = R(1.0) + te, sne = R(1.0) + te / R(3.0);
          for (int n = 2; n <= nkeep; n++) {
            int n2 = 2 * n;
            te = te2 * te;
            sde = sde + te;
            sne = sne + te / (R(1.0) + n2);
          }
          deef = sne / sde;
        }
        uvs2 = uvs2 + uv_part * (uui + uuip);
        uvs3 = uvs3 + uv_part * (vvi + vvip);
        uvs4 = uvs4 + uv_part * (wwi + wwip);
        uvs5_i = uvs5_i + uv_part * eem * deef;
        uvs5_k = uvs5_k + uv_part * (uui * uuip + vvi * vvip + wwi * wwip);
        uvs5_p = uvs5_p + R(4.0) * (uni * ppip + unip * ppi);
        uvs6 = uvs6 + (R(2.0)) * (ppi + ppip);
      } else {
        uvs2 = uvs2 + uv_part * (uui + uuip);
        uvs3 = uvs3 + uv_part * (vvi + vvip);
        uvs4 = uvs4 + uv_part * (wwi + wwip);
        uvs5 = uvs5 + uv_part * (enti + entip);
        uvs6 = uvs6 + (R(2.0)) * (ppi + ppip);
      }
    }
    R cl = R(c.p.cd1[l][lmax]);
    ft2 = ft2 + cl * uvs2;
    ft3 = ft3 + cl * uvs3;
    ft4 = ft4 + cl * uvs4;
    ft5 = ft5 + cl * (nkeep >= 0 ? (uvs5_i + uvs5_k + uvs5_p) : uvs5);
    ft6 = ft6 + cl * uvs6;
  }
  R fm0 = R(0.25) * ft2, fm1 = R(0.25) * ft3, fm2 = R(0.25) * ft4, fh5 = R(0.25) * ft5;
  if (fz) { fm0 = fm1 = fm2 = fh5 = R(0.0); }
  if (DIR == 0) fm0 = fm0 + R(0.5) * ft6;
  if (DIR == 1) fm1 = fm1 + R(0.5) * ft6;
  if (DIR == 2) fm2 = fm2 + R(0.5) * ft6;
  fh[NS] = fm0; fh[NS + 1] = fm1; fh[NS + 2] = fm2; fh[NS + 3] = fh5;
}

// Roe state (compute_roe_average, kernels_gpu.F90:2986-3295) between p and q.
template <int NS>
__device__ __forceinline__ void roe_state(const DevCtx &c, const double *__restrict__ wa, long long p, long long q,
                                          double &b1, double &b2, double &b3, double &rho_r, double &cr, double &ci,
                                          double &hr, double vel[3], double *yr, double *prhoi) {
  const DevGrid &g = c.g;
  const DevTab &t = c.t;
  const int J_U = NS + 1, J_V = NS + 2, J_W = NS + 3, J_H = NS + 4, J_P = NS + 6, J_R = NS + 11;
  double rho = FG(wa, p, J_R), uu = FG(wa, p, J_U), vv = FG(wa, p, J_V), ww = FG(wa, p, J_W);
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double h = FG(wa, p, J_H), pp = FG(wa, p, J_P);
  double ee = h - pp / rho - qq;
  double rho_L = rho, ee_L = ee;
  double rhop = FG(wa, q, J_R), up = FG(wa, q, J_U), vp = FG(wa, q, J_V), wp = FG(wa, q, J_W);
  double qqp = 0.5 * (up * up + vp * vp + wp * wp);
  double hp = FG(wa, q, J_H), ppp = FG(wa, q, J_P);
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
  double rm = 0.0, drho[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) {
    double yy = FG(wa, p, k + 1), yyp = FG(wa, q, k + 1);
    drho[k] = rhop * yyp - rho_L * yy;
    yy = (r * yyp + yy) * rp1;
    rm = rm + ldg(t.rgas + k) * yy;
    yr[k] = yy;
  }
  double told = p_over_rho / rm;
  double tt = temp_from_e<NS>(t, c.p, ee, told, yr);
  double cploc = mix_cp<NS>(t, tt, yr);
  double gamloc = cploc / (cploc - rm);
  double gm1loc = gamloc - 1.0;
  double p_e = rho * gm1loc;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    double eei = species_poly_int(t, t.cvi, tt, k + 1);
    prhoi[k] = ldg(t.rgas + k) * tt + gm1loc * (ee - eei);
  }
  double etot = ee + qq;
  double dp_SLV = ppp - pp, de_SLV = eep - ee_L;
  double pede = p_e * de_SLV;
  double dp_err = dp_SLV - pede;
  double den = pede * pede;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    double pr = prhoi[k] * drho[k];
    dp_err = dp_err - pr;
    den = den + pr * pr;
  }
  double dpfact = dp_err / dmax_(den, 0.000001);
  p_e = p_e * (1.0 + pede * dpfact);
#pragma unroll
  for (int k = 0; k < NS; k++) prhoi[k] = prhoi[k] * (1.0 + prhoi[k] * drho[k] * dpfact);
  double cc = p_over_rho / rho * p_e;
#pragma unroll
  for (int k = 0; k < NS; k++) cc = cc + yr[k] * prhoi[k];
  cr = sqrt(cc);
  ci = 1.0 / cr;
  b3 = etot;
  b2 = p_e / (rho * cc);
  b1 = -b2 * (etot - 2.0 * qq);
  rho_r = rho;
  hr = h;
  vel[0] = uu; vel[1] = vv; vel[2] = ww;
}

// Characteristic (Roe) WENO face flux with LLF splitting (kernels_gpu.F90:338-423).
template <int NS, int DIR>
__device__ __noinline__ void weno_char_flux(const DevCtx &c, const double *__restrict__ wa, long long p, long long st,
                                            double *fh) {
  const DevGrid &g = c.g;
  const int NV = NS + 4;
  const int J_U = NS + 1, J_H = NS + 4, J_P = NS + 6, J_C = NS + 7, J_R = NS + 11;
  const int T1 = DIR == 0 ? 1 : 0, T2 = DIR == 2 ? 1 : 2;
  const int ws = c.p.weno_scheme, wsz = 2 * ws;
  double b1, b2, b3, rr, cr, ci, hr, vr[3], yr[NS], prhoi[NS];
  roe_state<NS>(c, wa, p, p + st, b1, b2, b3, rr, cr, ci, hr, vr, yr, prhoi);
  const double un = vr[DIR], ut1 = vr[T1], ut2 = vr[T2];
  const double cci = ci * ci;
  double b1i[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) b1i[k] = b1 + prhoi[k] * cci;
  // LLF eigenvalue bounds over the stencil (:345-358)
  double ev1 = -1.0, ev2 = -1.0, ev4 = -1.0;
  for (int l = 1; l <= wsz; l++) {
    long long q = p + (l - ws) * st;
    double u = FG(wa, q, J_U + DIR), cq = FG(wa, q, J_C);
    ev1 = dmax_(fabs(u - cq), ev1);
    ev2 = dmax_(fabs(u), ev2);
    ev4 = dmax_(fabs(u + cq), ev4);
  }
  // per-point scalars
  double Qw[WMAX + 1], Qf[WMAX + 1], sw[WMAX + 1], sf[WMAX + 1];
  double Wn[WMAX + 1], Fn[WMAX + 1], Wt1[WMAX + 1], Ft1[WMAX + 1], Wt2[WMAX + 1], Ft2[WMAX + 1];
  double rl[WMAX + 1], rul[WMAX + 1];
  for (int l = 1; l <= wsz; l++) {
    long long q = p + (l - ws) * st;
    double rho = FG(wa, q, J_R), u0 = FG(wa, q, J_U), u1 = FG(wa, q, J_U + 1), u2 = FG(wa, q, J_U + 2);
    double h = FG(wa, q, J_H), pp = FG(wa, q, J_P);
    double vel[3] = {u0, u1, u2};
    double rhou = rho * vel[DIR];
    double Sw = 0.0, Sf = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int k = 0; k < NS; k++) {
      double y = FG(wa, q, k + 1);
      double wk = rho * y, fk = rhou * y;
      Sw = Sw + b1i[k] * wk;
      Sf = Sf + b1i[k] * fk;
      s1 = s1 + wk;
      s2 = s2 + fk;
    }
    double wm0 = rho * u0, wm1 = rho * u1, wm2 = rho * u2;
    double fm0 = u0 * rhou, fm1 = u1 * rhou, fm2 = u2 * rhou;
    if (DIR == 0) fm0 = fm0 + pp;
    if (DIR == 1) fm1 = fm1 + pp;
    if (DIR == 2) fm2 = fm2 + pp;
    double wE = rho * h - pp, fE = h * rhou;
    Qw[l] = Sw - b2 * (vr[0] * wm0 + vr[1] * wm1 + vr[2] * wm2) + b2 * wE;
    Qf[l] = Sf - b2 * (vr[0] * fm0 + vr[1] * fm1 + vr[2] * fm2) + b2 * fE;
    sw[l] = s1; sf[l] = s2;
    double wmv[3] = {wm0, wm1, wm2}, fmv[3] = {fm0, fm1, fm2};
    Wn[l] = wmv[DIR]; Fn[l] = fmv[DIR];
    Wt1[l] = wmv[T1]; Ft1[l] = fmv[T1];
    Wt2[l] = wmv[T2]; Ft2[l] = fmv[T2];
    rl[l] = rho; rul[l] = rhou;
  }
  // betascale (wenorec_1d, :2372-2381)
  const double u0 = c.p.u0, rho0 = c.p.rho0;
  const double r2u2 = rho0 * rho0 * (u0 * u0), r2u4 = r2u2 * (u0 * u0);
  const double bsA = 1.0 / r2u2, bsB = 1.0 / r2u4;
  int ord = ws < 1 ? 1 : ws;
  double fi[NV];
  double vp[WMAX + 1], vm[WMAX + 1];
  // characteristic 1 (u - c) and NS+4 (u + c)
#pragma unroll 1
  for (int side = 0; side < 2; side++) {
    double sg = side == 0 ? 1.0 : -1.0, ev = side == 0 ? ev1 : ev4;
    for (int l = 1; l <= wsz; l++) {
      double wc = 0.5 * (Qw[l] + sg * ci * (un * sw[l] - Wn[l]));
      double gc = 0.5 * (Qf[l] + sg * ci * (un * sf[l] - Fn[l]));
      double cc = 0.5 * (gc + ev * wc);
      vp[l] = cc; vm[l] = gc - cc;
    }
    double v = weno_rec(vp, vm, ws, ord, c.p.weno_version, bsA);
    if (side == 0) fi[0] = v; else fi[NV - 1] = v;
  }
  // species characteristics 1+lsp
#pragma unroll 1
  for (int k = 0; k < NS; k++) {
    for (int l = 1; l <= wsz; l++) {
      long long q = p + (l - ws) * st;
      double y = FG(wa, q, k + 1);
      double wc = rl[l] * y - yr[k] * Qw[l];
      double gc = rul[l] * y - yr[k] * Qf[l];
      double cc = 0.5 * (gc + ev2 * wc);
      vp[l] = cc; vm[l] = gc - cc;
    }
    fi[1 + k] = weno_rec(vp, vm, ws, ord, c.p.weno_version, bsA);
  }
  // tangential characteristics NS+2, NS+3
#pragma unroll 1
  for (int side = 0; side < 2; side++) {
    double ut = side == 0 ? ut1 : ut2;
    for (int l = 1; l <= wsz; l++) {
      double wc = (side == 0 ? Wt1[l] : Wt2[l]) - ut * sw[l];
      double gc = (side == 0 ? Ft1[l] : Ft2[l]) - ut * sf[l];
      double cc = 0.5 * (gc + ev2 * wc);
      vp[l] = cc; vm[l] = gc - cc;
    }
    fi[NS + 1 + side] = weno_rec(vp, vm, ws, ord, c.p.weno_version, bsB);
  }
  // back projection with the reference's summation order (eigenvectors_*, :415-420)
  const double f0 = fi[0], f4 = fi[NV - 1];
#pragma unroll
  for (int k = 0; k < NS; k++) fh[k] = (yr[k] * f0 + fi[1 + k]) + yr[k] * f4;
  double an = (un - cr) * f0, a1 = ut1 * f0, a2 = ut2 * f0, aE = (hr - un * cr) * f0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    double fk = fi[1 + k];
    an = an + un * fk;
    a1 = a1 + ut1 * fk;
    a2 = a2 + ut2 * fk;
    aE = aE + (b3 - prhoi[k] / b2 * cci) * fk;
  }
  a1 = a1 + fi[NS + 1];
  a2 = a2 + fi[NS + 2];
  aE = aE + ut1 * fi[NS + 1];
  aE = aE + ut2 * fi[NS + 2];
  an = an + (un + cr) * f4;
  a1 = a1 + ut1 * f4;
  a2 = a2 + ut2 * f4;
  aE = aE + (hr + un * cr) * f4;
  fh[NS + DIR] = an;
  fh[NS + T1] = a1;
  fh[NS + T2] = a2;
  fh[NS + 3] = aE;
}

// Component-wise Rusanov WENO face flux (kernels_gpu.F90:671-725).
template <int NS, int DIR>
__device__ __noinline__ void weno_rusanov_flux(const DevCtx &c, const double *__restrict__ wa, long long p, long long st,
                                               double *fh) {
  const DevGrid &g = c.g;
  const int J_U = NS + 1, J_H = NS + 4, J_P = NS + 6, J_C = NS + 7, J_R = NS + 11;
  const int ws = c.p.weno_scheme, wsz = 2 * ws;
  int ord = ws < 1 ? 1 : ws;
  double evmax = -1.0;
  for (int l = 1; l <= wsz; l++) {
    long long q = p + (l - ws) * st;
    double u = FG(wa, q, J_U + DIR), cq = FG(wa, q, J_C);
    evmax = dmax_(dmax_(fabs(u - cq), fabs(u + cq)), evmax);
  }
  const double u0 = c.p.u0, rho0 = c.p.rho0, u02 = u0 * u0;
  const double r2u2 = rho0 * rho0 * u02, r2u4 = r2u2 * u02, r2u4i = 1.0 / r2u4;
  double vp[WMAX + 1], vm[WMAX + 1];
#pragma unroll 1
  for (int m = 0; m < NS + 4; m++) {
    for (int l = 1; l <= wsz; l++) {
      long long q = p + (l - ws) * st;
      double rho = FG(wa, q, J_R), un = FG(wa, q, J_U + DIR);
      double rhou = rho * un, rhoevm = rho * evmax, evm, cc;
      if (m < NS) {
        double yy = FG(wa, q, m + 1);
        evm = rhou * yy;
        cc = 0.5 * (evm + rhoevm * yy);
      } else if (m < NS + 3) {
        int d = m - NS;
        double vd = FG(wa, q, J_U + d);
        evm = (d == DIR) ? vd * rhou + FG(wa, q, J_P) : vd * rhou;
        cc = 0.5 * (evm + rhoevm * vd);
      } else {
        double h = FG(wa, q, J_H), pp = FG(wa, q, J_P);
        evm = h * rhou;
        cc = 0.5 * (evm + evmax * (rho * h - pp));
      }
      vp[l] = cc; vm[l] = evm - cc;
    }
    double bs = m < NS ? 1.0 / r2u2 : (m < NS + 3 ? r2u4i : r2u4i / u02);
    fh[m] = weno_rec(vp, vm, ws, ord, c.p.weno_version, bs);
  }
}

// Hybrid face flux: Ducros test over the WENO stencil, then central or upwind.
template <int NS, int DIR, typename R>
__device__ __forceinline__ void face_flux(const DevCtx &c, const DevCtx *__restrict__ cg,
                                          const double *__restrict__ wa, long long p, long long st, int face, int nmax,
                                          R *fh) {
  const DevGrid &g = c.g;
  const int J_DUC = NS + 9;
  const int ws = c.p.weno_scheme;
  bool shk = false;
  for (int s = -ws + 1; s <= ws; s++) shk |= (FG(wa, p + s * st, J_DUC) > c.p.sensor_threshold);
  if (!shk) {
    bool fz = (face == 0 && c.p.fzf[2 * DIR] == 1) || (face == nmax && c.p.fzf[2 * DIR + 1] == 1);
    central_flux<NS, DIR, R>(c, wa, p, st, fz, fh);
  } else {
    // The out-of-line WENO fluxes take the context by reference and write
    // through a pointer.  They get the device-resident copy cg of the context
    // (the by-value kernel parameter c would otherwise be copied to local
    // memory by every thread) and their own output array (so fh stays in
    // registers on the central path).
    double fw[NS + 4];
    if (c.p.flux_splitting == 1) weno_rusanov_flux<NS, DIR>(*cg, wa, p, st, fw);
    else weno_char_flux<NS, DIR>(*cg, wa, p, st, fw);
#pragma unroll
    for (int m = 0; m < NS + 4; m++) fh[m] = (R)fw[m];
  }
}

// x sweep: the faces nmin-1..nmax of every (j, k) row are numbered as one
// sequence F = row * nf + (f - nmin + 1); CTA b of XB threads computes faces
// (XB - 1) b .. (XB - 1) b + XB - 1
// (one face shared with the next CTA), puts them in shared memory, and the
// threads whose face is not the first of its row form
// fl(i) += (fhat_i - fhat_{i-1}) * dxi/dx -- every thread busy for any nx.
template <int NS, typename R>
__global__ void __launch_bounds__(128, 4) k_euler_x(DevCtx c, const DevCtx *__restrict__ cg,
                                                    const double *__restrict__ wa, double *__restrict__ fl,
                                                    int nmin, int nmax, int overwrite) {
  const DevGrid &g = c.g;
  const int NV = NS + 4;
  constexpr int XB = xsweep_block(NS);
  __shared__ R sf[NV][XB];
  const long long nf = nmax - nmin + 2;
  const long long F = (long long)blockIdx.x * (XB - 1) + threadIdx.x;
  const bool act = F < nf * g.ny * g.nz;
  const long long row = F / nf;
  const int f = nmin - 1 + (int)(F - row * nf);
  const int j = 1 + (int)(row % g.ny), k = 1 + (int)(row / g.ny);
  if (act) {
    R fh[NV];
    long long p = gidx(g, f, j, k);
    face_flux<NS, 0, R>(c, cg, wa, p, 1, f, g.nx, fh);
#pragma unroll
    for (int m = 0; m < NV; m++) sf[m][threadIdx.x] = fh[m];
  }
  __syncthreads();
  if (threadIdx.x >= 1 && act && f >= nmin) {
    const int i = f;
    long long q = fidx(g, i, j, k);
    double met = ldg(g.dcsidx + i - 1);
#pragma unroll
    for (int m = 0; m < NV; m++) {
      double d = (double)((sf[m][threadIdx.x] - sf[m][threadIdx.x - 1]) * (R)met);
      FI(fl, q, m + 1) = overwrite ? d : FI(fl, q, m + 1) + d;
    }
  }
}

// y / z sweeps: a CTA is a tile of YZ_TI consecutive i (one warp, coalesced)
// by YZ_TF consecutive faces of the sweep; every thread computes one face, the
// faces go through shared memory, and rows 1..YZ_TF-1 form the YZ_TF-1 cells
// fl(f) += (fhat_f - fhat_{f-1}) * d(eta)/dy.  One redundant face per tile.
// (YZ_TI, YZ_TF) = (32, 8); (16, 6) for large mechanisms (shared memory)
template <int NS> struct YZTile {
  static constexpr int TI = NS > 20 ? 16 : 32, TF = NS > 20 ? 6 : 8;
};
#define YZ_TI (YZTile<NS>::TI)
#define YZ_TF (YZTile<NS>::TF)
template <int NS, int DIR, typename R>
__global__ void __launch_bounds__(YZ_TI * YZ_TF) k_euler_yz(DevCtx c, const DevCtx *__restrict__ cg,
                                                           const double *__restrict__ wa, double *__restrict__ fl,
                                                           int nmin, int nmax, int overwrite) {
  const DevGrid &g = c.g;
  const int NV = NS + 4;
  __shared__ R sf[NV][YZ_TF][YZ_TI];
  const int tx = threadIdx.x, ty = threadIdx.y;
  int i = blockIdx.x * YZ_TI + tx + 1;
  int tr = blockIdx.y + 1;                 // k for the y sweep, j for the z sweep
  int f = nmin - 1 + blockIdx.z * (YZ_TF - 1) + ty;
  long long st = DIR == 1 ? (long long)g.nxg : (long long)g.nxg * g.nyg;
  int nsw = DIR == 1 ? g.ny : g.nz;
  bool act = i <= g.nx && f <= nmax;
  if (act) {
    R fh[NV];
    long long p = DIR == 1 ? gidx(g, i, f, tr) : gidx(g, i, tr, f);
    face_flux<NS, DIR, R>(c, cg, wa, p, st, f, nsw, fh);
#pragma unroll
    for (int m = 0; m < NV; m++) sf[m][ty][tx] = fh[m];
  }
  __syncthreads();
  if (ty >= 1 && act) {
    const double *met = DIR == 1 ? g.detady : g.dzitdz;
    long long q = DIR == 1 ? fidx(g, i, f, tr) : fidx(g, i, tr, f);
    double mt = ldg(met + f - 1);
#pragma unroll
    for (int m = 0; m < NV; m++) {
      double d = (double)((sf[m][ty][tx] - sf[m][ty - 1][tx]) * (R)mt);
      FI(fl, q, m + 1) = overwrite ? d : FI(fl, q, m + 1) + d;
    }
  }
}

// ---------------------------------------------------------------- staged tiles
// The sweeps above give every face its own thread, which reads its six-point
// stencil from global memory and forms every stencil pair's KEEP factors
// itself: each cell's internal energy is formed by twelve faces and each pair's
// factors by up to three.  The staged sweep below works on a tile of TC cells
// along the sweep by NL lines:
//  1. the tile and its 3-cell halos (Y_k, u, v, w, h, p, rho, Ducros) are copied
//     into shared memory, coalesced along i;
//  2. every staged cell forms its internal energy once;
//  3. every stencil pair (a, a + d), d = 1..ep_order/2, forms its KEEP mass-flux
//     factor and energy term once (the same operations as central_flux);
//  4. every face sums its pairs from shared memory (the faces the Ducros sensor
//     marks take the WENO flux from global memory, as in face_flux);
//  5. every cell forms fl += (fhat_f - fhat_{f-1}) dxi/dx from the staged faces.
// It covers ep_order <= 6 and weno_scheme <= 3 (the 3-cell halo) and ns <= 20
// (shared memory); euler_r dispatches to the per-face sweeps otherwise.
// CTAs per SM the x tile's register budget is sized for: 5 (96 registers; its
// 39 KB of shared memory also admits 5) ran an x sweep of a developed 128^3
// field in 0.585 ms against 0.679 ms at 4 (128 registers), with the same
// results bit for bit.  y and z: 2, where their 91 KB of shared memory also
// sets the limit.  y / z tiles of 8 lines at 4 CTAs per SM (128 registers)
// ran the y and z sweeps of a developed 256^3 field in 2.84 ms against 2.73 ms
// at 16 lines, and in 3.23 ms at 3 CTAs per SM (168 registers), the same bits
#ifndef STX_ETILE_X_MINB
#define STX_ETILE_X_MINB 5
#endif
// lines (consecutive i) per CTA of the y / z tiles, and the CTAs per SM their
// register budget is sized for
#ifndef STX_ETILE_YZ_NL
#define STX_ETILE_YZ_NL 16
#endif
#ifndef STX_ETILE_YZ_MINB
#define STX_ETILE_YZ_MINB 2
#endif
template <int NS, int DIR, bool TMA = false> struct ETile {
  static constexpr int TC = DIR == 0 ? 64 : 16;        // cells per line updated by a CTA
  static constexpr int NL = DIR == 0 ? 2 : STX_ETILE_YZ_NL;   // lines per CTA
  static constexpr int H = 3;                          // halo cells each side
  static constexpr int S = TC + 2 * H;                 // staged cells per line
  static constexpr int NF = TC + 1;                    // faces per line
  static constexpr int NP = TC + 3;                    // pair origins per line and distance
  static constexpr int NVC = NS + 7;                   // staged fields
  static constexpr int NT = TC * NL;                   // threads
  // the cell stage of tensor copies (TMA), whose boxes start at an even x (the
  // 16-byte rule of tensor copies) and land at 128-byte-aligned addresses:
  //   x: per field and line a row of BX = S + 2 cells, at a row stride RS;
  //   y / z: per field a box of S sweep cells x BXI = NL + 2 cells in i (row
  //   stride RSI), the fields VS apart
  static constexpr int BX = S + 2;
  static constexpr int BXI = NL + 2;
  static constexpr int RS = TMA ? ((BX * 8 + 127) / 128) * 16 : S;   // x: row stride of the cell stage
  static constexpr int RSI = TMA ? BXI : NL;                         // y / z: row stride of the cell stage
  static constexpr int VS = DIR == 0 ? NL * RS : (TMA ? ((S * BXI * 8 + 127) / 128) * 16 : S * NL);
  // x sweep: the sweep is the contiguous direction, lines are rows (j, k);
  // y / z sweeps: lines are consecutive i
  __device__ static int sx(int s, int l) { return DIR == 0 ? l * S + s : s * NL + l; }     // per-cell arrays
  __device__ static int cx(int s, int l) { return DIR == 0 ? l * RS + s : s * RSI + l; }   // the cell stage
  __device__ static int px(int a, int l) { return DIR == 0 ? l * NP + a : a * NL + l; }
  __device__ static int fx(int f, int l) { return DIR == 0 ? l * NF + f : f * NL + l; }
};

template <int NS, typename R, bool TMA = false>
__host__ __device__ constexpr size_t etile_smem(int dir) {
  // cells (double) + faces (R) + pair factors (2 x 3 distances, R) + internal energy (R);
  // the TMA stage also takes 128 bytes of alignment slack
  return dir == 0 ? (size_t)ETile<NS, 0, TMA>::NVC * ETile<NS, 0, TMA>::VS * 8 + (TMA ? 128 : 0) +
                        (size_t)(NS + 4) * ETile<NS, 0>::NF * ETile<NS, 0>::NL * sizeof(R) +
                        (size_t)6 * ETile<NS, 0>::NP * ETile<NS, 0>::NL * sizeof(R) +
                        (size_t)ETile<NS, 0>::S * ETile<NS, 0>::NL * sizeof(R)
                  : (size_t)ETile<NS, 1, TMA>::NVC * ETile<NS, 1, TMA>::VS * 8 + (TMA ? 128 : 0) +
                        (size_t)(NS + 4) * ETile<NS, 1>::NF * ETile<NS, 1>::NL * sizeof(R) +
                        (size_t)6 * ETile<NS, 1>::NP * ETile<NS, 1>::NL * sizeof(R) +
                        (size_t)ETile<NS, 1>::S * ETile<NS, 1>::NL * sizeof(R);
}

// ---------------------------------------------------------------- tensor-memory-access staging
// mbarrier and tensor-copy primitives (PTX ISA: mbarrier, cp.async.bulk.tensor).
// Loads only, into this CTA's own shared memory, from this GPU's own memory, and
// never with .multicast::cluster.
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 2-D tile load of the box at (x, y) of the tensor map into dst, completing on bar
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, unsigned long long *bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      ::"r"(smem_u32(dst)), "l"((unsigned long long)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}
// 4-D tile load of the box at (x, y, z, w) of the tensor map into dst, completing on bar
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, unsigned long long *bar, int x, int y,
                                            int z, int w) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], [%2];"
      ::"r"(smem_u32(dst)), "l"((unsigned long long)map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
      : "memory");
}
// bounded wait for phase `phase` of bar: false if it did not complete within the limit
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, uint32_t phase) {
  for (int it = 0; it < (1 << 22); it++)
    if (mbar_try_wait(bar, phase)) return true;
  return false;
}

// staged field v -> w_aux field (1-based)
template <int NS>
__device__ __forceinline__ int etile_field(int v) {
  if (v < NS) return v + 1;
  switch (v - NS) {
    case 0: return NS + 1;    // u
    case 1: return NS + 2;    // v
    case 2: return NS + 3;    // w
    case 3: return NS + 4;    // h
    case 4: return NS + 6;    // p
    case 5: return NS + 11;   // rho
    default: return NS + 9;   // Ducros
  }
}

// TMA: the cell stage is filled by tensor copies (tmap: sweep_tmap) -- per
// staged row in x, per field in y / z -- issued by one thread and completed on
// an mbarrier; cells outside the ghosted box come back as zeros (the copies'
// out-of-bounds fill), as the loads of the plain staging give them.
// Everything after the staging is the same code on the same values.
template <int NS, int DIR, typename R, bool TMA = false>
__global__ void __launch_bounds__(ETile<NS, DIR>::NT, DIR == 0 ? STX_ETILE_X_MINB : STX_ETILE_YZ_MINB)
    k_euler_tile(DevCtx c, const DevCtx *__restrict__ cg, const double *__restrict__ wa, double *__restrict__ fl,
                 int nmin, int nmax, int overwrite, const double *__restrict__ fhw, long long cap,
                 const __grid_constant__ CUtensorMap tmap) {
  using T = ETile<NS, DIR, TMA>;
  constexpr int TC = T::TC, NL = T::NL, S = T::S, NF = T::NF, NP = T::NP, NVC = T::NVC, NT = T::NT;
  constexpr int NV = NS + 4;
  constexpr int vU = NS, vV = NS + 1, vW = NS + 2, vH = NS + 3, vP = NS + 4, vR = NS + 5, vD = NS + 6;
  const DevGrid &g = c.g;
  extern __shared__ __align__(16) unsigned char e_smem[];
  unsigned char *sbase = e_smem;
  if constexpr (TMA) sbase = e_smem + ((128u - (smem_u32(e_smem) & 127u)) & 127u);   // 128-byte aligned rows
  double *sc = (double *)sbase;                           // [NVC][cells]
  R *sf = (R *)(sc + NVC * T::VS);                        // [NV][faces]
  R *sup = sf + NV * NF * NL;                             // [3][pairs] mass-flux factor
  R *spe = sup + 3 * NP * NL;                             // [3][pairs] energy term
  R *see = spe + 3 * NP * NL;                             // [cells] internal energy
  const int t = threadIdx.x;
  const int c0 = nmin + blockIdx.y * TC;                  // first cell of the tile along the sweep
  const int nsw = DIR == 0 ? g.nx : (DIR == 1 ? g.ny : g.nz);
  // line l of this CTA -> (lateral coordinates), active?
  // x: rows r = blockIdx.x * NL + l over (j, k); y: i = blockIdx.x NL + l + 1, k = blockIdx.z + 1;
  // z: i = blockIdx.x NL + l + 1, j = blockIdx.z + 1
  const long long st = DIR == 0 ? 1LL : (DIR == 1 ? (long long)g.nxg : (long long)g.nxg * g.nyg);
  // per line: ghosted index of its cell at sweep coordinate 0 (-1: no such
  // line) and interior index of its cell at sweep coordinate 0, formed once
  // (x: rows r = blockIdx.x NL + l over (j, k); y / z: i = blockIdx.x NL + l + 1
  // with k resp. j = blockIdx.z + 1)
  __shared__ long long s_gb[NL], s_fb[NL];
  __shared__ __align__(8) unsigned long long s_bar;
  if constexpr (TMA) {
    if (t == 0) {
      mbar_init(&s_bar, 1);
      mbar_fence_init();
    }
  }
  if (t < NL) {
    const int l = t;
    long long gb = -1, fb = 0;
    if (DIR == 0) {
      long long r = (long long)blockIdx.x * NL + l;
      if (r < (long long)g.ny * g.nz) {
        int j = 1 + (int)(r % g.ny), k = 1 + (int)(r / g.ny);
        gb = gidx(g, 0, j, k);
        fb = fidx(g, 0, j, k);
      }
    } else {
      int i = blockIdx.x * NL + l + 1;
      if (i <= g.nx) {
        gb = DIR == 1 ? gidx(g, i, 0, blockIdx.z + 1) : gidx(g, i, blockIdx.z + 1, 0);
        fb = DIR == 1 ? fidx(g, i, 0, blockIdx.z + 1) : fidx(g, i, blockIdx.z + 1, 0);
      }
    }
    s_gb[l] = gb;
    s_fb[l] = fb;
  }
  __syncthreads();
  auto line_base = [&](int l, bool &act) -> long long {
    const long long gb = s_gb[l];
    act = gb >= 0;
    return gb;
  };
  // 1. stage the cells c0-3 .. c0+TC+2 of every line (zero outside the ghosted box)
  const double *scb = sc;                                 // staged cell 0 of field 0, line 0
  if constexpr (TMA) {
    if constexpr (DIR == 0) {
      const int xs = c0 - T::H + g.ng - 1;                // ghosted x index (0-based) of staged cell 0
      const int x0 = xs & ~1;                             // an even x: 16 bytes of doubles
      scb = sc + (xs - x0);
      if (t == 0) {
        int nact = 0;
        for (int l = 0; l < NL; l++) nact += s_gb[l] >= 0;
        fence_proxy_async();                              // the previous reads of this stage come first
        mbar_expect_tx(&s_bar, (uint32_t)(nact * NVC * T::BX * 8));
        const long long rows = (long long)g.nyg * g.nzg;
        for (int l = 0; l < NL; l++) {
          const long long gb = s_gb[l];
          if (gb < 0) continue;
          const long long line = (gb - (g.ng - 1)) / g.nxg;   // (j + ng - 1) + nyg (k + ng - 1)
          for (int v = 0; v < NVC; v++)
            tma_load_2d(sc + v * T::VS + l * T::RS, &tmap, &s_bar, x0,
                        (int)((etile_field<NS>(v) - 1) * rows + line));
        }
      }
      for (int e = t; e < NVC * T::VS; e += NT)           // lines outside the grid: zeros
        if (s_gb[(e / T::RS) % NL] < 0) sc[e] = 0.0;
    } else {
      // one box per field: BXI cells in i from an even x by S cells along the
      // sweep (tmap: w_aux as nxg x nyg x nzg x nv_aux); lines past nx stage
      // whatever lies there (the ghosts, or the copies' zero fill) and are
      // never used
      const int xg = blockIdx.x * NL + g.ng;              // ghosted i index (0-based) of line 0
      const int x0 = xg & ~1;
      scb = sc + (xg - x0);
      if (t == 0) {
        fence_proxy_async();
        mbar_expect_tx(&s_bar, (uint32_t)(NVC * T::BXI * S * 8));
        const int ss = c0 - T::H + g.ng - 1;              // ghosted sweep index of staged cell 0
        const int o = blockIdx.z + g.ng;                  // ghosted index of the other lateral direction
        for (int v = 0; v < NVC; v++)
          tma_load_4d(sc + v * T::VS, &tmap, &s_bar, x0, DIR == 1 ? ss : o, DIR == 1 ? o : ss,
                      etile_field<NS>(v) - 1);
      }
    }
    // every thread waits for the copies (bounded); on a time-out the CTA stops
    // together and the status word says so
    const bool ok = __syncthreads_and(mbar_wait_bounded(&s_bar, 0));
    if (!ok) {
      if (t == 0) set_status(c.p, STX_ST_WAIT_TIMEOUT);
      mbar_wait_bounded(&s_bar, 0);                       // the copies in flight, once more
      return;
    }
  } else {
    for (int e = t; e < NVC * S * NL; e += NT) {
      int s, l, v;
      if (DIR == 0) { s = e % S; l = (e / S) % NL; v = e / (S * NL); }
      else { l = e % NL; s = (e / NL) % S; v = e / (S * NL); }
      bool act;
      long long b = line_base(l, act);
      int x = c0 - T::H + s;
      double val = 0.0;
      if (act && x >= 1 - g.ng && x <= nsw + g.ng) val = FG(wa, b + x * st, etile_field<NS>(v));
      sc[v * T::VS + T::cx(s, l)] = val;
    }
  }
  __syncthreads();
  auto ld = [&](int v, int s, int l) -> R { return (R)scb[v * T::VS + T::cx(s, l)]; };
  const int nkeep = c.p.nkeep;
  int lmax = c.p.ep_order / 2;
  if (lmax < 1) lmax = 1;
  // 2. internal energy of every staged cell (central_flux: eei)
  if (nkeep >= 0) {
    for (int e = t; e < S * NL; e += NT) {
      int s = DIR == 0 ? e % S : e / NL, l = DIR == 0 ? e / S : e % NL;
      R rr = ld(vR, s, l), uu = ld(vU, s, l), vv = ld(vV, s, l), ww = ld(vW, s, l);
      see[T::sx(s, l)] = ld(vH, s, l) - ld(vP, s, l) / rr - R(0.5) * (uu * uu + vv * vv + ww * ww);
    }
    __syncthreads();
  }
  // 3. pair factors for origins a = 0..TC+2 and distances d = 1..lmax
  for (int e = t; e < lmax * NP * NL; e += NT) {
    int d = 1 + e / (NP * NL), r = e % (NP * NL);
    int a = DIR == 0 ? r % NP : r / NL, l = DIR == 0 ? r / NP : r % NL;
    int b = a + d;
    R rhoi = ld(vR, a, l), uni = ld(vU + DIR, a, l), rhoip = ld(vR, b, l), unip = ld(vU + DIR, b, l);
    R rhom = rhoi + rhoip, drhof;
    if (nkeep <= 0) {
      drhof = R(1.0);
    } else {
      R drho = R(2.0) * (rhoip - rhoi) / rhom;
      R tt = (R(0.5) * drho) * (R(0.5) * drho), t2 = tt;
      R sumden = R(1.0) + tt / R(3.0);
      for (int n = 2; n <= nkeep; n++) { int n2 = 2 * n; tt = t2 * tt; sumden = sumden + tt / (R(1.0) + n2); }
      drhof = R(1.0) / sumden;
    }
    R up = (uni + unip) * rhom * drhof;
    R pe = R(0.0);
    if (nkeep >= 0) {
      R eei = see[T::sx(a, l)], eeip = see[T::sx(b, l)];
      R eem = eei + eeip, deef;
      if (nkeep == 0) {
        deef = R(1.0);
      } else {
        R dee = R(2.0) * (eeip - eei) / eem;
        R te = (R(0.5) * dee) * (R(0.5) * dee);
        R te2 = te;
        R sde = R(1.0) + te, sne = R(1.0) + te / R(3.0);
        for (int n = 2; n <= nkeep; n++) {
          int n2 = 2 * n;
          te = te2 * te;
          sde = sde + te;
          sne = sne + te / (R(1.0) + n2);
        }
        deef = sne / sde;
      }
      pe = up * eem * deef;
    }
    sup[(d - 1) * NP * NL + T::px(a, l)] = up;
    spe[(d - 1) * NP * NL + T::px(a, l)] = pe;
  }
  __syncthreads();
  // 4. faces c0-1 .. c0+TC-1 (staged position of face f's left cell: f - c0 + 3)
  const int ws = c.p.weno_scheme;
  for (int e = t; e < NF * NL; e += NT) {
    int fr = DIR == 0 ? e % NF : e / NL, l = DIR == 0 ? e / NF : e % NL;
    int f = c0 - 1 + fr;
    bool act;
    long long b = line_base(l, act);
    if (!act || f < nmin - 1 || f > nmax) continue;
    const int q = fr + 2;
    R *fo = sf + T::fx(fr, l);                            // this face's fluxes, stride NF * NL
    bool shk = false;
    for (int s = -ws + 1; s <= ws; s++) shk |= (scb[vD * T::VS + T::cx(q + s, l)] > c.p.sensor_threshold);
    if (!shk) {
      bool fz = (f == 0 && c.p.fzf[2 * DIR] == 1) || (f == nsw && c.p.fzf[2 * DIR + 1] == 1);
#pragma unroll 1
      for (int lsp = 0; lsp < NS; lsp++) {
        R ft1 = R(0.0);
#pragma unroll
        for (int ll = 1; ll <= T::H; ll++) {
          if (ll <= lmax) {
            R uvs1 = R(0.0);
#pragma unroll
            for (int m = 0; m < ll; m++)
              uvs1 = uvs1 + sup[(ll - 1) * NP * NL + T::px(q - m, l)] * (ld(lsp, q - m, l) + ld(lsp, q - m + ll, l));
            ft1 = ft1 + R(c.p.cd1[ll][lmax]) * uvs1;
          }
        }
        fo[lsp * NF * NL] = fz ? R(0.0) : R(0.25) * ft1;
      }
      R ft2 = 0, ft3 = 0, ft4 = 0, ft5 = 0, ft6 = 0;
#pragma unroll
      for (int ll = 1; ll <= T::H; ll++) {
        if (ll > lmax) break;
        R uvs2 = 0, uvs3 = 0, uvs4 = 0, uvs5 = 0, uvs6 = 0, uvs5_i = 0, uvs5_k = 0, uvs5_p = 0;
#pragma unroll
        for (int m = 0; m < ll; m++) {
          const int a = q - m, bb = q - m + ll;
          R uui = ld(vU, a, l), vvi = ld(vV, a, l), wwi = ld(vW, a, l), ppi = ld(vP, a, l);
          R uuip = ld(vU, bb, l), vvip = ld(vV, bb, l), wwip = ld(vW, bb, l), ppip = ld(vP, bb, l);
          R uni = DIR == 0 ? uui : (DIR == 1 ? vvi : wwi);
          R unip = DIR == 0 ? uuip : (DIR == 1 ? vvip : wwip);
          R uv_part = sup[(ll - 1) * NP * NL + T::px(a, l)];
          uvs2 = uvs2 + uv_part * (uui + uuip);
          uvs3 = uvs3 + uv_part * (vvi + vvip);
          uvs4 = uvs4 + uv_part * (wwi + wwip);
          if (nkeep >= 0) {
            uvs5_i = uvs5_i + spe[(ll - 1) * NP * NL + T::px(a, l)];
            uvs5_k = uvs5_k + uv_part * (uui * uuip + vvi * vvip + wwi * wwip);
            uvs5_p = uvs5_p + R(4.0) * (uni * ppip + unip * ppi);
          } else {
            uvs5 = uvs5 + uv_part * (ld(vH, a, l) + ld(vH, bb, l));
          }
          uvs6 = uvs6 + R(2.0) * (ppi + ppip);
        }
        R cl = R(c.p.cd1[ll][lmax]);
        ft2 = ft2 + cl * uvs2;
        ft3 = ft3 + cl * uvs3;
        ft4 = ft4 + cl * uvs4;
        ft5 = ft5 + cl * (nkeep >= 0 ? (uvs5_i + uvs5_k + uvs5_p) : uvs5);
        ft6 = ft6 + cl * uvs6;
      }
      R fm0 = R(0.25) * ft2, fm1 = R(0.25) * ft3, fm2 = R(0.25) * ft4, fh5 = R(0.25) * ft5;
      if (fz) { fm0 = fm1 = fm2 = fh5 = R(0.0); }
      if (DIR == 0) fm0 = fm0 + R(0.5) * ft6;
      if (DIR == 1) fm1 = fm1 + R(0.5) * ft6;
      if (DIR == 2) fm2 = fm2 + R(0.5) * ft6;
      fo[NS * NF * NL] = fm0;
      fo[(NS + 1) * NF * NL] = fm1;
      fo[(NS + 2) * NF * NL] = fm2;
      fo[(NS + 3) * NF * NL] = fh5;
    } else if (fhw) {          // computed by k_weno_list
      long long id;
      if (DIR == 0) id = ((long long)blockIdx.x * NL + l) * (nmax - nmin + 2) + (f - nmin + 1);
      else id = ((long long)(f - nmin + 1) * (DIR == 1 ? g.nz : g.ny) + blockIdx.z) * g.nx + (blockIdx.x * NL + l);
#pragma unroll
      for (int m = 0; m < NV; m++) fo[m * NF * NL] = (R)fhw[m * cap + id];
    } else {
      double fw[NV];
      long long p = b + (long long)f * st;
      if (c.p.flux_splitting == 1) weno_rusanov_flux<NS, DIR>(*cg, wa, p, st, fw);
      else weno_char_flux<NS, DIR>(*cg, wa, p, st, fw);
#pragma unroll
      for (int m = 0; m < NV; m++) fo[m * NF * NL] = (R)fw[m];
    }
  }
  __syncthreads();
  // 5. divergence into fl for the cells c0 .. c0+TC-1
  {
    int sr = DIR == 0 ? t % TC : t / NL, l = DIR == 0 ? t / TC : t % NL;
    int i = c0 + sr;
    bool act;
    line_base(l, act);
    if (act && i <= nmax) {
      const long long fst = DIR == 0 ? 1LL : (DIR == 1 ? (long long)g.nx : (long long)g.nx * g.ny);
      const long long qf = s_fb[l] + (long long)i * fst;
      const double *met = DIR == 0 ? g.dcsidx : (DIR == 1 ? g.detady : g.dzitdz);
      double mt = ldg(met + i - 1);
#pragma unroll
      for (int m = 0; m < NV; m++) {
        double d = (double)((sf[m * NF * NL + T::fx(sr + 1, l)] - sf[m * NF * NL + T::fx(sr, l)]) * (R)mt);
        FI(fl, qf, m + 1) = overwrite ? d : FI(fl, qf, m + 1) + d;
      }
    }
  }
}

// ---------------------------------------------------------------- listed WENO faces
// The Ducros sensor marks a minority of the faces of a turbulent field, spread
// over the grid; computed in line, every warp holding one marked face runs the
// characteristic WENO flux with most of its lanes idle.  Instead, k_weno_mark
// lists the marked faces (warp-aggregated appends), k_weno_list computes their
// fluxes with every lane busy into a face-indexed buffer, and the staged sweep
// reads them there.  Each face's flux is the same function of the same inputs,
// so the result does not depend on the list's order.
//
// Face ids of a sweep over cells nmin..nmax (faces nmin-1..nmax, fr = f - nmin + 1,
// nf = nmax - nmin + 2): x: row (j, k) * nf + fr; y: (fr * nz + k - 1) * nx + i - 1;
// z: (fr * ny + j - 1) * nx + i - 1 (i fastest: coalesced along the grid).
template <int DIR>
__device__ __forceinline__ void weno_face(const DevGrid &g, long long id, int nmin, int nmax, long long &p, int &f) {
  if (DIR == 0) {
    long long nf = nmax - nmin + 2, r = id / nf;
    f = nmin - 1 + (int)(id - r * nf);
    p = gidx(g, f, 1 + (int)(r % g.ny), 1 + (int)(r / g.ny));
  } else {
    int i = 1 + (int)(id % g.nx);
    long long t = id / g.nx;
    int no = DIR == 1 ? g.nz : g.ny;
    int o = 1 + (int)(t % no);
    f = nmin - 1 + (int)(t / no);
    p = DIR == 1 ? gidx(g, i, f, o) : gidx(g, i, o, f);
  }
}

template <int NS, int DIR>
__global__ void __launch_bounds__(256) k_weno_mark(DevCtx c, const double *__restrict__ wa, int nmin, int nmax,
                                                   long long total, unsigned int *count, int *list) {
  const DevGrid &g = c.g;
  const int J_DUC = NS + 9, ws = c.p.weno_scheme;
  const long long st = DIR == 0 ? 1LL : (DIR == 1 ? (long long)g.nxg : (long long)g.nxg * g.nyg);
  const int lane = threadIdx.x & 31;
  for (long long base = (long long)blockIdx.x * blockDim.x; base < total; base += (long long)gridDim.x * blockDim.x) {
    long long id = base + threadIdx.x;
    bool shk = false;
    if (id < total) {
      long long p;
      int f;
      weno_face<DIR>(g, id, nmin, nmax, p, f);
      for (int q = -ws + 1; q <= ws; q++) shk |= (FG(wa, p + q * st, J_DUC) > c.p.sensor_threshold);
    }
    unsigned m = __ballot_sync(0xffffffffu, shk);
    if (m) {
      unsigned b0 = 0;
      if (lane == 0) b0 = atomicAdd(count, (unsigned)__popc(m));
      b0 = __shfl_sync(0xffffffffu, b0, 0);
      if (shk) list[b0 + __popc(m & ((1u << lane) - 1u))] = (int)id;
    }
  }
}

// CTAs per SM the listed-WENO pass's register budget is sized for: 4 (128
// registers) ran a y sweep of a developed 128^3 field (mark, list and tile) in
// 0.921 ms, 6 (80 registers) in 0.939 ms and 8 (64) in 0.945 ms, with the same
// results bit for bit
#ifndef STX_WLIST_MINB
#define STX_WLIST_MINB 4
#endif
template <int NS, int DIR>
__global__ void __launch_bounds__(128, STX_WLIST_MINB) k_weno_list(DevCtx c, const DevCtx *__restrict__ cg,
                                                      const double *__restrict__ wa, int nmin, int nmax,
                                                      const unsigned int *__restrict__ count,
                                                      const int *__restrict__ list, double *__restrict__ fh,
                                                      long long cap) {
  const DevGrid &g = c.g;
  const long long st = DIR == 0 ? 1LL : (DIR == 1 ? (long long)g.nxg : (long long)g.nxg * g.nyg);
  const long long n = *count;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    long long id = list[q], p;
    int f;
    weno_face<DIR>(g, id, nmin, nmax, p, f);
    double fw[NS + 4];
    if (c.p.flux_splitting == 1) weno_rusanov_flux<NS, DIR>(*cg, wa, p, st, fw);
    else weno_char_flux<NS, DIR>(*cg, wa, p, st, fw);
#pragma unroll
    for (int m = 0; m < NS + 4; m++) fh[m * cap + id] = fw[m];
  }
}

long long weno_scratch_faces(const DevGrid &g) {
  long long a = (long long)(g.nx + 1) * g.ny * g.nz, b = (long long)g.nx * (g.ny + 1) * g.nz,
            d = (long long)g.nx * g.ny * (g.nz + 1);
  long long m = a > b ? a : b;
  return m > d ? m : d;
}

// The staged sweeps' tensor maps over w_aux, encoded through the driver's
// entry point and cached per (pointer, grid, direction):
//   x: 2-D, nxg doubles per row, nyg nzg nv_aux rows; box: one staged row of
//      ETile::BX doubles;
//   y / z: 4-D, nxg x nyg x nzg x nv_aux; box: ETile::BXI doubles in i by
//      ETile::S cells along the sweep (one field).
// No map -- false -- when the layout breaks a rule of tensor copies (a row
// stride that is not a multiple of 16 bytes, i.e. odd nxg; a base that is not
// 16-byte aligned; more rows than a 32-bit coordinate) or the entry point is
// missing: the sweep then stages with plain loads.  STX_TMA=0 turns the tensor
// copies off.
static bool sweep_tmap(int dir, const DevGrid &g, int nv_aux, const double *wa, CUtensorMap *out) {
  static std::mutex mu;
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  static bool tried = false, off = false;
  static std::map<std::tuple<uintptr_t, int, int, int, int, int>, CUtensorMap> cache;
  const long long rows = (long long)g.nyg * g.nzg * nv_aux;
  if ((g.nxg & 1) || (((uintptr_t)wa) & 15) || rows >= 0x7fffffffLL) return false;
  std::lock_guard<std::mutex> lk(mu);
  if (!tried) {
    tried = true;
    const char *env = std::getenv("STX_TMA");
    off = env && std::strcmp(env, "0") == 0;
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (!off && cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  if (off || !encode) return false;
  auto key = std::make_tuple((uintptr_t)wa, g.nxg, g.nyg, g.nzg, nv_aux, dir);
  auto it = cache.find(key);
  if (it != cache.end()) {
    *out = it->second;
    return true;
  }
  CUtensorMap m;
  CUresult r;
  if (dir == 0) {
    const cuuint64_t dims[2] = {(cuuint64_t)g.nxg, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)g.nxg * sizeof(double)};
    const cuuint32_t box[2] = {(cuuint32_t)ETile<9, 0, true>::BX, 1};
    const cuuint32_t estr[2] = {1, 1};
    r = encode(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, (void *)wa, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  } else {
    const cuuint64_t dims[4] = {(cuuint64_t)g.nxg, (cuuint64_t)g.nyg, (cuuint64_t)g.nzg, (cuuint64_t)nv_aux};
    const cuuint64_t strides[3] = {(cuuint64_t)g.nxg * sizeof(double), (cuuint64_t)g.nxg * g.nyg * sizeof(double),
                                   (cuuint64_t)g.npg * sizeof(double)};
    const cuuint32_t bi = (cuuint32_t)ETile<9, 1, true>::BXI, bs = (cuuint32_t)ETile<9, 1, true>::S;
    const cuuint32_t box[4] = {bi, dir == 1 ? bs : 1u, dir == 1 ? 1u : bs, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    r = encode(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, (void *)wa, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  }
  if (r != CUDA_SUCCESS) return false;
  if (cache.size() > 64) cache.clear();
  cache[key] = m;
  *out = m;
  return true;
}

template <int NS, int DIR, typename R>
static int euler_tile_launch(const DevCtx &c, const DevCtx *cg, cudaStream_t s, const double *wa, double *fl,
                             int nmin, int nmax, int ow, const WenoScratch *wsc) {
  using T = ETile<NS, DIR>;
  const DevGrid &g = c.g;
  // listed WENO faces where the scratch holds the sweep's faces
  const long long lines = DIR == 0 ? (long long)g.ny * g.nz : (long long)g.nx * (DIR == 1 ? g.nz : g.ny);
  const long long total = (long long)(nmax - nmin + 2) * lines;
  const double *fhw = nullptr;
  long long cap = 0;
  if (wsc && wsc->cap >= total && total < 0x7fffffffLL) {
    int dev = 0, nsm = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    STX_CUDA_TRY(cudaMemsetAsync(wsc->count, 0, sizeof(unsigned int), s));
    long long nb = (total + 255) / 256;
    if (nb > (long long)nsm * 16) nb = (long long)nsm * 16;
    k_weno_mark<NS, DIR><<<(unsigned)nb, 256, 0, s>>>(c, wa, nmin, nmax, total, wsc->count, wsc->list);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)k_weno_list<NS, DIR>, 128, 0);
    k_weno_list<NS, DIR><<<nsm * (per < 1 ? 1 : per), 128, 0, s>>>(c, cg, wa, nmin, nmax, wsc->count, wsc->list,
                                                                    wsc->fh, wsc->cap);
    STX_CUDA_TRY(cudaGetLastError());
    fhw = wsc->fh;
    cap = wsc->cap;
  }
  constexpr size_t smem = etile_smem<NS, R>(DIR);   // opted in by launch_euler_setup
  long long tiles = (nmax - nmin + 1 + T::TC - 1) / T::TC;
  long long lgrp = DIR == 0 ? ((long long)g.ny * g.nz + T::NL - 1) / T::NL : (g.nx + T::NL - 1) / T::NL;
  int other = DIR == 0 ? 1 : (DIR == 1 ? g.nz : g.ny);
  if (lgrp > 0x7fffffffLL || tiles > 65535 || other > 65535) return STX_E_INVALID;
  // sweep tiles in gridDim.y: the tiles that share halos run close together
  dim3 grid((unsigned)lgrp, (unsigned)tiles, (unsigned)other);
  CUtensorMap tm;
  std::memset(&tm, 0, sizeof(tm));
  if (sweep_tmap(DIR, g, c.p.nv_aux, wa, &tm))
    k_euler_tile<NS, DIR, R, true><<<grid, T::NT, etile_smem<NS, R, true>(DIR), s>>>(c, cg, wa, fl, nmin, nmax, ow,
                                                                                     fhw, cap, tm);
  else
    k_euler_tile<NS, DIR, R><<<grid, T::NT, smem, s>>>(c, cg, wa, fl, nmin, nmax, ow, fhw, cap, tm);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

template <int NS, typename R>
static int euler_r(const DevCtx &c, const DevCtx *cg, cudaStream_t s, int dir, const double *wa, double *fl, int nmin,
                   int nmax, int ow, const WenoScratch *wsc) {
  const DevGrid &g = c.g;
  if (nmax - nmin < 0) return STX_OK;
  if (2 * c.p.weno_scheme > WMAX) return STX_E_UNSUPPORTED;
  // staged tiles where they apply and the context selects them (the default)
  if (NS <= 14 && c.p.ep_order / 2 <= 3 && c.p.weno_scheme <= 3 && g.ng >= 3 && c.p.sweep_kind[dir] == 0) {
    if constexpr (NS <= 14) {
      if (dir == 0) return euler_tile_launch<NS, 0, R>(c, cg, s, wa, fl, nmin, nmax, ow, wsc);
      if (dir == 1) return euler_tile_launch<NS, 1, R>(c, cg, s, wa, fl, nmin, nmax, ow, wsc);
      return euler_tile_launch<NS, 2, R>(c, cg, s, wa, fl, nmin, nmax, ow, wsc);
    }
  }
  if (dir == 0) {
    long long nface = (long long)(nmax - nmin + 2) * g.ny * g.nz;
    constexpr int XB = xsweep_block(NS);
    long long nb = (nface - 1 + XB - 2) / (XB - 1);   // CTA b covers faces (XB-1) b .. (XB-1) b + XB-1
    if (nb > 0x7fffffffLL) return STX_E_INVALID;
    k_euler_x<NS, R><<<(unsigned)nb, XB, 0, s>>>(c, cg, wa, fl, nmin, nmax, ow);
  } else {
    int ncell = nmax - nmin + 1;
    dim3 grid((g.nx + YZ_TI - 1) / YZ_TI, dir == 1 ? g.nz : g.ny, (ncell + YZ_TF - 2) / (YZ_TF - 1));
    dim3 block(YZ_TI, YZ_TF);
    if (dir == 1) k_euler_yz<NS, 1, R><<<grid, block, 0, s>>>(c, cg, wa, fl, nmin, nmax, ow);
    else k_euler_yz<NS, 2, R><<<grid, block, 0, s>>>(c, cg, wa, fl, nmin, nmax, ow);
  }
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

// the plain form computes the central faces in FP64, the mixed form in FP32
template <int NS>
static int euler_t(const DevCtx &c, const DevCtx *cg, cudaStream_t s, int dir, const double *wa, double *fl, int nmin,
                   int nmax, int ow, const WenoScratch *wsc) {
  return c.p.mixed ? euler_r<NS, float>(c, cg, s, dir, wa, fl, nmin, nmax, ow, wsc)
                   : euler_r<NS, double>(c, cg, s, dir, wa, fl, nmin, nmax, ow, wsc);
}

// the staged sweeps' shared memory exceeds the 48 KB default: opt in once per
// instantiation, outside any stream capture (at context creation)
template <int NS>
static int euler_setup_t() {
  if constexpr (NS <= 14) {
    STX_CUDA_TRY(cudaFuncSetAttribute(k_euler_tile<NS, 0, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)etile_smem<NS, double>(0)));
    STX_CUDA_TRY(cudaFuncSetAttribute(k_euler_tile<NS, 1, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)etile_smem<NS, double>(1)));
    STX_CUDA_TRY(cudaFuncSetAttribute(k_euler_tile<NS, 2, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)etile_smem<NS, double>(2)));
    STX_CUDA_TRY(cudaFuncSetAttribute(k_euler_tile<NS, 0, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)etile_smem<NS, float>(0)));
    STX_CUDA_TRY(cudaFuncSetAttribute(k_euler_tile<NS, 0, double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)etile_smem<NS, double, true>(0)));
    STX_CUDA_TRY(cudaFuncSetAttribute(k_euler_tile<NS, 0, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)etile_smem<NS, float, true>(0)));
    STX_CUDA_TRY(cudaFuncSetAttribute(k_euler_tile<NS, 1, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)etile_smem<NS, float>(1)));
    STX_CUDA_TRY(cudaFuncSetAttribute(k_euler_tile<NS, 2, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)etile_smem<NS, float>(2)));
    STX_CUDA_TRY(cudaFuncSetAttribute(k_euler_tile<NS, 1, double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)etile_smem<NS, double, true>(1)));
    STX_CUDA_TRY(cudaFuncSetAttribute(k_euler_tile<NS, 2, double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)etile_smem<NS, double, true>(2)));
    STX_CUDA_TRY(cudaFuncSetAttribute(k_euler_tile<NS, 1, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)etile_smem<NS, float, true>(1)));
    STX_CUDA_TRY(cudaFuncSetAttribute(k_euler_tile<NS, 2, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)etile_smem<NS, float, true>(2)));
  }
  return STX_OK;
}

// once per device and species count: the attribute stays with the function for
// the life of the process, and setting it again is not free while other work
// runs (contexts are created while a server's solves are in flight)
int launch_euler_setup(int ns) {
  static std::mutex mu;
  static std::set<std::pair<int, int>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({dev, ns})) return STX_OK;
  int rc = STX_E_UNSUPPORTED;
  switch (ns) {
#define X(N) case N: rc = euler_setup_t<N>(); break;
    STX_FOR_NS(X)
#undef X
    default: break;
  }
  if (rc == STX_OK) done.insert({dev, ns});
  return rc;
}

int launch_euler(const DevCtx &c, const DevCtx *cg, cudaStream_t s, int dir, const double *wa, double *fl, int nmin,
                 int nmax, int ow, const WenoScratch *wsc) {
  switch (c.t.ns) {
#define X(N) case N: return euler_t<N>(c, cg, s, dir, wa, fl, nmin, nmax, ow, wsc);
    STX_FOR_NS(X)
#undef X
    default: return STX_E_UNSUPPORTED;
  }
}
