// stx_aux.cu -- primitive/transport recovery, Ducros sensor, ghost fills,
// RK bookkeeping and the CFL reduction (sm_100a).
//
// These kernels are HBM-bound stencils or point-wise maps over the reference's
// SoA fields; each thread owns one point and every field is read and written
// once with unit-stride (i-fastest) coalesced accesses.
#include "stx_kernels.cuh"

// CTAs per SM the eval_aux register budget is sized for: 8 (64 registers, some
// spilled) ran compute_aux on a developed 128^3 field in 1.09 ms against 1.48 ms
// unconstrained (154 registers), 1.22 ms at 4 and 1.14 ms at 6, with the same
// results bit for bit
#ifndef STX_AUX_MINB
#define STX_AUX_MINB 8
#endif

// ============================================================== eval_aux
// eval_aux_cuf (kernels_gpu.F90:6154-6308).  Differences in arithmetic order
// from the reference: the Wilke factor sqrt(mu_m/mu_l) is formed as
// sqrt(mu_m)*(1/sqrt(mu_l)) and the constant pair factors 1/sqrt(1+W_l/W_m),
// (W_m/W_l)^0.25 come from a host table; both change results only at rounding
// level.  The species clip is stored only where it changes w.
// The Wilke and Bird loops over the first species index stay rolled (the inner
// loops are unrolled): unrolled in both indices the body outgrew the
// instruction cache, and instruction fetch was the kernel's first stall; rolled,
// a 256^3 call took 8.33 ms against 9.31 ms, with the same results bit for bit.
template <int NS, typename R>
__global__ void __launch_bounds__(128, STX_AUX_MINB) k_eval_aux(DevCtx c, double *__restrict__ w, double *__restrict__ wa,
                                                  int i0, int j0, int k0, int ni, int nj, int nk) {
  const DevGrid &g = c.g;
  const DevTab &t = c.t;
  long long n = (long long)ni * nj * nk;
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= n) return;
  int i = i0 + (int)(tid % ni);
  long long r = tid / ni;
  int j = j0 + (int)(r % nj);
  int k = k0 + (int)(r / nj);
  long long p = gidx(g, i, j, k);
  const int J_U = NS + 1, J_V = NS + 2, J_W = NS + 3, J_H = NS + 4, J_T = NS + 5, J_P = NS + 6, J_C = NS + 7;
  const int J_MU = NS + 8, J_R = NS + 11, J_Z = NS + 12, J_K = NS + 13;
  double Y[NS], rw[NS];
#pragma unroll
  for (int k2 = 0; k2 < NS; k2++) {
    double v = FG(w, p, k2 + 1);
    double vc = v > 0.0 ? v : 0.0;   // max(w, 0); NaN -> 0 as the oracle's max
    if (__double_as_longlong(vc) != __double_as_longlong(v)) FG(w, p, k2 + 1) = vc;
    rw[k2] = vc;
  }
  double rho = rw[0];
#pragma unroll
  for (int k2 = 1; k2 < NS; k2++) rho = rho + rw[k2];
  double ri = 1.0 / rho;
#pragma unroll
  for (int k2 = 0; k2 < NS; k2++) { Y[k2] = rw[k2] * ri; FG(wa, p, k2 + 1) = Y[k2]; }
  double rhou = FG(w, p, NS + 1), rhov = FG(w, p, NS + 2), rhow = FG(w, p, NS + 3), rhoe = FG(w, p, NS + 4);
  double uu = rhou * ri, vv = rhov * ri, ww = rhow * ri;
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double ee = rhoe * ri - qq;
  double tt = temp_from_e<NS>(t, c.p, ee, FG(wa, p, J_T), Y);
  double rm = ldg(t.rgas) * Y[0];
#pragma unroll
  for (int k2 = 1; k2 < NS; k2++) rm = rm + ldg(t.rgas + k2) * Y[k2];
  double cploc = mix_cp<NS>(t, tt, Y);
  double gamloc = cploc / (cploc - rm);
  double pp = rho * tt * rm;
  double cc = sqrt(gamloc * pp * ri);
  FG(wa, p, J_R) = rho;
  FG(wa, p, J_U) = uu;
  FG(wa, p, J_V) = vv;
  FG(wa, p, J_W) = ww;
  FG(wa, p, J_H) = (rhoe + pp) * ri;
  FG(wa, p, J_T) = tt;
  FG(wa, p, J_P) = pp;
  FG(wa, p, J_C) = cc;
  if (t.n_eoi != 1) {
    double Beta = 0.0;
    for (int le = 1; le <= t.n_eoi; le++) {
      double yatm = 0.0;
#pragma unroll
      for (int k2 = 0; k2 < NS; k2++)
        if (Y[k2] > 1e-14)
          yatm = yatm + t.nainsp[(long long)(le - 1) * NS + k2] * ldg(t.aw_eoi + le - 1) * Y[k2] * ldg(t.mwinv + k2);
      Beta = Beta + ldg(t.coeff_eoi + le - 1) * yatm / ldg(t.aw_eoi + le - 1);
    }
    FG(wa, p, J_Z) = (Beta - ldg(t.beta0 + 1)) / (ldg(t.beta0) - ldg(t.beta0 + 1));
  } else {
    FG(wa, p, J_Z) = 0.5;
  }
  int itt;
  double dtt;
  table_pos(t, tt, itt, dtt);
  const double *v0 = t.visc_r + (long long)(itt - 1) * NS, *v1 = v0 + NS;
  const double *l0 = t.lam_r + (long long)(itt - 1) * NS, *l1 = l0 + NS;
  R mwmixt = (R)(t.Ru / rm);
  R X[NS];
#pragma unroll
  for (int k2 = 0; k2 < NS; k2++) X[k2] = (R)Y[k2] * mwmixt * (R)ldg(t.mwinv + k2);
  // Mathur
  R k_cond = R(0.0), k_cond2 = R(0.0);
#pragma unroll
  for (int k2 = 0; k2 < NS; k2++) {
    R a = (R)ldg(l0 + k2);
    R klsp = a + ((R)ldg(l1 + k2) - a) * (R)dtt;
    k_cond = k_cond + X[k2] * klsp;
    k_cond2 = k_cond2 + X[k2] / klsp;
  }
  k_cond = R(0.5) * (k_cond + R(1.0) / k_cond2);
  // Wilke
  R muk[NS], smu[NS];
#pragma unroll
  for (int k2 = 0; k2 < NS; k2++) {
    R a = (R)ldg(v0 + k2);
    muk[k2] = a + ((R)ldg(v1 + k2) - a) * (R)dtt;
    smu[k2] = sqrt(muk[k2]);
  }
  R mu = R(0.0);
#pragma unroll 1
  for (int l = 0; l < NS; l++) {
    R isl = R(1.0) / smu[l];
    R mu_den = R(0.0);
#pragma unroll
    for (int m = 0; m < NS; m++) {
      R t1 = R(1.0) + (smu[m] * isl) * (R)ldg(t.wk_b + l * NS + m);
      R phi_lm = (R)ldg(t.wk_a + l * NS + m) * (t1 * t1);
      mu_den = mu_den + (R)Y[m] * phi_lm * (R)ldg(t.mwinv + m);
    }
    mu = mu + muk[l] * (R)Y[l] * (R)ldg(t.mwinv + l) / mu_den;
  }
  mu = (R)sqrt(8.0) * mu;
  FG(wa, p, J_MU) = (double)mu;
  FG(wa, p, J_K) = (double)k_cond;
  // Bird
  const double *d0 = t.diff_r + (long long)(itt - 1) * NS * NS, *d1 = d0 + NS * NS;
#pragma unroll 1
  for (int l = 0; l < NS; l++) {
    R diff_den = R(0.0);
#pragma unroll
    for (int m = 0; m < NS; m++) {
      if (m != l) {
        R a = (R)ldg(d0 + l * NS + m);
        R dij = a + ((R)ldg(d1 + l * NS + m) - a) * (R)dtt;
        diff_den = diff_den + X[m] / dij;
      }
    }
    FG(wa, p, J_K + 1 + l) = diff_den > R(1.0e-15) ? (double)((R)(1.0 - Y[l]) / diff_den) * c.p.p0 / pp * rho : 0.0;
  }
}

// ============================================================== eval_aux2
// eval_aux2_cuf (kernels_gpu.F90:6310-6382)
__global__ void __launch_bounds__(256) k_eval_aux2(DevCtx c, double *__restrict__ wa, int ns) {
  const DevGrid &g = c.g;
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= g.npi) return;
  int i = 1 + (int)(tid % g.nx);
  long long r = tid / g.nx;
  int j = 1 + (int)(r % g.ny);
  int k = 1 + (int)(r / g.ny);
  long long p = gidx(g, i, j, k);
  const int J_U = ns + 1, J_V = ns + 2, J_W = ns + 3, J_DUC = ns + 9, J_DIV = ns + 10;
  int lmax = c.p.visc_order / 2;
  long long sx = 1, sy = g.nxg, sz = (long long)g.nxg * g.nyg;
  double ux = 0, vx = 0, wx = 0, uy = 0, vy = 0, wy = 0, uz = 0, vz = 0, wz = 0;
  for (int l = 1; l <= lmax; l++) {
    double ccl = c.p.cd1[l][lmax];
    ux = ux + ccl * (FG(wa, p + l * sx, J_U) - FG(wa, p - l * sx, J_U));
    vx = vx + ccl * (FG(wa, p + l * sx, J_V) - FG(wa, p - l * sx, J_V));
    wx = wx + ccl * (FG(wa, p + l * sx, J_W) - FG(wa, p - l * sx, J_W));
    uy = uy + ccl * (FG(wa, p + l * sy, J_U) - FG(wa, p - l * sy, J_U));
    vy = vy + ccl * (FG(wa, p + l * sy, J_V) - FG(wa, p - l * sy, J_V));
    wy = wy + ccl * (FG(wa, p + l * sy, J_W) - FG(wa, p - l * sy, J_W));
    uz = uz + ccl * (FG(wa, p + l * sz, J_U) - FG(wa, p - l * sz, J_U));
    vz = vz + ccl * (FG(wa, p + l * sz, J_V) - FG(wa, p - l * sz, J_V));
    wz = wz + ccl * (FG(wa, p + l * sz, J_W) - FG(wa, p - l * sz, J_W));
  }
  double dx = ldg(g.dcsidx + i - 1), dy = ldg(g.detady + j - 1), dz = ldg(g.dzitdz + k - 1);
  ux = ux * dx; vx = vx * dx; wx = wx * dx;
  uy = uy * dy; vy = vy * dy; wy = wy * dy;
  uz = uz * dz; vz = vz * dz; wz = wz * dz;
  double div = ux + vy + wz;
  double div3l = div / 3.0;
  double ox = wy - vz, oy = uz - wx, oz = vx - uy;
  double omod2 = ox * ox + oy * oy + oz * oz;
  double s = -div / sqrt(omod2 + div * div + c.p.eps_sensor);
  if (c.p.sensor_type == 0) {
    FG(wa, p, J_DUC) = s * s;
  } else {
    double q = s > 0.0 ? s : 0.0;
    FG(wa, p, J_DUC) = q * q;
  }
  FG(wa, p, J_DIV) = div3l;
}

// ============================================================== ghost fills
// bcextr_var_cuf (kernels_gpu.F90:5147-5207): all six faces in one launch;
// sources are interior points, destinations ghosts, so faces are independent.
__global__ void k_bcextr_var(DevCtx c, double *__restrict__ v) {
  const DevGrid &g = c.g;
  long long nxf = (long long)g.ny * g.nz, nyf = (long long)g.nx * g.nz, nzf = (long long)g.nx * g.ny;
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int face;
  long long q;
  if (tid < 2 * nxf) { face = (int)(tid / nxf); q = tid % nxf; }
  else if (tid < 2 * nxf + 2 * nyf) { tid -= 2 * nxf; face = 2 + (int)(tid / nyf); q = tid % nyf; }
  else if (tid < 2 * nxf + 2 * nyf + 2 * nzf) { tid -= 2 * nxf + 2 * nyf; face = 4 + (int)(tid / nzf); q = tid % nzf; }
  else return;
  for (int l = 1; l <= g.ng; l++) {
    if (face == 0) { int j = 1 + (int)(q % g.ny), k = 1 + (int)(q / g.ny); v[gidx(g, 1 - l, j, k)] = v[gidx(g, 1, j, k)]; }
    if (face == 1) { int j = 1 + (int)(q % g.ny), k = 1 + (int)(q / g.ny); v[gidx(g, g.nx + l, j, k)] = v[gidx(g, g.nx, j, k)]; }
    if (face == 2) { int i = 1 + (int)(q % g.nx), k = 1 + (int)(q / g.nx); v[gidx(g, i, 1 - l, k)] = v[gidx(g, i, 1, k)]; }
    if (face == 3) { int i = 1 + (int)(q % g.nx), k = 1 + (int)(q / g.nx); v[gidx(g, i, g.ny + l, k)] = v[gidx(g, i, g.ny, k)]; }
    if (face == 4) { int i = 1 + (int)(q % g.nx), j = 1 + (int)(q / g.nx); v[gidx(g, i, j, 1 - l)] = v[gidx(g, i, j, 1)]; }
    if (face == 5) { int i = 1 + (int)(q % g.nx), j = 1 + (int)(q / g.nx); v[gidx(g, i, j, g.nz + l)] = v[gidx(g, i, j, g.nz)]; }
  }
}

// Periodic self-exchange on one GPU, the single-rank case of base_gpu%bcswap
// (base_gpu.F90:1132-1196, :155-207, :297-383).  One thread per (direction,
// transverse point, variable) stages the 2*ng source values in registers before
// writing, which reproduces the reference's pack-then-unpack order even when
// the extent is smaller than ng; directions read and write disjoint sets.
#define STX_MAXNG 4
__global__ void k_bcswap(DevCtx c, double *__restrict__ f, int nvar, int px, int py, int pz) {
  const DevGrid &g = c.g;
  long long nxf = px ? (long long)g.ny * g.nz : 0, nyf = py ? (long long)g.nx * g.nz : 0,
            nzf = pz ? (long long)g.nx * g.ny : 0;
  long long per = nxf + nyf + nzf;
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= per * nvar) return;
  int m = 1 + (int)(tid / per);
  long long q = tid % per;
  int ng = g.ng;
  double lo[STX_MAXNG], hi[STX_MAXNG];
  if (q < nxf) {
    int j = 1 + (int)(q % g.ny), k = 1 + (int)(q / g.ny);
    for (int i = 1; i <= ng; i++) { lo[i - 1] = FG(f, gidx(g, i, j, k), m); hi[i - 1] = FG(f, gidx(g, g.nx - ng + i, j, k), m); }
    for (int i = 1; i <= ng; i++) { FG(f, gidx(g, i - ng, j, k), m) = hi[i - 1]; FG(f, gidx(g, g.nx + i, j, k), m) = lo[i - 1]; }
  } else if (q < nxf + nyf) {
    q -= nxf;
    int i = 1 + (int)(q % g.nx), k = 1 + (int)(q / g.nx);
    for (int j = 1; j <= ng; j++) { lo[j - 1] = FG(f, gidx(g, i, j, k), m); hi[j - 1] = FG(f, gidx(g, i, g.ny - ng + j, k), m); }
    for (int j = 1; j <= ng; j++) { FG(f, gidx(g, i, j - ng, k), m) = hi[j - 1]; FG(f, gidx(g, i, g.ny + j, k), m) = lo[j - 1]; }
  } else {
    q -= nxf + nyf;
    int i = 1 + (int)(q % g.nx), j = 1 + (int)(q / g.nx);
    for (int k = 1; k <= ng; k++) { lo[k - 1] = FG(f, gidx(g, i, j, k), m); hi[k - 1] = FG(f, gidx(g, i, j, g.nz - ng + k), m); }
    for (int k = 1; k <= ng; k++) { FG(f, gidx(g, i, j, k - ng), m) = hi[k - 1]; FG(f, gidx(g, i, j, g.nz + k), m) = lo[k - 1]; }
  }
}

// update_ghost face kernels without thermodynamics, one thread per (variable,
// boundary point), all ng ghost layers: bcfree_cuf (kernels_gpu.F90:5073, left
// side), bcextr_cuf (:5209), bcsym_cuf (:5395, y sides: the normal velocity of
// the first / last row set to zero, ghosts mirrored about row 1 / row ny with
// the normal momentum reversed), bcoutopenfoam_cuf (:5290: zero-gradient, with
// the normal momentum's ghosts zero where the boundary cell's flow enters; the
// lower z side tests the x momentum, as the reference does), bcwall_ad_cuf
// (:5749).  One launch per face, faces in the reference's order.
__global__ void k_bc_face(DevCtx c, double *__restrict__ w, int ilat, int tag, int nv, const double *__restrict__ winf) {
  const DevGrid &g = c.g;
  int dir = (ilat - 1) / 2, hi = (ilat - 1) % 2;
  int na = dir == 0 ? g.ny : g.nx, nb = dir == 2 ? g.ny : g.nz;
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long per = (long long)na * nb;
  if (tid >= per * nv) return;
  int m = 1 + (int)(tid / per);
  long long q = tid % per;
  int a = 1 + (int)(q % na), b = 1 + (int)(q / na);
  int n = dir == 0 ? g.nx : (dir == 1 ? g.ny : g.nz);
  int ns = nv - 4;
  auto at = [&](int nn) -> long long {
    return dir == 0 ? gidx(g, nn, a, b) : (dir == 1 ? gidx(g, a, nn, b) : gidx(g, a, b, nn));
  };
  const int mn = ns + 1 + dir;                       // the normal momentum
  double sg = (tag == 8 && m >= ns + 1 && m <= ns + 3) ? -1.0 : 1.0;
  bool zero = false;
  if (tag == 5) {
    if (dir != 1) return;
    if (m == mn) FG(w, at(hi ? n : 1), m) = 0.0;
    if (m == mn) sg = -1.0;
  } else if (tag == 7 && m == mn) {
    const int mt = ilat == 5 ? ns + 1 : mn;
    double v = FG(w, at(hi ? n : 1), mt);
    zero = hi ? v < 0.0 : v > 0.0;
  }
  for (int l = 1; l <= g.ng; l++) {
    int dst = hi ? n + l : 1 - l;
    int src;
    if (tag == 2 || tag == 7) src = hi ? n : 1;
    else if (tag == 5) src = hi ? n - l : l;
    else src = hi ? n + 1 - l : l;   // tag 8
    long long pd = at(dst);
    if (tag == 1) FG(w, pd, m) = winf[m - 1];
    else FG(w, pd, m) = zero ? 0.0 : sg * FG(w, at(src), m);
  }
}

// get_mixture_e_from_temperature_dev (kernels_gpu.F90:7047-7102) with the mass
// fractions Y: the species ranges located at tt, the constants then the
// integrated terms l = icl..icr, each over the species in order.
template <int NS>
__device__ double mix_e_at(const DevTab &t, double tt, const double *Y) {
  int nrange[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) nrange[k] = t.nset > 1 ? locate_range(t, tt, k + 1) : 1;
  double ee = 0.0;
#pragma unroll
  for (int k = 0; k < NS; k++) ee = ee + cpc(t, t.cv, t.icr + 1, k + 1, nrange[k]) * Y[k];
  for (int l = t.icl; l <= t.icr; l++) {
    double tprod = l == -1 ? log(tt) : ipow(tt, l + 1) / (l + 1.0);
    double cv_l = 0.0;
#pragma unroll
    for (int k = 0; k < NS; k++) cv_l = cv_l + cpc(t, t.cv, l, k + 1, nrange[k]) * Y[k];
    ee = ee + cv_l * tprod;
  }
  return ee;
}

// update_ghost face kernels that need the thermodynamics and w_aux, one thread
// per boundary point, all ng layers:
//  * tag 4, bcextr_sub_cuf (kernels_gpu.F90:4092-4327), every side: the
//    boundary cell's mass fractions into w_aux; ghosts with its species and
//    momentum and the energy at T = p0 / (rho R_mix);
//  * tag 6, bcwall_cuf (:5437-5545), y sides only: the first ng interior rows'
//    mass fractions into w_aux; ghost 1-l (ny+l) mirrors row l (ny+1-l) with the
//    velocity reversed, the pressure kept and T' = max(2 T_wall - T, 200 K), T
//    from e by the Newton iteration started at the row's w_aux(J_T).
template <int NS>
__global__ void k_bc_face_thermo(DevCtx c, double *__restrict__ w, double *__restrict__ wa, int ilat, int tag) {
  const DevGrid &g = c.g;
  const DevTab &t = c.t;
  int dir = (ilat - 1) / 2, hi = (ilat - 1) % 2;
  int na = dir == 0 ? g.ny : g.nx, nb = dir == 2 ? g.ny : g.nz;
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (long long)na * nb) return;
  int a = 1 + (int)(tid % na), b = 1 + (int)(tid / na);
  int n = dir == 0 ? g.nx : (dir == 1 ? g.ny : g.nz);
  auto at = [&](int nn) -> long long {
    return dir == 0 ? gidx(g, nn, a, b) : (dir == 1 ? gidx(g, a, nn, b) : gidx(g, a, b, nn));
  };
  if (tag == 4) {
    long long p = at(hi ? n : 1);
    double rho = FG(w, p, 1);
#pragma unroll
    for (int k = 1; k < NS; k++) rho = rho + FG(w, p, k + 1);
    double Y[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) { Y[k] = FG(w, p, k + 1) / rho; FG(wa, p, k + 1) = Y[k]; }
    double rm = ldg(t.rgas) * Y[0];
#pragma unroll
    for (int k = 1; k < NS; k++) rm = rm + ldg(t.rgas + k) * Y[k];
    const double tt = c.p.p0 / rho / rm;
    const double ee = mix_e_at<NS>(t, tt, Y);
    const double rhou = FG(w, p, NS + 1), rhov = FG(w, p, NS + 2), rhow = FG(w, p, NS + 3);
    const double rhoE = rho * ee + 0.5 * (rhou * rhou + rhov * rhov + rhow * rhow) / rho;
    for (int l = 1; l <= g.ng; l++) {
      long long q = at(hi ? n + l : 1 - l);
#pragma unroll
      for (int k = 0; k < NS; k++) FG(w, q, k + 1) = FG(w, p, k + 1);
      FG(w, q, NS + 1) = rhou;
      FG(w, q, NS + 2) = rhov;
      FG(w, q, NS + 3) = rhow;
      FG(w, q, NS + 4) = rhoE;
    }
    return;
  }
  // tag 6 (the host launches it for the y sides only)
  for (int l = 1; l <= g.ng; l++) {
    long long p = at(hi ? n + 1 - l : l);
    double rho = FG(w, p, 1);
#pragma unroll
    for (int k = 1; k < NS; k++) rho = rho + FG(w, p, k + 1);
#pragma unroll
    for (int k = 0; k < NS; k++) FG(wa, p, k + 1) = FG(w, p, k + 1) / rho;
  }
  for (int l = 1; l <= g.ng; l++) {
    long long p = at(hi ? n + 1 - l : l), q = at(hi ? n + l : 1 - l);
    double rho = FG(w, p, 1);
#pragma unroll
    for (int k = 1; k < NS; k++) rho = rho + FG(w, p, k + 1);
    double uu = FG(w, p, NS + 1) / rho, vv = FG(w, p, NS + 2) / rho, ww = FG(w, p, NS + 3) / rho;
    double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
    double ee = FG(w, p, NS + 4) / rho - qq;
    double Y[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) Y[k] = FG(wa, p, k + 1);
    double tt = temp_from_e<NS>(t, c.p, ee, FG(wa, p, NS + 5), Y);
    double rm = ldg(t.rgas) * Y[0];
#pragma unroll
    for (int k = 1; k < NS; k++) rm = rm + ldg(t.rgas + k) * Y[k];
    double pp = rho * tt * rm;
    tt = 2.0 * c.p.T_wall - tt;
    if (tt < 200.0) tt = 200.0;
    ee = mix_e_at<NS>(t, tt, Y);
    rho = pp / tt / rm;
#pragma unroll
    for (int k = 0; k < NS; k++) FG(w, q, k + 1) = rho * Y[k];
    FG(w, q, NS + 1) = -rho * uu;
    FG(w, q, NS + 2) = -rho * vv;
    FG(w, q, NS + 3) = -rho * ww;
    FG(w, q, NS + 4) = rho * (ee + qq);
  }
}

// ---------------------------------------------------------------- characteristic boundaries
// Entries of the left (el(n, m): variable n, wave m) and right (er(m, n): wave m,
// variable n) eigenvectors of eigenvectors_{x,y,z} (kernels_gpu.F90:2703-2984),
// 1-based, formed on the fly from the point state instead of stored as
// (ns+4)^2 matrices.
struct NrPoint {
  double b1, b2, b3, c, ci, cci, h, un, v1, v2, vel[3];
  int dir, it1, it2;
};
template <int NS>
__device__ __forceinline__ double nr_el(const NrPoint &R, const double *yy, const double *prhoi, int n, int m) {
  const int In = NS + 1 + R.dir, It1 = NS + 1 + R.it1, It2 = NS + 1 + R.it2, IE = NS + 4;
  if (n <= NS) {
    const double b1n = R.b1 + prhoi[n - 1] * R.cci;
    if (m == 1) return 0.5 * (b1n + R.un * R.ci);
    if (m <= NS + 1) return (n == m - 1 ? 1.0 : 0.0) - b1n * yy[m - 2];
    if (m == NS + 2) return -R.v1;
    if (m == NS + 3) return -R.v2;
    return 0.5 * (b1n - R.un * R.ci);
  }
  if (m >= 2 && m <= NS + 1) return n == IE ? -R.b2 * yy[m - 2] : R.b2 * R.vel[n - NS - 1] * yy[m - 2];
  if (m == 1) {
    if (n == In) return -0.5 * (R.b2 * R.un + R.ci);
    if (n == It1) return -0.5 * (R.b2 * R.v1);
    if (n == It2) return -0.5 * (R.b2 * R.v2);
    return 0.5 * R.b2;
  }
  if (m == NS + 2) return n == It1 ? 1.0 : 0.0;
  if (m == NS + 3) return n == It2 ? 1.0 : 0.0;
  if (n == In) return -0.5 * (R.b2 * R.un - R.ci);
  if (n == It1) return -0.5 * (R.b2 * R.v1);
  if (n == It2) return -0.5 * (R.b2 * R.v2);
  return 0.5 * R.b2;
}
template <int NS>
__device__ __forceinline__ double nr_er(const NrPoint &R, const double *yy, const double *prhoi, int m, int n) {
  const int In = NS + 1 + R.dir, It1 = NS + 1 + R.it1, It2 = NS + 1 + R.it2, IE = NS + 4;
  if (n <= NS) {                                       // species columns
    if (m == 1 || m == NS + 4) return yy[n - 1];
    return m == n + 1 ? 1.0 : 0.0;
  }
  if (m >= 2 && m <= NS + 1) {                         // species waves
    if (n == IE) return R.b3 - prhoi[m - 2] / R.b2 * R.cci;
    return R.vel[n - NS - 1];
  }
  if (m == 1) {
    if (n == In) return R.un - R.c;
    if (n == It1) return R.v1;
    if (n == It2) return R.v2;
    return R.h - R.un * R.c;
  }
  if (m == NS + 2) return n == It1 ? 1.0 : (n == IE ? R.v1 : 0.0);
  if (m == NS + 3) return n == It2 ? 1.0 : (n == IE ? R.v2 : 0.0);
  if (n == In) return R.un + R.c;
  if (n == It1) return R.v1;
  if (n == It2) return R.v2;
  return R.h + R.un * R.c;
}

// bc_nr_lat_{x,y,z}_kernel (kernels_gpu.F90:4330-4793), one thread per boundary
// cell of face ilat: the one-sided derivative of w projected on the waves, the
// wave amplitudes of treatment nr_type (1 incoming acoustic waves removed; 2 / 3
// incoming waves from the difference to the outer ghost / to winf; 6 reflecting
// wall), projected back and added to fl.
template <int NS>
__global__ void k_bc_nr(DevCtx c, const double *__restrict__ wa, const double *__restrict__ w, double *__restrict__ fl,
                        const double *__restrict__ winf, int ilat, int nr_type) {
  constexpr int NV = NS + 4;
  const DevGrid &g = c.g;
  const int dir = (ilat - 1) / 2, se = (ilat - 1) % 2 + 1;
  const int na = dir == 0 ? g.ny : g.nx, nb = dir == 2 ? g.ny : g.nz;
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= (long long)na * nb) return;
  const int a = 1 + (int)(tid % na), b = 1 + (int)(tid / na);
  const int n = dir == 0 ? g.nx : (dir == 1 ? g.ny : g.nz);
  const int ib = se == 1 ? 1 : n, sgn = se == 1 ? 1 : -1;
  auto at = [&](int nn) -> long long {
    return dir == 0 ? gidx(g, nn, a, b) : (dir == 1 ? gidx(g, a, nn, b) : gidx(g, a, b, nn));
  };
  const double c_one[3] = {-1.5, 2.0, -0.5};
  const long long p = at(ib);
  double dw[NV], dwo[NV];
  for (int m = 1; m <= NV; m++) {
    double d = 0.0;
    for (int l = 1; l <= 3; l++) d = d + sgn * c_one[l - 1] * FG(w, at(ib + sgn * (l - 1)), m);
    dw[m - 1] = d;
    double w_target = 0.0;
    if (nr_type == 2) w_target = FG(w, at(ib - sgn), m);
    else if (nr_type == 3) w_target = winf ? winf[m - 1] : 0.0;
    dwo[m - 1] = sgn * (FG(w, p, m) - w_target);
  }
  double yy[NS], prhoi[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) yy[k] = FG(wa, p, k + 1);
  const double rho = FG(wa, p, NS + 11), uu = FG(wa, p, NS + 1), vv = FG(wa, p, NS + 2), ww = FG(wa, p, NS + 3);
  const double h = FG(wa, p, NS + 4), tt = FG(wa, p, NS + 5), pp = FG(wa, p, NS + 6), cs = FG(wa, p, NS + 7);
  const double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  const double cc = cs * cs, rmix_tt = pp / rho, gamloc = cc / rmix_tt, gm1loc = gamloc - 1.0;
  const double p_e = rho * gm1loc, etot = h - rmix_tt;
  NrPoint R;
  R.b3 = etot;
  R.b2 = p_e / (rho * cc);
  R.b1 = -R.b2 * (etot - 2.0 * qq);
  for (int k = 0; k < NS; k++) {
    const double eei = species_poly_int(c.t, c.t.cvi, tt, k + 1);
    prhoi[k] = ldg(c.t.rgas + k) * tt + gm1loc * (etot - qq - eei);
  }
  R.c = cs;
  R.ci = 1.0 / cs;
  R.cci = R.ci * R.ci;
  R.h = h;
  R.vel[0] = uu; R.vel[1] = vv; R.vel[2] = ww;
  R.dir = dir;
  R.it1 = dir == 0 ? 1 : 0;
  R.it2 = dir == 2 ? 1 : 2;
  R.un = R.vel[dir];
  R.v1 = R.vel[R.it1];
  R.v2 = R.vel[R.it2];
  double dwc[NV];
  for (int m = 1; m <= NV; m++) {
    double s1 = 0.0, s2 = 0.0;
    for (int mm = 1; mm <= NV; mm++) {
      const double e = nr_el<NS>(R, yy, prhoi, mm, m);
      s1 = s1 + e * dw[mm - 1];
      s2 = s2 + e * dwo[mm - 1];
    }
    double ev = (m == 1) ? R.un - cs : (m == NV ? R.un + cs : R.un);
    if (nr_type == 1) ev = sgn * dmin_(sgn * ev, 0.0);
    if ((nr_type == 2 || nr_type == 3) && sgn * ev > 0.0) s1 = s2;
    dwc[m - 1] = ev * s1;
  }
  if (nr_type == 6) {
    for (int m = 2; m <= NS + 3; m++) dwc[m - 1] = 0.0;
    if (se == 1) dwc[NV - 1] = dwc[0];
    else dwc[0] = dwc[NV - 1];
  }
  const double *met = dir == 0 ? g.dcsidx : (dir == 1 ? g.detady : g.dzitdz);
  const double mt = ldg(met + ib - 1);
  const int ii = dir == 0 ? ib : a, jj = dir == 1 ? ib : (dir == 0 ? a : b), kk = dir == 2 ? ib : b;
  const long long q = fidx(g, ii, jj, kk);
  for (int m = 1; m <= NV; m++) {
    double df = 0.0;
    for (int mm = 1; mm <= NV; mm++) df = df + nr_er<NS>(R, yy, prhoi, mm, m) * dwc[mm - 1];
    FI(fl, q, m) = FI(fl, q, m) + df * mt;
  }
}

// ============================================================== RK bookkeeping
// init_flux_cuf / init_flux_simpler_cuf / update_flux_cuf / update_simpler_flux_cuf
// (kernels_gpu.F90:28-66, 3297-3334); fl is (nx,ny,nz,nv) so these are flat maps.
// dt_d (captured CFL-driven steps): rhodt / gamdt hold the RK coefficient, and
// the scalar is coefficient * (scale * dt) with dt from device memory
__global__ void k_init_flux(double *__restrict__ fl, double *__restrict__ fln, const double *__restrict__ fl_sav,
                            double rhodt, long long n, const double *__restrict__ dt_d, double scale) {
  if (dt_d) rhodt = rhodt * (scale * *dt_d);
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; q < n; q += (long long)gridDim.x * blockDim.x) {
    double f = fl[q];
    fln[q] = fl_sav ? -rhodt * (f - fl_sav[q]) : -rhodt * f;
    fl[q] = 0.0;
  }
}
__global__ void k_update_flux(const double *__restrict__ fl, double *__restrict__ fln, const double *__restrict__ fl_sav,
                              double gamdt, long long n, const double *__restrict__ dt_d, double scale) {
  if (dt_d) gamdt = gamdt * (scale * *dt_d);
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; q < n; q += (long long)gridDim.x * blockDim.x)
    fln[q] = fl_sav ? fln[q] - gamdt * (fl[q] - fl_sav[q]) : fln[q] - gamdt * fl[q];
}
__global__ void k_copy(const double *__restrict__ a, double *__restrict__ b, long long n) {
  long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (; q < n; q += (long long)gridDim.x * blockDim.x) b[q] = a[q];
}
// update_field_cuf (kernels_gpu.F90:3336-3355), optionally fused with
// update_flux: fln -= gamdt*fl (or gamdt*(fl - fl_sav)); w += fln where fluid.
__global__ void k_update_field(DevCtx c, double *__restrict__ w, const double *__restrict__ fl, double *__restrict__ fln,
                               const double *__restrict__ fl_sav, const int32_t *__restrict__ mask, double gamdt,
                               int fused, int nv, double scale) {
  const DevGrid &g = c.g;
  if (c.p.dt_d) gamdt = gamdt * (scale * *c.p.dt_d);
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= g.npi) return;
  int i = 1 + (int)(tid % g.nx);
  long long r = tid / g.nx;
  int j = 1 + (int)(r % g.ny);
  int k = 1 + (int)(r / g.ny);
  long long p = gidx(g, i, j, k);
  bool fluid = (mask == nullptr) || (mask[p] == 0);
  for (int m = 1; m <= nv; m++) {
    double a;
    if (fused) {
      a = fl_sav ? FI(fln, tid, m) - gamdt * (FI(fl, tid, m) - FI(fl_sav, tid, m)) : FI(fln, tid, m) - gamdt * FI(fl, tid, m);
      FI(fln, tid, m) = a;
    } else {
      a = FI(fln, tid, m);
    }
    if (fluid) FG(w, p, m) = FG(w, p, m) + a;
  }
}

// ============================================================== compute_dt
// compute_dt_cuf (kernels_gpu.F90:6075-6152): nine maxima, warp shuffles then one
// atomicMax per block on the bit patterns (non-negative doubles order as integers).
template <int NS>
__global__ void __launch_bounds__(256) k_compute_dt(DevCtx c, const double *__restrict__ wa, const int32_t *__restrict__ mask,
                                                    unsigned long long *__restrict__ out) {
  const DevGrid &g = c.g;
  double v[9];
#pragma unroll
  for (int q = 0; q < 9; q++) v[q] = 0.0;
  for (long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x; tid < g.npi;
       tid += (long long)gridDim.x * blockDim.x) {
    int i = 1 + (int)(tid % g.nx);
    long long r = tid / g.nx;
    int j = 1 + (int)(r % g.ny);
    int k = 1 + (int)(r / g.ny);
    long long p = gidx(g, i, j, k);
    if (mask != nullptr && mask[p] != 0) continue;
    double Y[NS];
#pragma unroll
    for (int s = 0; s < NS; s++) Y[s] = FG(wa, p, s + 1);
    double rho = FG(wa, p, NS + 11), ri = 1.0 / rho;
    double uu = FG(wa, p, NS + 1), vv = FG(wa, p, NS + 2), ww = FG(wa, p, NS + 3), tt = FG(wa, p, NS + 5);
    double mu = FG(wa, p, NS + 8), cc = FG(wa, p, NS + 7), kc = FG(wa, p, NS + 13);
    double cploc = mix_cp<NS>(c.t, tt, Y);
    double nu = ri * mu, kr = kc * ri / cploc;
    double a[9] = {(fabs(uu) + cc) * ldg(g.dcsidx + i - 1), (fabs(vv) + cc) * ldg(g.detady + j - 1),
                   (fabs(ww) + cc) * ldg(g.dzitdz + k - 1), nu * ldg(g.dcsidxs + i - 1), nu * ldg(g.detadys + j - 1),
                   nu * ldg(g.dzitdzs + k - 1), kr * ldg(g.dcsidxs + i - 1), kr * ldg(g.detadys + j - 1),
                   kr * ldg(g.dzitdzs + k - 1)};
#pragma unroll
    for (int q = 0; q < 9; q++) v[q] = dmax_(v[q], a[q]);
  }
#pragma unroll
  for (int q = 0; q < 9; q++) {
    for (int o = 16; o > 0; o >>= 1) v[q] = dmax_(v[q], __shfl_xor_sync(0xffffffffu, v[q], o));
  }
  __shared__ double sm[9][8];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    for (int q = 0; q < 9; q++) sm[q][wid] = v[q];
  __syncthreads();
  if (threadIdx.x < 9) {
    double m = 0.0;
    for (int wv = 0; wv < (int)(blockDim.x >> 5); wv++) m = dmax_(m, sm[threadIdx.x][wv]);
    atomicMax(out + threadIdx.x, (unsigned long long)__double_as_longlong(m));
  }
}

// compute_residual_cuf + compute_rho_t_p_minmax_cuf (kernels_gpu.F90:5991-6011,
// 6038-6073): the sum of (fln(I_U)/dt)^2 and the extrema of rho, T and p over
// the fluid interior cells.  The sum is deterministic: a fixed grid of
// RES_BLOCKS blocks, each writing its partial sum (warp shuffles in a fixed
// order) to part[block]; the host adds the partials in block order.  The
// extrema of these positive quantities are exact: atomicMin / atomicMax on the
// bit patterns of the doubles (mm[0..2] minima of rho, T, p; mm[3..5] maxima).
template <int NS>
__global__ void __launch_bounds__(256) k_residual_minmax(DevCtx c, const double *__restrict__ fln,
                                                         const double *__restrict__ wa, const int32_t *__restrict__ mask,
                                                         double dt, double *__restrict__ part,
                                                         unsigned long long *__restrict__ mm) {
  const DevGrid &g = c.g;
  double sum = 0.0, vmin[3] = {INFINITY, INFINITY, INFINITY}, vmax[3] = {0.0, 0.0, 0.0};
  for (long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x; tid < g.npi;
       tid += (long long)gridDim.x * blockDim.x) {
    int i = 1 + (int)(tid % g.nx);
    long long r = tid / g.nx;
    int j = 1 + (int)(r % g.ny);
    int k = 1 + (int)(r / g.ny);
    long long p = gidx(g, i, j, k);
    if (mask != nullptr && mask[p] != 0) continue;
    double f = FI(fln, tid, NS + 1) / dt;
    sum = sum + f * f;
    double v[3] = {FG(wa, p, NS + 11), FG(wa, p, NS + 5), FG(wa, p, NS + 6)};
#pragma unroll
    for (int q = 0; q < 3; q++) { vmin[q] = dmin_(vmin[q], v[q]); vmax[q] = dmax_(vmax[q], v[q]); }
  }
  for (int o = 16; o > 0; o >>= 1) {
    sum = sum + __shfl_xor_sync(0xffffffffu, sum, o);
#pragma unroll
    for (int q = 0; q < 3; q++) {
      vmin[q] = dmin_(vmin[q], __shfl_xor_sync(0xffffffffu, vmin[q], o));
      vmax[q] = dmax_(vmax[q], __shfl_xor_sync(0xffffffffu, vmax[q], o));
    }
  }
  __shared__ double sm[7][8];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    sm[0][wid] = sum;
    for (int q = 0; q < 3; q++) { sm[1 + q][wid] = vmin[q]; sm[4 + q][wid] = vmax[q]; }
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    const int nw = (int)(blockDim.x >> 5), q = threadIdx.x;
    double m = sm[q][0];
    for (int wv = 1; wv < nw; wv++) m = q == 0 ? m + sm[q][wv] : (q < 4 ? dmin_(m, sm[q][wv]) : dmax_(m, sm[q][wv]));
    if (q == 0) part[blockIdx.x] = m;
    else if (q < 4) atomicMin(mm + q - 1, (unsigned long long)__double_as_longlong(m));
    else atomicMax(mm + q - 1, (unsigned long long)__double_as_longlong(m));
  }
}

// ============================================================== launchers
template <int NS>
static int eval_aux_t(const DevCtx &c, cudaStream_t s, double *w, double *wa, int i0, int i1, int j0, int j1, int k0, int k1) {
  int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
  if (ni <= 0 || nj <= 0 || nk <= 0) return STX_OK;
  long long n = (long long)ni * nj * nk;
  // transport properties: FP64 (plain form) or FP32 (mixed form)
  if (c.p.mixed) k_eval_aux<NS, float><<<grid1d(n, 128), 128, 0, s>>>(c, w, wa, i0, j0, k0, ni, nj, nk);
  else k_eval_aux<NS, double><<<grid1d(n, 128), 128, 0, s>>>(c, w, wa, i0, j0, k0, ni, nj, nk);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_eval_aux(const DevCtx &c, cudaStream_t s, double *w, double *wa, int i0, int i1, int j0, int j1, int k0, int k1) {
  switch (c.t.ns) {
#define X(N) case N: return eval_aux_t<N>(c, s, w, wa, i0, i1, j0, j1, k0, k1);
    STX_FOR_NS(X)
#undef X
    default: return STX_E_UNSUPPORTED;
  }
}

int launch_eval_aux2(const DevCtx &c, cudaStream_t s, double *wa) {
  k_eval_aux2<<<grid1d(c.g.npi, 256), 256, 0, s>>>(c, wa, c.t.ns);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_bcextr_var(const DevCtx &c, cudaStream_t s, double *v) {
  const DevGrid &g = c.g;
  long long n = 2LL * ((long long)g.ny * g.nz + (long long)g.nx * g.nz + (long long)g.nx * g.ny);
  k_bcextr_var<<<grid1d(n, 256), 256, 0, s>>>(c, v);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_bcswap(const DevCtx &c, cudaStream_t s, double *f, int nvar, const int *periodic) {
  const DevGrid &g = c.g;
  if (g.ng > STX_MAXNG) return STX_E_UNSUPPORTED;
  long long per = (periodic[0] ? (long long)g.ny * g.nz : 0) + (periodic[1] ? (long long)g.nx * g.nz : 0) +
                  (periodic[2] ? (long long)g.nx * g.ny : 0);
  if (per == 0) return STX_OK;
  k_bcswap<<<grid1d(per * nvar, 256), 256, 0, s>>>(c, f, nvar, periodic[0], periodic[1], periodic[2]);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_bc_face(const DevCtx &c, cudaStream_t s, double *w, int ilat, int tag, const double *winf) {
  const DevGrid &g = c.g;
  int dir = (ilat - 1) / 2;
  int na = dir == 0 ? g.ny : g.nx, nb = dir == 2 ? g.ny : g.nz;
  int nv = c.t.ns + 4;
  if (tag == 1 && (ilat != 1 || winf == nullptr)) return STX_OK;   // bcfree_cuf acts on the left side only
  long long n = (long long)na * nb * nv;
  k_bc_face<<<grid1d(n, 256), 256, 0, s>>>(c, w, ilat, tag, nv, winf);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_bc_face_thermo(const DevCtx &c, cudaStream_t s, double *w, double *wa, int ilat, int tag) {
  int dir = (ilat - 1) / 2;
  if (tag == 6 && dir != 1) return STX_OK;           // bcwall_cuf acts on the y sides only
  long long n = (long long)(dir == 0 ? c.g.ny : c.g.nx) * (dir == 2 ? c.g.ny : c.g.nz);
  switch (c.t.ns) {
#define X(N) case N: k_bc_face_thermo<N><<<grid1d(n, 128), 128, 0, s>>>(c, w, wa, ilat, tag); break;
    STX_FOR_NS(X)
#undef X
    default: return STX_E_UNSUPPORTED;
  }
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_bc_nr(const DevCtx &c, cudaStream_t s, const double *wa, const double *w, double *fl, const double *winf,
                 int ilat, int nr_type) {
  int dir = (ilat - 1) / 2;
  long long n = (long long)(dir == 0 ? c.g.ny : c.g.nx) * (dir == 2 ? c.g.ny : c.g.nz);
  switch (c.t.ns) {
#define X(N) case N: k_bc_nr<N><<<grid1d(n, 64), 64, 0, s>>>(c, wa, w, fl, winf, ilat, nr_type); break;
    STX_FOR_NS(X)
#undef X
    default: return STX_E_UNSUPPORTED;
  }
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_init_flux(const DevCtx &c, cudaStream_t s, double *fl, double *fln, const double *fl_sav, double rhodt,
                     double scale) {
  long long n = c.g.npi * (c.t.ns + 4);
  int nb = grid1d(n, 256);
  if (nb > 148 * 32) nb = 148 * 32;
  k_init_flux<<<nb, 256, 0, s>>>(fl, fln, fl_sav, rhodt, n, c.p.dt_d, scale);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_update_flux(const DevCtx &c, cudaStream_t s, const double *fl, double *fln, const double *fl_sav, double gamdt,
                       double scale) {
  long long n = c.g.npi * (c.t.ns + 4);
  int nb = grid1d(n, 256);
  if (nb > 148 * 32) nb = 148 * 32;
  k_update_flux<<<nb, 256, 0, s>>>(fl, fln, fl_sav, gamdt, n, c.p.dt_d, scale);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_copy(const DevCtx &c, cudaStream_t s, const double *a, double *b) {
  long long n = c.g.npi * (c.t.ns + 4);
  int nb = grid1d(n, 256);
  if (nb > 148 * 32) nb = 148 * 32;
  k_copy<<<nb, 256, 0, s>>>(a, b, n);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_update_field(const DevCtx &c, cudaStream_t s, double *w, const double *fl, double *fln, const double *fl_sav,
                        const int32_t *mask, double gamdt, int fused, double scale) {
  k_update_field<<<grid1d(c.g.npi, 256), 256, 0, s>>>(c, w, fl, fln, fl_sav, mask, gamdt, fused, c.t.ns + 4, scale);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

__global__ void k_dt_from_max(const unsigned long long *__restrict__ max9, double cfl, double *__restrict__ dt) {
  double m = __longlong_as_double((long long)max9[0]);
  for (int q = 1; q < 9; q++) {
    const double v = __longlong_as_double((long long)max9[q]);
    if (v > m) m = v;
  }
  *dt = cfl / m;
}
__global__ void k_time_advance(double *__restrict__ t, const double *__restrict__ dt) { *t = *t + *dt; }

int launch_dt_from_max(cudaStream_t s, const unsigned long long *max9, double cfl, double *dt) {
  k_dt_from_max<<<1, 1, 0, s>>>(max9, cfl, dt);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}
int launch_time_advance(cudaStream_t s, double *t, const double *dt) {
  k_time_advance<<<1, 1, 0, s>>>(t, dt);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_compute_dt(const DevCtx &c, cudaStream_t s, const double *wa, const int32_t *mask, unsigned long long *out9) {
  STX_CUDA_TRY(cudaMemsetAsync(out9, 0, 9 * sizeof(unsigned long long), s));
  int nb = grid1d(c.g.npi, 256);
  if (nb > 148 * 8) nb = 148 * 8;
  switch (c.t.ns) {
#define X(N) case N: k_compute_dt<N><<<nb, 256, 0, s>>>(c, wa, mask, out9); break;
    STX_FOR_NS(X)
#undef X
    default: return STX_E_UNSUPPORTED;
  }
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_residual_minmax(const DevCtx &c, cudaStream_t s, const double *fln, const double *wa, const int32_t *mask,
                           double dt, double *part, unsigned long long *mm) {
  // minima start at +inf (0x7ff0...), maxima at +0
  static const unsigned long long init[6] = {0x7ff0000000000000ull, 0x7ff0000000000000ull, 0x7ff0000000000000ull,
                                             0ull, 0ull, 0ull};
  STX_CUDA_TRY(cudaMemcpyAsync(mm, init, sizeof(init), cudaMemcpyHostToDevice, s));
  switch (c.t.ns) {
#define X(N) case N: k_residual_minmax<N><<<STX_RES_BLOCKS, 256, 0, s>>>(c, fln, wa, mask, dt, part, mm); break;
    STX_FOR_NS(X)
#undef X
    default: return STX_E_UNSUPPORTED;
  }
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}
