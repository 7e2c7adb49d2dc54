// stx_visc.cu -- mixture-averaged viscous, heat and species-diffusion fluxes
// (visflx mode 1: visflx_{x,y,z}_cuf, kernels_gpu.F90:3658-4031) fused with their
// divergence, and the collocated cross/dilatation terms (mode 2:
// visflx_reduced_cuf, :3539-3656).
//
// The x sweep exchanges face fluxes through shared memory (threads along the
// contiguous i index); the y/z sweeps march along the sweep with the previous
// face flux -- and the species enthalpies of the shared point -- in registers.
// Prefetching (prefetch.global.L1 / .L2) the point and residual cell of the
// face 1, 2 or 3 ahead made a 256^3 mode-1 call slower (FP64: 16.0-16.2 ms
// against 15.5 ms), so the sweeps issue none.
#include "stx_kernels.cuh"

// CTAs per SM the viscous sweeps' register budget is sized for.  Unconstrained
// they take 164 registers (3 CTAs per SM), and their loads are latency-bound at
// 12 warps per SM.  On a developed 128^3 field, mode 1: 5 CTAs per SM (102
// registers, some spilled) ran a call in 2.06 ms, 4 in 2.41 ms, 6 in 2.13 ms,
// and the unconstrained kernel about 1.45x slower than 4, with the same results
// bit for bit.  With 53 species (spilled at any budget) a 48^3 call took
// 3.41-3.50 ms unconstrained, at 4 and at 5
#ifndef STX_VISC_MINB
#define STX_VISC_MINB 5
#endif

// One staggered face between points p (left) and q = p + st (right), computed in
// R (double: plain form; float: mixed form, fields rounded once on load).  hl
// carries the species enthalpies at
// the left point in and those of the right point out (reused by the next face).
template <int NS, typename R>
__device__ __forceinline__ void visc_face(const DevCtx &c, const double *__restrict__ wa, long long p, long long q,
                                          R dxf, R *hl, bool have_hl, R *fh) {
  const DevGrid &g = c.g;
  const DevTab &t = c.t;
  auto ld = [&](long long r, int m) -> R { return (R)FG(wa, r, m); };
  const int J_U = NS + 1, J_V = NS + 2, J_W = NS + 3, J_T = NS + 5, J_MU = NS + 8, J_K = NS + 13, J_D = NS + 13;
  R uu = ld(p, J_U), uup = ld(q, J_U), vv = ld(p, J_V), vvp = ld(q, J_V);
  R ww = ld(p, J_W), wwp = ld(q, J_W), tt = ld(p, J_T), ttp = ld(q, J_T);
  R mu = ld(p, J_MU), mup = ld(q, J_MU), kc = ld(p, J_K), kcp = ld(q, J_K);
  R qq = R(0.5) * (uu * uu + vv * vv + ww * ww);
  R qqp = R(0.5) * (uup * uup + vvp * vvp + wwp * wwp);
  R sigx = uup - uu, sigy = vvp - vv, sigz = wwp - ww;
  R sigq_tt = ttp - tt, sigq_qq = qqp - qq;
  R muf = mu + mup;
  muf = R(0.5) * muf / dxf;
  R kf = kc + kcp;
  kf = R(0.5) * kf / dxf;
  sigx = sigx * muf; sigy = sigy * muf; sigz = sigz * muf;
  R sigq = sigq_tt * kf + sigq_qq * muf;
  R yl[NS], yp[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) { yl[k] = ld(p, k + 1); yp[k] = ld(q, k + 1); }
  R rm = (R)ldg(t.rgas) * yl[0];
#pragma unroll
  for (int k = 1; k < NS; k++) rm = rm + (R)ldg(t.rgas + k) * yl[k];
  R mwm = R(t.Ru) / rm;
  rm = (R)ldg(t.rgas) * yp[0];
#pragma unroll
  for (int k = 1; k < NS; k++) rm = rm + (R)ldg(t.rgas + k) * yp[k];
  R mwmp = R(t.Ru) / rm;
  R mwmif = R(0.5) * (mwmp + mwm) / (mwmp * mwm);
  mwmif = mwmif / dxf;
  R rd[NS];
  R fhat_tmp = R(0.0);
#pragma unroll
  for (int k = 0; k < NS; k++) {
    rd[k] = R(0.5) * (ld(p, J_D + 1 + k) + ld(q, J_D + 1 + k));
    R xxp = yp[k] * mwmp, xx = yl[k] * mwm;
    fhat_tmp = fhat_tmp + (xxp - xx) * rd[k];
  }
  fhat_tmp = fhat_tmp * mwmif;
  R et = R(0.0);
#pragma unroll
  for (int k = 0; k < NS; k++) {
    R yyf = R(0.5) * (yp[k] + yl[k]);
    R xxp = yp[k] * mwmp, xx = yl[k] * mwm;
    R sig = -rd[k] * (xxp - xx) * mwmif + fhat_tmp * yyf;
    fh[k] = sig;
    R hh = have_hl ? hl[k] : (R)species_poly_int(t, t.cpi, (double)tt, k + 1);
    R hhp = (R)species_poly_int(t, t.cpi, (double)ttp, k + 1);
    hl[k] = hhp;
    R hhf = R(0.5) * (hh + hhp);
    et = et + sig * hhf;
  }
  fh[NS] = -sigx;
  fh[NS + 1] = -sigy;
  fh[NS + 2] = -sigz;
  fh[NS + 3] = -sigq + et;
}

// x sweep: the faces 0..nx of every (j, k) row are numbered as one sequence
// F = row * (nx + 1) + f; CTA b of XB threads computes faces (XB-1) b ..
// (XB-1) b + XB-1 (one shared with the next CTA) into shared memory, and the
// threads whose face is not the first of its row form the divergence -- every
// thread busy for any nx.
template <int NS, typename R>
__global__ void __launch_bounds__(128, STX_VISC_MINB) k_visc_x(DevCtx c, const double *__restrict__ wa, double *__restrict__ fl) {
  const DevGrid &g = c.g;
  const int NV = NS + 4;
  constexpr int XB = xsweep_block(NS);
  __shared__ R sf[NV][XB];
  const long long nf = g.nx + 1;
  const long long F = (long long)blockIdx.x * (XB - 1) + threadIdx.x;
  const bool act = F < nf * g.ny * g.nz;
  const long long row = F / nf;
  const int f = (int)(F - row * nf);
  const int j = 1 + (int)(row % g.ny), k = 1 + (int)(row / g.ny);
#define XC(i) ldg(g.x + (i) + g.ng - 1)
  if (act) {
    R fh[NV], hl[NS];
    long long p = gidx(g, f, j, k);
    visc_face<NS, R>(c, wa, p, p + 1, (R)(XC(f + 1) - XC(f)), hl, false, fh);
#pragma unroll
    for (int m = 0; m < NV; m++) sf[m][threadIdx.x] = fh[m];
  }
  __syncthreads();
  int i = f;
  if (threadIdx.x >= 1 && act && i >= 1) {
    long long q = fidx(g, i, j, k);
    double dxhl = 2.0 / (XC(i + 1) - XC(i - 1));
#pragma unroll
    for (int m = 0; m < NV; m++)
      FI(fl, q, m + 1) = FI(fl, q, m + 1) + (double)((R)dxhl * (sf[m][threadIdx.x] - sf[m][threadIdx.x - 1]));
  }
#undef XC
}

template <int NS, int DIR, typename R>
__global__ void __launch_bounds__(128, STX_VISC_MINB) k_visc_yz(DevCtx c, const double *__restrict__ wa, double *__restrict__ fl, int chunk) {
  const DevGrid &g = c.g;
  const int NV = NS + 4;
  int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > g.nx) return;
  int tr = blockIdx.y + 1;
  int n = DIR == 1 ? g.ny : g.nz;
  int c0 = 1 + blockIdx.z * chunk;
  int c1 = min(c0 + chunk - 1, n);
  long long st = DIR == 1 ? (long long)g.nxg : (long long)g.nxg * g.nyg;
  const double *xc = DIR == 1 ? g.y : g.z;
#define XC(i) ldg(xc + (i) + g.ng - 1)
  R prev[NV], cur[NV], hl[NS];
  {
    int f = c0 - 1;
    long long p = DIR == 1 ? gidx(g, i, f, tr) : gidx(g, i, tr, f);
    visc_face<NS, R>(c, wa, p, p + st, (R)(XC(f + 1) - XC(f)), hl, false, prev);
  }
  for (int f = c0; f <= c1; f++) {
    long long p = DIR == 1 ? gidx(g, i, f, tr) : gidx(g, i, tr, f);
    visc_face<NS, R>(c, wa, p, p + st, (R)(XC(f + 1) - XC(f)), hl, true, cur);
    long long q = DIR == 1 ? fidx(g, i, f, tr) : fidx(g, i, tr, f);
    double dxhl = 2.0 / (XC(f + 1) - XC(f - 1));
#pragma unroll
    for (int m = 0; m < NV; m++) {
      FI(fl, q, m + 1) = FI(fl, q, m + 1) + (double)((R)dxhl * (cur[m] - prev[m]));
      prev[m] = cur[m];
    }
  }
#undef XC
}

// visflx_reduced_cuf (kernels_gpu.F90:3539-3656)
__global__ void __launch_bounds__(256) k_visc_reduced(DevCtx c, const double *__restrict__ wa, double *__restrict__ fl, int ns) {
  const DevGrid &g = c.g;
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= g.npi) return;
  int i = 1 + (int)(tid % g.nx);
  long long r = tid / g.nx;
  int j = 1 + (int)(r % g.ny);
  int k = 1 + (int)(r / g.ny);
  long long p = gidx(g, i, j, k);
  const int J_U = ns + 1, J_V = ns + 2, J_W = ns + 3, J_MU = ns + 8, J_DIV = ns + 10;
  double uu = FG(wa, p, J_U), vv = FG(wa, p, J_V), ww = FG(wa, p, J_W), mu = FG(wa, p, J_MU), div3l = FG(wa, p, J_DIV);
  int lmax = c.p.visc_order / 2;
  long long sx = 1, sy = g.nxg, sz = (long long)g.nxg * g.nyg;
  double ux = 0, vx = 0, wx = 0, mux = 0, dx3 = 0, uy = 0, vy = 0, wy = 0, muy = 0, dy3 = 0;
  double uz = 0, vz = 0, wz = 0, muz = 0, dz3 = 0;
  for (int l = 1; l <= lmax; l++) {
    double ccl = c.p.cd1[l][lmax];
#define D(s, J) (FG(wa, p + l * (s), J) - FG(wa, p - l * (s), J))
    ux = ux + ccl * D(sx, J_U); vx = vx + ccl * D(sx, J_V); wx = wx + ccl * D(sx, J_W);
    mux = mux + ccl * D(sx, J_MU); dx3 = dx3 + ccl * D(sx, J_DIV);
    uy = uy + ccl * D(sy, J_U); vy = vy + ccl * D(sy, J_V); wy = wy + ccl * D(sy, J_W);
    muy = muy + ccl * D(sy, J_MU); dy3 = dy3 + ccl * D(sy, J_DIV);
    uz = uz + ccl * D(sz, J_U); vz = vz + ccl * D(sz, J_V); wz = wz + ccl * D(sz, J_W);
    muz = muz + ccl * D(sz, J_MU); dz3 = dz3 + ccl * D(sz, J_DIV);
#undef D
  }
  double dx = ldg(g.dcsidx + i - 1), dy = ldg(g.detady + j - 1), dz = ldg(g.dzitdz + k - 1);
  ux = ux * dx; vx = vx * dx; wx = wx * dx; mux = mux * dx; dx3 = dx3 * dx;
  uy = uy * dy; vy = vy * dy; wy = wy * dy; muy = muy * dy; dy3 = dy3 * dy;
  uz = uz * dz; vz = vz * dz; wz = wz * dz; muz = muz * dz; dz3 = dz3 * dz;
  double s11 = ux - 2.0 * div3l, s12 = vx, s13 = wx;
  double s21 = uy, s22 = vy - 2.0 * div3l, s23 = wy;
  double s31 = uz, s32 = vz, s33 = wz - 2.0 * div3l;
  double sigx = mux * s11 + muy * s12 + muz * s13 + mu * dx3;
  double sigy = mux * s21 + muy * s22 + muz * s23 + mu * dy3;
  double sigz = mux * s31 + muy * s32 + muz * s33 + mu * dz3;
  double sigah = (s11 * ux + s12 * uy + s13 * uz + s21 * vx + s22 * vy + s23 * vz + s31 * wx + s32 * wy + s33 * wz) * mu;
  double sigq = sigx * uu + sigy * vv + sigz * ww + sigah;
  FI(fl, tid, ns + 1) = FI(fl, tid, ns + 1) - sigx;
  FI(fl, tid, ns + 2) = FI(fl, tid, ns + 2) - sigy;
  FI(fl, tid, ns + 3) = FI(fl, tid, ns + 3) - sigz;
  FI(fl, tid, ns + 4) = FI(fl, tid, ns + 4) - sigq;
}

template <int NS, typename R>
static int visc_r(const DevCtx &c, cudaStream_t s, int dir, const double *wa, double *fl) {
  const DevGrid &g = c.g;
  if (dir == 0) {
    constexpr int XB = xsweep_block(NS);
    long long nface = (long long)(g.nx + 1) * g.ny * g.nz;
    long long nb = (nface - 1 + XB - 2) / (XB - 1);
    if (nb > 0x7fffffffLL) return STX_E_INVALID;
    k_visc_x<NS, R><<<(unsigned)nb, XB, 0, s>>>(c, wa, fl);
  } else {
    int chunk = 8;
    int n = dir == 1 ? g.ny : g.nz;
    dim3 grid((g.nx + 127) / 128, dir == 1 ? g.nz : g.ny, (n + chunk - 1) / chunk);
    if (dir == 1) k_visc_yz<NS, 1, R><<<grid, 128, 0, s>>>(c, wa, fl, chunk);
    else k_visc_yz<NS, 2, R><<<grid, 128, 0, s>>>(c, wa, fl, chunk);
  }
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

// the plain form in FP64, the mixed form in FP32 (accumulated into the FP64 residual)
template <int NS>
static int visc_t(const DevCtx &c, cudaStream_t s, int dir, const double *wa, double *fl) {
  return c.p.mixed ? visc_r<NS, float>(c, s, dir, wa, fl) : visc_r<NS, double>(c, s, dir, wa, fl);
}

int launch_visflx(const DevCtx &c, cudaStream_t s, int dir, const double *wa, double *fl) {
  switch (c.t.ns) {
#define X(N) case N: return visc_t<N>(c, s, dir, wa, fl);
    STX_FOR_NS(X)
#undef X
    default: return STX_E_UNSUPPORTED;
  }
}

int launch_visflx_reduced(const DevCtx &c, cudaStream_t s, const double *wa, double *fl) {
  k_visc_reduced<<<grid1d(c.g.npi, 256), 256, 0, s>>>(c, wa, fl, c.t.ns);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}
