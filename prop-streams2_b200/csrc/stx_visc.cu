// stx_visc.cu -- mixture-averaged viscous, heat and species-diffusion fluxes
// (visflx mode 1: visflx_{x,y,z}_cuf, kernels_gpu.F90:3658-4031) fused with their
// divergence, and the collocated cross/dilatation terms (mode 2:
// visflx_reduced_cuf, :3539-3656).
//
// The x sweep exchanges face fluxes through shared memory (threads along the
// contiguous i index); the y/z sweeps march along the sweep with the previous
// face flux -- and the species enthalpies of the shared point -- in registers.
#include "stx_kernels.cuh"

// One staggered face between points p (left) and q = p + st (right); xl, xr
// are the coordinates of the two points.  hl carries the species enthalpies at
// the left point in and those of the right point out (reused by the next face).
template <int NS>
__device__ __forceinline__ void visc_face(const DevCtx &c, const double *__restrict__ wa, long long p, long long q,
                                          double dxf, double *hl, bool have_hl, double *fh) {
  const DevGrid &g = c.g;
  const DevTab &t = c.t;
  const int J_U = NS + 1, J_V = NS + 2, J_W = NS + 3, J_T = NS + 5, J_MU = NS + 8, J_K = NS + 13, J_D = NS + 13;
  double uu = FG(wa, p, J_U), uup = FG(wa, q, J_U), vv = FG(wa, p, J_V), vvp = FG(wa, q, J_V);
  double ww = FG(wa, p, J_W), wwp = FG(wa, q, J_W), tt = FG(wa, p, J_T), ttp = FG(wa, q, J_T);
  double mu = FG(wa, p, J_MU), mup = FG(wa, q, J_MU), kc = FG(wa, p, J_K), kcp = FG(wa, q, J_K);
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double qqp = 0.5 * (uup * uup + vvp * vvp + wwp * wwp);
  double sigx = uup - uu, sigy = vvp - vv, sigz = wwp - ww;
  double sigq_tt = ttp - tt, sigq_qq = qqp - qq;
  double muf = mu + mup;
  muf = 0.5 * muf / dxf;
  double kf = kc + kcp;
  kf = 0.5 * kf / dxf;
  sigx = sigx * muf; sigy = sigy * muf; sigz = sigz * muf;
  double sigq = sigq_tt * kf + sigq_qq * muf;
  double yl[NS], yp[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) { yl[k] = FG(wa, p, k + 1); yp[k] = FG(wa, q, k + 1); }
  double rm = ldg(t.rgas) * yl[0];
#pragma unroll
  for (int k = 1; k < NS; k++) rm = rm + ldg(t.rgas + k) * yl[k];
  double mwm = t.Ru / rm;
  rm = ldg(t.rgas) * yp[0];
#pragma unroll
  for (int k = 1; k < NS; k++) rm = rm + ldg(t.rgas + k) * yp[k];
  double mwmp = t.Ru / rm;
  double mwmif = 0.5 * (mwmp + mwm) / (mwmp * mwm);
  mwmif = mwmif / dxf;
  double rd[NS];
  double fhat_tmp = 0.0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    rd[k] = 0.5 * (FG(wa, p, J_D + 1 + k) + FG(wa, q, J_D + 1 + k));
    double xxp = yp[k] * mwmp, xx = yl[k] * mwm;
    fhat_tmp = fhat_tmp + (xxp - xx) * rd[k];
  }
  fhat_tmp = fhat_tmp * mwmif;
  double et = 0.0;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    double yyf = 0.5 * (yp[k] + yl[k]);
    double xxp = yp[k] * mwmp, xx = yl[k] * mwm;
    double sig = -rd[k] * (xxp - xx) * mwmif + fhat_tmp * yyf;
    fh[k] = sig;
    double hh = have_hl ? hl[k] : species_poly_int(t, t.cp, tt, k + 1);
    double hhp = species_poly_int(t, t.cp, ttp, k + 1);
    hl[k] = hhp;
    double hhf = 0.5 * (hh + hhp);
    et = et + sig * hhf;
  }
  fh[NS] = -sigx;
  fh[NS + 1] = -sigy;
  fh[NS + 2] = -sigz;
  fh[NS + 3] = -sigq + et;
}

template <int NS>
__global__ void __launch_bounds__(128) k_visc_x(DevCtx c, const double *__restrict__ wa, double *__restrict__ fl) {
  const DevGrid &g = c.g;
  const int NV = NS + 4;
  __shared__ double sf[NV][128];
  int j = blockIdx.y + 1, k = blockIdx.z + 1;
  int f0 = blockIdx.x * 127;            // faces 0..nx
  int f = f0 + threadIdx.x;
#define XC(i) ldg(g.x + (i) + g.ng - 1)
  if (f <= g.nx) {
    double fh[NV], hl[NS];
    long long p = gidx(g, f, j, k);
    visc_face<NS>(c, wa, p, p + 1, XC(f + 1) - XC(f), hl, false, fh);
#pragma unroll
    for (int m = 0; m < NV; m++) sf[m][threadIdx.x] = fh[m];
  }
  __syncthreads();
  int i = f;
  if (threadIdx.x >= 1 && i <= g.nx) {
    long long q = fidx(g, i, j, k);
    double dxhl = 2.0 / (XC(i + 1) - XC(i - 1));
#pragma unroll
    for (int m = 0; m < NV; m++) FI(fl, q, m + 1) = FI(fl, q, m + 1) + dxhl * (sf[m][threadIdx.x] - sf[m][threadIdx.x - 1]);
  }
#undef XC
}

template <int NS, int DIR>
__global__ void __launch_bounds__(128) k_visc_yz(DevCtx c, const double *__restrict__ wa, double *__restrict__ fl, int chunk) {
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
  double prev[NV], cur[NV], hl[NS];
  {
    int f = c0 - 1;
    long long p = DIR == 1 ? gidx(g, i, f, tr) : gidx(g, i, tr, f);
    visc_face<NS>(c, wa, p, p + st, XC(f + 1) - XC(f), hl, false, prev);
  }
  for (int f = c0; f <= c1; f++) {
    long long p = DIR == 1 ? gidx(g, i, f, tr) : gidx(g, i, tr, f);
    visc_face<NS>(c, wa, p, p + st, XC(f + 1) - XC(f), hl, true, cur);
    long long q = DIR == 1 ? fidx(g, i, f, tr) : fidx(g, i, tr, f);
    double dxhl = 2.0 / (XC(f + 1) - XC(f - 1));
#pragma unroll
    for (int m = 0; m < NV; m++) {
      FI(fl, q, m + 1) = FI(fl, q, m + 1) + dxhl * (cur[m] - prev[m]);
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

template <int NS>
static int visc_t(const DevCtx &c, cudaStream_t s, int dir, const double *wa, double *fl) {
  const DevGrid &g = c.g;
  if (dir == 0) {
    dim3 grid((g.nx + 1 + 126) / 127, g.ny, g.nz);
    k_visc_x<NS><<<grid, 128, 0, s>>>(c, wa, fl);
  } else {
    int chunk = 16;
    int n = dir == 1 ? g.ny : g.nz;
    dim3 grid((g.nx + 127) / 128, dir == 1 ? g.nz : g.ny, (n + chunk - 1) / chunk);
    if (dir == 1) k_visc_yz<NS, 1><<<grid, 128, 0, s>>>(c, wa, fl, chunk);
    else k_visc_yz<NS, 2><<<grid, 128, 0, s>>>(c, wa, fl, chunk);
  }
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
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
