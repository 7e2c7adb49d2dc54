// stx_chem.cu -- stiff chemistry cell updates (sm_100a).
//
//  * rosenbrock_krylov_kernel (ROK4, kernels_gpu.F90:10360-11205)
//  * rosenbrock_kernel (full-Jacobian 4-stage Rosenbrock, :8928-9501)
//  * compute_chemistry_cuf (explicit source, :9503-9674)
//
// Work per cell is uneven (adaptive sub-steps), so the Rosenbrock kernels run as
// a persistent grid (a few CTAs per SM) in which every thread repeatedly claims
// the next cell from a device counter (warp-aggregated atomicAdd) until all
// cells are done.  Each cell is integrated by exactly the same sequence of
// operations as the reference, so the result is independent of the schedule.
// This file is compiled without FMA contraction so that its arithmetic matches
// the FP64 oracle operation by operation (libm vs CUDA exp/pow/log10 aside).
#include "stx_chem.cuh"

// CTAs per SM the ROK4 kernel's register budget is sized for
#ifndef STX_ROK4_MINB
#define STX_ROK4_MINB 4
#endif

// cg: a device-resident copy of c.  The right-hand side is one out-of-line
// function that takes the context by reference; given the kernel parameter c,
// every thread would keep its own local copy of the whole context (~0.9 KB),
// given cg all threads read the one copy through L1.
template <int NS>
__global__ void __launch_bounds__(chem_block(NS), STX_ROK4_MINB)
    k_rok4(DevCtx c, const DevCtx *__restrict__ cg, double *__restrict__ w, const double *__restrict__ wa,
           const double *__restrict__ fl_sav, double dttry, double t0, double t1, int simpler,
           unsigned int *counter) {
  const DevGrid &g = c.g;
  const int NV = NS + 4;
  const double eps_Z = 5e-4;
  if (c.p.dt_d) dttry = dttry * *c.p.dt_d;   // captured CFL-driven step: dttry holds the splitting's factor
  if (c.p.time_d) {                 // captured step: the window starts at the device-held time
    t0 = *c.p.time_d;
    t1 = t0 + dttry;
  }
  // counter == nullptr: the plain launch, one thread per cell (cell = global
  // thread index) and no work stealing; otherwise the persistent grid claims cells
  const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  for (bool first = true;; first = false) {
    long long cell = counter ? claim(counter) : (first ? gt : g.npi);
    if (cell >= g.npi) break;
    int i = 1 + (int)(cell % g.nx);
    long long r = cell / g.nx;
    int j = 1 + (int)(r % g.ny);
    int k = 1 + (int)(r / g.ny);
    long long p = gidx(g, i, j, k);
    double Z = FG(wa, p, NS + 12);
    if (!(Z > eps_Z && Z < 1.0 - eps_Z)) continue;
    double VEC[NV];
#pragma unroll
    for (int m = 0; m < NV; m++) VEC[m] = FG(w, p, m + 1);
    rok4_cell<NS>(*cg, VEC, FG(wa, p, NS + 5), simpler == 1 ? fl_sav + cell : nullptr, g.npi, dttry, t0, t1,
                  simpler);
#pragma unroll
    for (int m = 0; m < NV; m++) FG(w, p, m + 1) = VEC[m];
  }
}

// n independent adiabatic constant-pressure 0-D reactors, one thread each,
// claimed from the work-stealing counter (reactors ignite at very different
// times, so their step counts differ by orders of magnitude).  Y0 / Y are
// (n, ns) with the reactor index fastest.  cg: the device-resident context (the
// right-hand side takes it by reference, see k_rok4); maxsteps: the step cap.
// A: the storage of the Krylov basis and stage vectors (double; float for the
// FP32/FP64-split form, rok4_core).
template <int NS, typename A = double>
__global__ void __launch_bounds__(chem_block(NS), STX_ROK4_MINB)
    k_batch0d(const DevCtx *__restrict__ cg, int maxsteps, int n, const double *__restrict__ T0,
              const double *__restrict__ p0,
              const double *__restrict__ Y0, double t_max, double dttry, double ign_factor, double end_factor,
              double *__restrict__ Y, double *__restrict__ T, double *__restrict__ t_ign, double *__restrict__ t_end,
              int *__restrict__ nsteps, unsigned int *counter) {
  const DevCtx &c = *cg;
  for (;;) {
    long long r = claim(counter);
    if (r >= n) break;
    double VEC[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) VEC[k] = Y0[(long long)k * n + r];
    const double T0r = T0[r];
    double h = 0.0;
#pragma unroll 1
    for (int k = 0; k < NS; k++) h = h + VEC[k] * species_poly_int(c.t, c.t.cpi, T0r, k + 1);
    Rok4ConstP<NS> f{c, h, p0[r], T0r, ign_factor, end_factor, -1.0, 0.0, T0r, 0};
    rok4_core<NS, Rok4ConstP<NS>, A>(c, f, VEC, T0r, nullptr, 0, dttry, 0.0, t_max, 0, maxsteps);
#pragma unroll
    for (int k = 0; k < NS; k++) Y[(long long)k * n + r] = VEC[k];
    T[r] = f.T_final;
    t_ign[r] = f.t_ign;
    t_end[r] = f.time_reached;
    __threadfence_system();   // nsteps last (see k_batch0d_w)
    nsteps[r] = f.steps;
  }
}

// ---------------------------------------------------------------- full Jacobian
// rosenbrock_rhs (kernels_gpu.F90:9195-9381): updates the cell state in place.
// The production terms run over the per-reaction sparse stoichiometry lists
// (chem_source_sp: the same terms in the same order as the dense species
// loops, so the same bits) with per-thread rows in shared memory: launch with
// chem_block(NS) threads.  At 53 species / 325 reactions the dense loops read
// 3 x 53 stoichiometric coefficients per reaction for a handful of non-zeros.
template <int NS>
__device__ void ros_rhs(const DevCtx &c, double *wc, double *Y, double &T, double *rhs) {
  const DevTab &t = c.t;
  double conc[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) wc[k] = wc[k] > 0.0 ? wc[k] : 0.0;
  double rho = wc[0];
#pragma unroll
  for (int k = 1; k < NS; k++) rho = rho + wc[k];
  double ri = 1.0 / rho;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    Y[k] = wc[k] * ri;
    conc[k] = rho * Y[k] / ldg(t.mw + k);
  }
  double uu = wc[NS] * ri, vv = wc[NS + 1] * ri, ww = wc[NS + 2] * ri;
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double ee = wc[NS + 3] * ri - qq;
  T = temp_from_e<NS>(t, c.p, ee, T, Y);
#pragma unroll
  for (int m = 0; m < NS + 4; m++) rhs[m] = 0.0;
  constexpr int CB = chem_block(NS);
  __shared__ double s_conc[NS * CB], s_rhs[NS * CB];
  double *cs = s_conc + threadIdx.x, *rs = s_rhs + threadIdx.x;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    cs[k * CB] = conc[k];
    rs[k * CB] = 0.0;
  }
  chem_source_sp<NS, CB>(t, T, cs, rs);
#pragma unroll
  for (int k = 0; k < NS; k++) rhs[k] = rs[k * CB];
}

template <int NV>
__device__ void lu_full(double *a, int *indx) {
#define AM(r, s) a[((s) - 1) * NV + (r) - 1]
  const double tiny = 1.5e-16;
  double vv[NV];
  for (int i = 1; i <= NV; i++) {
    double amax = 0.0;
    for (int j = 1; j <= NV; j++) if (fabs(AM(i, j)) > amax) amax = fabs(AM(i, j));
    if (amax < tiny) return;
    vv[i - 1] = 1.0 / amax;
  }
  for (int j = 1; j <= NV; j++) {
    for (int i = 1; i <= j - 1; i++) {
      double summ = AM(i, j);
      for (int k = 1; k <= i - 1; k++) summ = summ - AM(i, k) * AM(k, j);
      AM(i, j) = summ;
    }
    double amax = 0.0;
    int imax = j;
    for (int i = j; i <= NV; i++) {
      double summ = AM(i, j);
      for (int k = 1; k <= j - 1; k++) summ = summ - AM(i, k) * AM(k, j);
      AM(i, j) = summ;
      double dum = vv[i - 1] * fabs(summ);
      if (dum >= amax) { imax = i; amax = dum; }
    }
    if (j != imax) {
      for (int k = 1; k <= NV; k++) { double dum = AM(imax, k); AM(imax, k) = AM(j, k); AM(j, k) = dum; }
      vv[imax - 1] = vv[j - 1];
    }
    indx[j - 1] = imax;
    if (fabs(AM(j, j)) < tiny) AM(j, j) = tiny;
    if (j != NV) {
      double dum = 1.0 / AM(j, j);
      for (int i = j + 1; i <= NV; i++) AM(i, j) = AM(i, j) * dum;
    }
  }
}
template <int NV>
__device__ void lu_solve(const double *a, const int *indx, double *b) {
  int ii = 0;
  for (int i = 1; i <= NV; i++) {
    int ll = indx[i - 1];
    double summ = b[ll - 1];
    b[ll - 1] = b[i - 1];
    if (ii != 0) { for (int j = ii; j <= i - 1; j++) summ = summ - AM(i, j) * b[j - 1]; }
    else if (summ != 0.0) ii = i;
    b[i - 1] = summ;
  }
  for (int i = NV; i >= 1; i--) {
    double summ = b[i - 1];
    if (i < NV) for (int j = i + 1; j <= NV; j++) summ = summ - AM(i, j) * b[j - 1];
    b[i - 1] = summ / AM(i, i);
  }
#undef AM
}

template <int NS>
__device__ void rosenbrock_cell(const DevCtx &c, double *wc, double *Y, double &T, double dttry, double time_start,
                                double time_end) {
  const int NV = NS + 4;
  const double safety = 0.9, grow = 1.5, pgrow = -0.25, shrnk = 0.5, pshrnk = -1.0 / 3.0, errcon = 0.1296;
  const double gam = 1.0 / 2.0, a21 = 2.0, a31 = 48.0 / 25.0, a32 = 6.0 / 25.0;
  const double c21 = -8.0, c31 = 372.0 / 25.0, c32 = 12.0 / 5.0;
  const double c41 = -112.0 / 125.0, c42 = -54.0 / 125.0, c43 = -2.0 / 5.0;
  const double b1 = 19.0 / 9.0, b2 = 1.0 / 2.0, b3 = 25.0 / 108.0, b4 = 125.0 / 108.0;
  const double e1 = 17.0 / 54.0, e2 = 7.0 / 36.0, e3 = 0.0, e4 = 125.0 / 108.0;
  double jac[NV * NV], amat[NV * NV], w_sav[NV], rhs_sav[NV], yscal[NV], err[NV];
  double rhs[NV], g1[NV], g2[NV], g3[NV], g4[NV];
  int indx[NV];
  int finish = 0;
  double time = time_start, dt = dttry, itol = 1.0 / c.p.ros_eps, dtnext = dt;
  for (int iter = 1; iter <= c.p.ros_maxsteps; iter++) {
    double t0 = time;
    for (int n = 0; n < NV; n++) {
      double rp[NV];
      double wtmp = wc[n];
      double h = wtmp * 1.0e-06 + 1.0e-14;
      wc[n] = wtmp + h;
      ros_rhs<NS>(c, wc, Y, T, rp);
      wc[n] = wtmp - h;
      ros_rhs<NS>(c, wc, Y, T, rhs);
      wc[n] = wtmp;
      for (int m = 0; m < NV; m++) jac[n * NV + m] = (rp[m] - rhs[m]) / (2.0 * h);
    }
    ros_rhs<NS>(c, wc, Y, T, rhs_sav);
    for (int m = 0; m < NV; m++) { w_sav[m] = wc[m]; yscal[m] = dmax_(1.0, fabs(w_sav[m])); }
    bool accepted = false;
    for (int jtry = 1; jtry <= c.p.ros_maxtry; jtry++) {
      for (int n = 0; n < NV; n++) {
        for (int m = 0; m < NV; m++) amat[n * NV + m] = -jac[n * NV + m];
        amat[n * NV + n] = amat[n * NV + n] + 1.0 / (gam * dt);
      }
      for (int q = 0; q < NV; q++) indx[q] = q + 1;
      lu_full<NV>(amat, indx);
      for (int m = 0; m < NV; m++) g1[m] = rhs_sav[m];
      lu_solve<NV>(amat, indx, g1);
      for (int m = 0; m < NV; m++) wc[m] = w_sav[m] + a21 * g1[m];
      time = t0 + 1.0 * dt;
      ros_rhs<NS>(c, wc, Y, T, rhs);
      for (int m = 0; m < NV; m++) g2[m] = rhs[m] + c21 * g1[m] / dt;
      lu_solve<NV>(amat, indx, g2);
      for (int m = 0; m < NV; m++) wc[m] = w_sav[m] + a31 * g1[m] + a32 * g2[m];
      time = t0 + (3.0 / 5.0) * dt;
      ros_rhs<NS>(c, wc, Y, T, rhs);
      for (int m = 0; m < NV; m++) g3[m] = rhs[m] + (c31 * g1[m] + c32 * g2[m]) / dt;
      lu_solve<NV>(amat, indx, g3);
      for (int m = 0; m < NV; m++) g4[m] = rhs[m] + (c41 * g1[m] + c42 * g2[m] + c43 * g3[m]) / dt;
      lu_solve<NV>(amat, indx, g4);
      for (int m = 0; m < NV; m++) {
        wc[m] = w_sav[m] + b1 * g1[m] + b2 * g2[m] + b3 * g3[m] + b4 * g4[m];
        err[m] = e1 * g1[m] + e2 * g2[m] + e3 * g3[m] + e4 * g4[m];
      }
      time = t0 + dt;
      double errmax = 0.0;
      for (int m = 0; m < NV; m++) errmax = dmax_(errmax, fabs(err[m] / yscal[m]));
      errmax = errmax * itol;
      if (errmax < 1.0 || finish == 1) {
        dtnext = (errmax > errcon) ? safety * dt * pow(errmax, pgrow) : grow * dt;
        accepted = true;
        break;
      } else {
        dtnext = safety * dt * pow(errmax, pshrnk);
        double mag = dmax_(fabs(dtnext), shrnk * fabs(dt));
        dt = dt >= 0 ? mag : -mag;
      }
    }
    if (!accepted) set_status(c.p, STX_ST_ROS_TRY_CAP);
    double remaining = time_end - time;
    if (finish == 1 || remaining < 1.0e-012 * time_end) break;
    if (dtnext * 1.5 > remaining) { dt = remaining; finish = 1; }
    else { dt = dtnext; finish = 0; }
    if (iter == c.p.ros_maxsteps) set_status(c.p, STX_ST_ROS_STEPS_CAP);
  }
}

template <int NS>
__global__ void __launch_bounds__(chem_block(NS)) k_rosenbrock(DevCtx c, double *__restrict__ w, double *__restrict__ wa,
                                                    double dttry, double t0, double t1, unsigned int *counter) {
  const DevGrid &g = c.g;
  const int NV = NS + 4;
  if (c.p.dt_d) dttry = dttry * *c.p.dt_d;   // captured CFL-driven step: dttry holds the splitting's factor
  if (c.p.time_d) {                 // captured step: the window starts at the device-held time
    t0 = *c.p.time_d;
    t1 = t0 + dttry;
  }
  for (;;) {
    long long cell = claim(counter);
    if (cell >= g.npi) break;
    int i = 1 + (int)(cell % g.nx);
    long long r = cell / g.nx;
    int j = 1 + (int)(r % g.ny);
    int k = 1 + (int)(r / g.ny);
    long long p = gidx(g, i, j, k);
    double wc[NV], Y[NS], T;
    for (int m = 0; m < NV; m++) wc[m] = FG(w, p, m + 1);
    for (int m = 0; m < NS; m++) Y[m] = FG(wa, p, m + 1);
    T = FG(wa, p, NS + 5);
    rosenbrock_cell<NS>(c, wc, Y, T, dttry, t0, t1);
    for (int m = 0; m < NV; m++) FG(w, p, m + 1) = wc[m];
    for (int m = 0; m < NS; m++) FG(wa, p, m + 1) = Y[m];
    FG(wa, p, NS + 5) = T;
  }
}

// compute_chemistry_cuf (kernels_gpu.F90:9503-9674)
template <int NS>
__global__ void __launch_bounds__(128) k_chem_explicit(DevCtx c, double *__restrict__ w, double *__restrict__ wa,
                                                       double *__restrict__ fl) {
  const DevGrid &g = c.g;
  long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= g.npi) return;
  int i = 1 + (int)(tid % g.nx);
  long long r = tid / g.nx;
  int j = 1 + (int)(r % g.ny);
  int k = 1 + (int)(r / g.ny);
  long long p = gidx(g, i, j, k);
  double Y[NS], conc[NS], wl[NS];
#pragma unroll
  for (int s = 0; s < NS; s++) {
    double v = FG(w, p, s + 1);
    double vc = v > 0.0 ? v : 0.0;
    if (__double_as_longlong(vc) != __double_as_longlong(v)) FG(w, p, s + 1) = vc;
    wl[s] = vc;
  }
  double rho = wl[0];
#pragma unroll
  for (int s = 1; s < NS; s++) rho = rho + wl[s];
  double ri = 1.0 / rho;
#pragma unroll
  for (int s = 0; s < NS; s++) {
    Y[s] = wl[s] * ri;
    FG(wa, p, s + 1) = Y[s];
    conc[s] = rho * Y[s] / ldg(c.t.mw + s);
  }
  double uu = FG(w, p, NS + 1) * ri, vv = FG(w, p, NS + 2) * ri, ww = FG(w, p, NS + 3) * ri;
  double rhoe = FG(w, p, NS + 4);
  double qq = 0.5 * (uu * uu + vv * vv + ww * ww);
  double ee = rhoe * ri - qq;
  double tt = temp_from_e<NS>(c.t, c.p, ee, FG(wa, p, NS + 5), Y);
  FG(wa, p, NS + 5) = tt;
  double src[NS + 4];
#pragma unroll
  for (int s = 0; s < NS; s++) src[s] = FI(fl, tid, s + 1);
  chem_source<NS>(c.t, tt, conc, src, true);
#pragma unroll
  for (int s = 0; s < NS; s++) FI(fl, tid, s + 1) = src[s];
}

// persistent grid: want CTAs per SM (0 or above the occupancy limit: the limit)
static int persistent_blocks(const void *fn, int block, int want = 0) {
  int dev = 0, nsm = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, block, 0);
  if (per < 1) per = 1;
  if (want > 0 && want < per) per = want;
  return nsm * per;
}

int chem_ctas_limit(int ns) {
  int per = 1;
  switch (ns) {
#define X(N) case N: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)k_rok4<N>, chem_block(N), 0); break;
    STX_FOR_NS(X)
#undef X
    default: return 0;
  }
  return per < 1 ? 1 : per;
}

template <int NS>
static int rok4_t(const DevCtx &c, const DevCtx *cg, cudaStream_t s, double *w, const double *wa, const double *fl_sav,
                  double dttry, double t0, double t1, int simpler, unsigned int *counter) {
  long long need = (c.g.npi + chem_block(NS) - 1) / chem_block(NS);
  if (c.p.chem_ctas_per_sm < 0) {            // the plain launch: a thread per cell, no work stealing
    k_rok4<NS><<<(unsigned)need, chem_block(NS), 0, s>>>(c, cg, w, wa, fl_sav, dttry, t0, t1, simpler, nullptr);
    STX_CUDA_TRY(cudaGetLastError());
    return STX_OK;
  }
  STX_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned int), s));
  int nb = persistent_blocks((const void *)k_rok4<NS>, chem_block(NS), c.p.chem_ctas_per_sm);
  if (nb > need) nb = (int)need;
  k_rok4<NS><<<nb, chem_block(NS), 0, s>>>(c, cg, w, wa, fl_sav, dttry, t0, t1, simpler, counter);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

template <int NS>
static int ros_t(const DevCtx &c, cudaStream_t s, double *w, double *wa, double dttry, double t0, double t1,
                 unsigned int *counter) {
  STX_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned int), s));
  constexpr int CB = chem_block(NS);
  int nb = persistent_blocks((const void *)k_rosenbrock<NS>, CB);
  long long need = (c.g.npi + CB - 1) / CB;
  if (nb > need) nb = (int)need;
  k_rosenbrock<NS><<<nb, CB, 0, s>>>(c, w, wa, dttry, t0, t1, counter);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_rok4(const DevCtx &c, const DevCtx *cg, cudaStream_t s, double *w, const double *wa, const double *fl_sav,
                double dttry, double t0, double t1, int simpler, unsigned int *counter) {
  switch (c.t.ns) {
#define X(N) case N: return rok4_t<N>(c, cg, s, w, wa, fl_sav, dttry, t0, t1, simpler, counter);
    STX_FOR_NS(X)
#undef X
    default: return STX_E_UNSUPPORTED;
  }
}

template <int NS>
static int batch0d_t(const DevCtx &c, const DevCtx *cg, cudaStream_t s, int n, const double *T0, const double *p0,
                     const double *Y0,
                     double t_max, double dttry, double ign, double endf, double *Y, double *T, double *t_ign,
                     double *t_end, int *nsteps, unsigned int *counter) {
  STX_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned int), s));
  // the context's mixed precision form selects the FP32/FP64-split reactors
  const bool split = c.p.mixed != 0;
  int nb = persistent_blocks(split ? (const void *)k_batch0d<NS, float> : (const void *)k_batch0d<NS>,
                             chem_block(NS));
  long long need = ((long long)n + chem_block(NS) - 1) / chem_block(NS);
  if (nb > need) nb = (int)need;
  if (c.p.batch_ctas_max > 0 && nb > c.p.batch_ctas_max) nb = c.p.batch_ctas_max;
  if (split)
    k_batch0d<NS, float><<<nb, chem_block(NS), 0, s>>>(cg, c.p.ros_maxsteps, n, T0, p0, Y0, t_max, dttry, ign, endf,
                                                       Y, T, t_ign, t_end, nsteps, counter);
  else
    k_batch0d<NS><<<nb, chem_block(NS), 0, s>>>(cg, c.p.ros_maxsteps, n, T0, p0, Y0, t_max, dttry, ign, endf, Y, T,
                                                t_ign, t_end, nsteps, counter);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}

int launch_batch0d(const DevCtx &c, const DevCtx *cg, cudaStream_t s, int n, const double *T0, const double *p0,
                   const double *Y0, double t_max, double dttry, double ign, double endf, double *Y, double *T,
                   double *t_ign, double *t_end, int *nsteps, unsigned int *counter) {
  switch (c.t.ns) {
#define X(N) case N: return batch0d_t<N>(c, cg, s, n, T0, p0, Y0, t_max, dttry, ign, endf, Y, T, t_ign, t_end, nsteps, counter);
    STX_FOR_NS(X)
#undef X
    default: return STX_E_UNSUPPORTED;
  }
}

int launch_rosenbrock(const DevCtx &c, cudaStream_t s, double *w, double *wa, double dttry, double t0, double t1,
                      unsigned int *counter) {
  switch (c.t.ns) {
#define X(N) case N: return ros_t<N>(c, s, w, wa, dttry, t0, t1, counter);
    STX_FOR_NS(X)
#undef X
    default: return STX_E_UNSUPPORTED;
  }
}

int launch_chem_explicit(const DevCtx &c, cudaStream_t s, double *w, double *wa, double *fl) {
  switch (c.t.ns) {
#define X(N) case N: k_chem_explicit<N><<<grid1d(c.g.npi, 128), 128, 0, s>>>(c, w, wa, fl); break;
    STX_FOR_NS(X)
#undef X
    default: return STX_E_UNSUPPORTED;
  }
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
}
