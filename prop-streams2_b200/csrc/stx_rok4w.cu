// stx_rok4w.cu -- the ROK4 integration (kernels_gpu.F90:10360-11205) with one
// warp per state vector, for the batched 0-D reactors.
//
// The thread-per-cell kernels suit large grids: 32 cells per warp amortise the
// Krylov algebra.  A batch of reactors is different: the reactors that ignite
// late take tens of thousands of steps, and the launch lasts as long as the
// slowest one, integrated serially by a single thread.  Here a warp integrates
// one reactor:
//  * lane m holds component m of every vector (state, Krylov basis, stages);
//    dot products and norms are warp butterfly sums (every lane obtains the
//    same bits);
//  * the right-hand side evaluates the reaction rates one reaction per lane
//    (the per-reaction arithmetic of chem_source_sp), then lane k sums its
//    species' terms in ascending reaction order from shared memory (the
//    species-major lists t.sk_*), so the production rates equal those of the
//    thread kernels bit for bit;
//  * the temperature Newton iteration and the 4 x 4 Krylov algebra run
//    redundantly in every lane.
// The dot products are summed in a different order than the sequential loops
// of the reference (rounding-level differences).  Compiled without FMA
// contraction, like the other chemistry kernels.
#include <mutex>
#include <set>
#include <utility>

#include "stx_chem.cuh"

#define WFULL 0xffffffffu
#define WNRMAX 64          // reactions per mechanism the warp kernels take (two per lane)

__device__ __forceinline__ double wsum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = x + __shfl_xor_sync(WFULL, x, o);
  return x;
}

// Warp ROK4 of one state of NV <= 32 components (lane m holds component m;
// lanes >= NV hold 0).  f.rhs(y, T, lane) returns the lane's component of the
// right-hand side; f.accept / f.done as in rok4_core.
template <int NV, class F>
__device__ void rok4_core_w(const DevCtx &c, F &f, double &v, double T_iter, double fls, double dttry,
                            double time_start, double time_end, int simpler, int lane) {
  const double gam = 0.572816062482135;
  const double alpha[4][3] = {{0, 0, 0},
                              {0.432364435748567, 0, 0},
                              {-0.514211316876170, 1.382271144617360, 0},
                              {-0.514211316876170, 1.382271144617360, 0.0}};
  const double gmc[4][3] = {{0, 0, 0},
                            {-0.602765307997356, 0, 0},
                            {-1.389195789724843, 1.072950969011413, 0},
                            {0.992356412977094, -1.390032613873701, -0.440875890223325}};
  const double bsv[4] = {0.194335256262729, 0.483167813989227, 0.0, 0.322496929748044};
  const double btv[4] = {-0.217819895945721, 1.03130847478467, 0.186511421161047, 0.0};
  double V[STX_MMAX + 1], Ks[STX_NSTAGE], inv[STX_MMAX * STX_MMAX];
  int mA = 0;
#pragma unroll
  for (int q = 0; q < STX_MMAX * STX_MMAX; q++) inv[q] = 0.0;
#pragma unroll
  for (int q = 0; q < STX_NSTAGE; q++) Ks[q] = 0.0;
  double time = time_start, dt = dttry, errn = 1.0;
  int it = 0;
  while (time < (time_end - 1.0e-12)) {
    dt = dmin_(dt, time_end - time);
    it = it + 1;
    // ---- arnoldi (:10664-10792)
    double rs;
    {
      const double TOL = 1e-6, eps = 1.0e-08;
      double HH[(STX_MMAX + 1) * STX_MMAX], HI[STX_MMAX * STX_MMAX], prj[STX_MMAX], lam[STX_MMAX];
#pragma unroll
      for (int q = 0; q < (STX_MMAX + 1) * STX_MMAX; q++) HH[q] = 0.0;
#pragma unroll
      for (int q = 0; q < STX_MMAX * STX_MMAX; q++) HI[q] = 0.0;
#pragma unroll
      for (int q = 0; q <= STX_MMAX; q++) V[q] = 0.0;
      mA = 0;
      rs = f.rhs(v, T_iter, lane);
      if (simpler == 1) rs = rs - fls;
      double nrm = sqrt(wsum(rs * rs));
      V[0] = rs / nrm;
#pragma unroll
      for (int kk = 1; kk <= STX_MMAX; kk++) {
        double jac = f.rhs(v + (eps * V[kk - 1]), T_iter, lane);
        if (simpler == 1) jac = jac - fls;
        jac = (jac - rs) / eps;
#pragma unroll
        for (int jj = 1; jj <= kk; jj++) {
          double dot = wsum(V[jj - 1] * jac);
          HH[(kk - 1) * (STX_MMAX + 1) + jj - 1] = dot;
          jac = jac - (dot * V[jj - 1]);
        }
        double hn = sqrt(wsum(jac * jac));
        HH[(kk - 1) * (STX_MMAX + 1) + kk] = hn;
        V[kk] = jac / hn;
#pragma unroll
        for (int ll = 1; ll <= STX_MMAX; ll++) prj[ll - 1] = (ll <= kk) ? wsum(V[ll - 1] * rs) : 0.0;
#pragma unroll
        for (int n = 1; n <= kk; n++)
#pragma unroll
          for (int nn = 1; nn <= kk; nn++) {
            double h = -(dt * gam * HH[(nn - 1) * (STX_MMAX + 1) + n - 1]);
            if (n == nn) h = h + 1.0;
            HI[(nn - 1) * STX_MMAX + n - 1] = h;
          }
#pragma unroll
        for (int n = kk + 1; n <= STX_MMAX; n++) HI[(n - 1) * STX_MMAX + n - 1] = 1.0;
        inv_matrix_k(HI, kk);
#pragma unroll
        for (int ll = 1; ll <= STX_MMAX; ll++) {
          double s = 0.0;
#pragma unroll
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
    // ---- stages: B F = A (Vb^T F), this lane's row of A from V and inv
    double vb[STX_MMAX];
#pragma unroll
    for (int q = 0; q < STX_MMAX; q++) vb[q] = (q < mA) ? V[q] : 0.0;
#pragma unroll
    for (int ii = 1; ii <= STX_NSTAGE; ii++) {
      double ys = v;
#pragma unroll
      for (int jj = 1; jj <= ii - 1; jj++) ys = ys + dt * alpha[ii - 1][jj - 1] * Ks[jj - 1];
      double F = f.rhs(ys, T_iter, lane);
      double GK = 0.0;
#pragma unroll
      for (int jj = 1; jj <= ii - 1; jj++) GK = GK + gmc[ii - 1][jj - 1] / gam * Ks[jj - 1];
      F = F + GK;
      if (simpler == 1) F = F - fls;
      double s = 0.0;
#pragma unroll
      for (int kk = 0; kk < STX_MMAX; kk++) {
        double pf = (kk < mA) ? wsum(V[kk] * F) : 0.0;
        double a = vb[0] * ((kk == 0 ? 1.0 : 0.0) - inv[kk * STX_MMAX + 0]);
#pragma unroll
        for (int jj = 1; jj < STX_MMAX; jj++) a = a + vb[jj] * ((jj == kk ? 1.0 : 0.0) - inv[kk * STX_MMAX + jj]);
        s = s + a * pf;
      }
      Ks[ii - 1] = F - s - GK;
    }
    double a = v, b = v;
#pragma unroll
    for (int ii = 0; ii < STX_NSTAGE; ii++) {
      a = a + dt * bsv[ii] * Ks[ii];
      b = b + dt * btv[ii] * Ks[ii];
    }
    double errv = (b - a) / ((1.0e-4) * a + 1.0e-8);
    double errmax = sqrt(wsum(errv * errv));
    double fac = 0.625 * pow(errn, 0.1) / pow(errmax, 0.175);
    double dtnext = dt * dmin_(5.0, dmax_(0.2, fac));
    if (errmax < 1.0) {
      time = time + dt;
      v = a;
      f.accept(v, time, T_iter, time_end, lane);
    }
    dt = dtnext;
    errn = errmax;
    if (it > c.p.ros_maxsteps) {
      if (lane == 0) set_status(c.p, STX_ST_ROS_STEPS_CAP);
      break;
    }
  }
  f.done(time, T_iter, it);
}

// Right-hand side of the constant-pressure reactor (cp_rhs) for the state held
// one component per lane; returns this lane's component.  sm: per-warp shared
// scratch of NS + WNRMAX doubles (concentrations, then the reaction rates).
template <int NS>
__device__ __noinline__ double cp_rhs_w(const DevCtx &c, double y, double T_iter, double h, double p, double *sm,
                                        int lane) {
  const DevTab &t = c.t;
  double Yc[NS];
#pragma unroll
  for (int k = 0; k < NS; k++) {
    double yk = __shfl_sync(WFULL, y, k);
    Yc[k] = yk > 0.0 ? yk : 0.0;
  }
  double tt = temp_from_poly<NS>(t, t.cp, c.p, h, T_iter, Yc);
  double rm = 0.0;
#pragma unroll
  for (int k = 0; k < NS; k++) rm = rm + ldg(t.rgas + k) * Yc[k];
  double rho = p / (rm * tt);
  double *conc = sm, *qr = sm + NS;
  if (lane < NS) conc[lane] = rho * (y > 0.0 ? y : 0.0) / ldg(t.mw + lane);
  __syncwarp();
  const int nr = t.nr;
  double Rtti = 1.0 / (t.Ru * tt);
  int itt;
  double dtt;
  kc_pos(t, tt, itt, dtt);
  for (int lr = lane; lr < nr; lr += 32) {
    int ty = __ldg(t.reac_ty + lr);
    double tbs = 1.0;
    if (ty != 0) {
      tbs = 0.0;
#pragma unroll 1
      for (int k = 0; k < NS; k++) tbs = tbs + ldg(t.tb_eff + (long long)k * nr + lr) * conc[k];
    }
    double kf, kb;
    rate_consts<false>(t, lr, ty, tt, Rtti, itt, dtt, tbs, kf, kb);
    const int cnt = __ldg(t.sp_cnt + lr);
    const unsigned char *ix = t.sp_idx + (long long)lr * STX_SPW;
    const double *cf = t.sp_coef + (long long)lr * STX_SPW;
    double q1 = 1.0, q2 = 1.0;
#pragma unroll 1
    for (int n = 0; n < (cnt & 255); n++) {
      double x = conc[__ldg(ix + n)], e = ldg(cf + n);
      if (e == 1.0) q1 = q1 * x;
      else q1 = q1 * stoich_pow(x, e);
    }
#pragma unroll 1
    for (int n = 0; n < ((cnt >> 8) & 255); n++) {
      double x = conc[__ldg(ix + STX_SPR + n)], e = ldg(cf + STX_SPR + n);
      if (e == 1.0) q2 = q2 * x;
      else q2 = q2 * stoich_pow(x, e);
    }
    double tb = (ty == 1) ? tbs : 1.0;
    qr[lr] = tb * (kf * q1 - kb * q2);
  }
  __syncwarp();
  double acc = 0.0;
  if (lane < NS) {
    const double mwk = ldg(t.mw + lane);
    const int n0 = __ldg(t.sk_ptr + lane), n1 = __ldg(t.sk_ptr + lane + 1);
#pragma unroll 1
    for (int n = n0; n < n1; n++) {
      double wdtkj = ldg(t.sk_c + n) * qr[__ldg(t.sk_r + n)];
      acc = acc + wdtkj * mwk;
    }
  }
  __syncwarp();
  return lane < NS ? acc / rho : 0.0;
}

template <int NS>
struct Rok4ConstPW {
  const DevCtx &c;
  double h, p, T0, ign_factor, end_factor;
  double *sm;
  double t_ign, time_reached, T_final;
  int steps;
  __device__ __forceinline__ double rhs(double y, double T_iter, int lane) const {
    return cp_rhs_w<NS>(c, y, T_iter, h, p, sm, lane);
  }
  __device__ __forceinline__ void accept(double v, double time, double &T_iter, double &time_end, int) {
    double Yc[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) {
      double yk = __shfl_sync(WFULL, v, k);
      Yc[k] = yk > 0.0 ? yk : 0.0;
    }
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

// One warp per reactor, reactors claimed from the work-stealing counter.
template <int NS>
__global__ void __launch_bounds__(128) k_batch0d_w(DevCtx c, int n, const double *__restrict__ T0,
                                                   const double *__restrict__ p0, const double *__restrict__ Y0,
                                                   double t_max, double dttry, double ign_factor, double end_factor,
                                                   double *__restrict__ Y, double *__restrict__ T,
                                                   double *__restrict__ t_ign, double *__restrict__ t_end,
                                                   int *__restrict__ nsteps, unsigned int *counter) {
  __shared__ double sm_all[4][NS + WNRMAX];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double *sm = sm_all[wid];
  for (;;) {
    unsigned int r0 = 0;
    if (lane == 0) r0 = atomicAdd(counter, 1u);
    const long long r = (long long)__shfl_sync(WFULL, r0, 0);
    if (r >= n) break;
    double v = lane < NS ? Y0[(long long)lane * n + r] : 0.0;
    const double T0r = T0[r];
    double h = 0.0;
#pragma unroll 1
    for (int k = 0; k < NS; k++) h = h + Y0[(long long)k * n + r] * species_poly_int(c.t, c.t.cpi, T0r, k + 1);
    Rok4ConstPW<NS> f{c, h, p0[r], T0r, ign_factor, end_factor, sm, -1.0, 0.0, T0r, 0};
    rok4_core_w<NS>(c, f, v, T0r, 0.0, dttry, 0.0, t_max, 0, lane);
    if (lane < NS) Y[(long long)lane * n + r] = v;
    if (lane == 0) {
      T[r] = f.T_final;
      t_ign[r] = f.t_ign;
      t_end[r] = f.time_reached;
    }
    // nsteps last, after every lane's outputs are visible system-wide: a caller
    // whose outputs are mapped host memory polls it to collect finished reactors
    __threadfence_system();
    __syncwarp();
    if (lane == 0) nsteps[r] = f.steps;
  }
}

template <int NS>
static int batch0d_w_t(const DevCtx &c, cudaStream_t s, int n, const double *T0, const double *p0, const double *Y0,
                       double t_max, double dttry, double ign, double endf, double *Y, double *T, double *t_ign,
                       double *t_end, int *nsteps, unsigned int *counter, int force) {
  if constexpr (NS > 32) {
    return STX_E_UNSUPPORTED;
  } else {
  if (c.t.nr > WNRMAX) return STX_E_UNSUPPORTED;
  int dev = 0, nsm = 148, per = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)k_batch0d_w<NS>, 128, 0);
  long long nb = (long long)nsm * (per < 1 ? 1 : per);
  long long need = ((long long)n + 3) / 4;      // four reactors (warps) per CTA
  // More reactors than resident warps: a thread per reactor finishes the batch
  // sooner (all of them run at once); the warp kernel only where every reactor
  // gets its own warp from the start, unless forced.
  if (!force && need > nb) return STX_E_UNSUPPORTED;
  STX_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned int), s));
  if (nb > need) nb = need;
  if (c.p.batch_ctas_max > 0 && nb > c.p.batch_ctas_max) nb = c.p.batch_ctas_max;   // after the choice of kernel
  k_batch0d_w<NS><<<(int)nb, 128, 0, s>>>(c, n, T0, p0, Y0, t_max, dttry, ign, endf, Y, T, t_ign, t_end, nsteps,
                                          counter);
  STX_CUDA_TRY(cudaGetLastError());
  return STX_OK;
  }
}

// The warp-per-reactor kernel (the one small, served batches take) is persistent
// and can stay resident for seconds.
// An SM holding one of their CTAs keeps its shared-memory/L1 split until the CTA
// exits, and a kernel that needs a larger shared-memory share (the staged
// convective sweeps, ~90 KB per CTA) cannot start a CTA there meanwhile; on a
// server that runs grid solves beside reactor launches those solves then wait
// for the reactors.  So the warp kernel asks for the largest shared-memory split,
// which every other kernel fits beside.  (The thread-per-reactor kernel, for
// large batches, keeps the default: its local working set needs the L1.)
template <int NS>
static void batch0d_carveout_t() {
  cudaFuncSetAttribute(k_batch0d_w<NS>, cudaFuncAttributePreferredSharedMemoryCarveout,
                       (int)cudaSharedmemCarveoutMaxShared);
}

int launch_batch0d_setup(int ns) {
  static std::mutex mu;
  static std::set<std::pair<int, int>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({dev, ns})) return STX_OK;
  switch (ns) {
#define X(N) case N: batch0d_carveout_t<N>(); break;
    STX_FOR_NS(X)
#undef X
    default: break;
  }
  done.insert({dev, ns});
  return cudaGetLastError() == cudaSuccess ? STX_OK : STX_E_CUDA;
}

int launch_batch0d_warp(const DevCtx &c, cudaStream_t s, int n, const double *T0, const double *p0, const double *Y0,
                        double t_max, double dttry, double ign, double endf, double *Y, double *T, double *t_ign,
                        double *t_end, int *nsteps, unsigned int *counter, int force) {
  switch (c.t.ns) {
#define X(N) case N: return batch0d_w_t<N>(c, s, n, T0, p0, Y0, t_max, dttry, ign, endf, Y, T, t_ign, t_end, nsteps, counter, force);
    STX_FOR_NS(X)
#undef X
    default: return STX_E_UNSUPPORTED;
  }
}
