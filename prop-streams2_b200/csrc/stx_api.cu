// stx_api.cu -- the extern "C" boundary of libstx.so (include/stx.h): context
// creation (table upload and repacking), the per-kernel entry points and the
// rk_sync / advance_solution sequencing on the caller's stream.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "stx_kernels.cuh"

struct stx_ctx {
  DevCtx d;
  stx_params par;
  int periodic[3];
  int ns, nv;
  double *winf_d;
  unsigned int *status_d;         // device status word
  unsigned int *counter_d;        // work-stealing cell counter of the Rosenbrock kernels
  unsigned long long *dt_d;       // the nine CFL maxima
  double *res_d;                  // residual partial sums (STX_RES_BLOCKS) of stx_compute_residual
  unsigned long long *mm_d;       // its six rho / T / p extrema
  double *time_d;                 // simulation time of captured steps (stx_graph_*)
  double *dtv_d;                  // step size of captured CFL-driven steps (stx_graph_create_cfl)
  const DevCtx *dctx_d;           // device copy of d, for device functions that take the context by reference
  stx_exchange_fn xfn = nullptr;   // ghost exchange at STX_BC_EXCHANGE faces (stx_set_exchange)
  void *xuser = nullptr;
  WenoScratch weno;               // listed WENO faces of the staged sweeps (cap 0: none)
  int weno_list[3];               // per sweep direction: use the listed WENO faces
  std::vector<void *> allocs;
  // The device's setup stream (setup_stream): the context's tables and scratch
  // are allocated, uploaded and freed stream-ordered on it
  // (cudaMallocFromPoolAsync / cudaFreeAsync), so creating or destroying a
  // context never waits for other work on the device (a plain cudaFree
  // synchronises the whole device).
  cudaStream_t cs = nullptr;
  cudaStream_t us = nullptr;      // stream of the creation's uploads: cs, or the caller's (stx_ctx_create_like_on)
  int device;
  // instrumentation (stx_profile_*)
  int prof_on;
  long long launches[STX_NK];
  std::vector<cudaEvent_t> ev[STX_NK];   // begin/end pairs
  size_t ev_used[STX_NK];
  double bytes[STX_NK];                  // algorithmic bytes of the timed calls
};

// algorithmic FP64 bytes per point of each kernel (every field it must read or
// write, once): ns species, nv = ns + 4
static inline double B8(double n) { return 8.0 * n; }

namespace {
// Counts the kernels an entry point launches and, with profiling on, brackets
// them with a pair of events on the launching stream.
struct Prof {
  stx_ctx *c;
  cudaStream_t s;
  int cls;
  cudaEvent_t e1 = nullptr;
  Prof(stx_ctx *c_, cudaStream_t s_, int cls_, int nlaunch, double bytes = 0.0) : c(c_), s(s_), cls(cls_) {
    c->launches[cls] += nlaunch;
    if (!c->prof_on) return;
    c->bytes[cls] += bytes;
    size_t k = c->ev_used[cls];
    while (c->ev[cls].size() < k + 2) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return;
      c->ev[cls].push_back(e);
    }
    cudaEventRecord(c->ev[cls][k], s);
    e1 = c->ev[cls][k + 1];
    c->ev_used[cls] = k + 2;
  }
  ~Prof() {
    if (e1) cudaEventRecord(e1, s);
  }
};
}  // namespace

namespace {

// The library's memory pool on a device, for context tables and scratch.  Its
// release threshold is the maximum, so memory freed by a destroyed context stays
// in the pool for the next one instead of being unmapped at the next
// synchronisation (contexts come and go while other work runs, e.g. one per
// served request).
cudaMemPool_t ctx_pool(int dev) {
  static std::mutex mu;
  static std::vector<cudaMemPool_t> pools;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)pools.size() <= dev) pools.resize(dev + 1, nullptr);
  if (!pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    pools[dev] = pool;
  }
  return pools[dev];
}

// The setup stream of a device: one non-blocking stream, created at the first
// context on the device and kept for the process, that carries only context
// set-up and tear-down (uploads, zero fills, frees, device-context refreshes).
// One stream instead of one per context: CUDA maps streams onto a fixed set of
// hardware queues (CUDA_DEVICE_MAX_CONNECTIONS), and every stream created
// beyond that shares a queue with an earlier one, whose long-running kernels
// (a persistent reactor batch runs for seconds) then hold up the set-up work
// queued behind them -- and the synchronisations that wait for it.
cudaStream_t setup_stream(int dev) {
  static std::mutex mu;
  static std::vector<cudaStream_t> streams;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)streams.size() <= dev) streams.resize(dev + 1, nullptr);
  if (!streams[dev] && cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking) != cudaSuccess)
    streams[dev] = nullptr;
  return streams[dev];
}

template <typename T>
int upload(stx_ctx *c, const T *host, size_t n, const T **out) {
  void *p = nullptr;
  if (n == 0) n = 1;
  cudaMemPool_t pool = ctx_pool(c->device);
  if (!pool || cudaMallocFromPoolAsync(&p, n * sizeof(T), pool, c->us) != cudaSuccess) return STX_E_NOMEM;
  c->allocs.push_back(p);
  // pageable host source: the copy is staged before the call returns
  if (host && cudaMemcpyAsync(p, host, n * sizeof(T), cudaMemcpyHostToDevice, c->us) != cudaSuccess) return STX_E_CUDA;
  if (!host && cudaMemsetAsync(p, 0, n * sizeof(T), c->us) != cudaSuccess) return STX_E_CUDA;
  *out = (const T *)p;
  return STX_OK;
}

bool ns_supported(int ns) {
#define X(N) if (ns == N) return true;
  STX_FOR_NS(X)
#undef X
  return false;
}

inline cudaStream_t S(void *s) { return (cudaStream_t)s; }

// mean time of reps launches of fn on s after one untimed launch, in ms (-1 on error)
template <class F>
float time_launches(cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1, int reps, F fn) {
  if (fn() != STX_OK) return -1.f;
  cudaEventRecord(e0, s);
  for (int r = 0; r < reps; r++)
    if (fn() != STX_OK) return -1.f;
  cudaEventRecord(e1, s);
  if (cudaEventSynchronize(e1) != cudaSuccess) return -1.f;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  return ms / reps;
}

}  // namespace

#define TRY(x)                 \
  do {                         \
    int rc_ = (x);             \
    if (rc_ != STX_OK) return rc_; \
  } while (0)

extern "C" {

int stx_abi_version(void) { return STX_ABI_VERSION; }

const char *stx_strerror(int code) {
  switch (code) {
    case STX_OK: return "ok";
    case STX_E_INVALID: return "invalid argument";
    case STX_E_CUDA: return "CUDA runtime error";
    case STX_E_NOMEM: return "device allocation failed";
    case STX_E_UNSUPPORTED: return "option outside the supported hot path";
    case STX_E_TOO_LARGE: return "more cells than the allocation-free entry point's fixed scratch allows (2^31)";
    case STX_E_LOCAL_MEM:
      return "the device's per-thread stack limit (cudaLimitStackSize) is below the allocation-free kernel's local "
             "frame; raise it once with cudaDeviceSetLimit before calling";
    default: return "unknown error";
  }
}

int stx_ctx_destroy(stx_ctx *c) {
  if (!c) return STX_E_INVALID;
  // stream-ordered frees on the setup stream, without waiting for them: the
  // caller has finished its work on the context (its own streams are
  // synchronised), and the pool hands the memory out again only to allocations
  // ordered after the frees
  if (c->cs)
    for (void *p : c->allocs) cudaFreeAsync(p, c->cs);
  for (int k = 0; k < STX_NK; k++)
    for (cudaEvent_t e : c->ev[k]) cudaEventDestroy(e);
  delete c;
  return STX_OK;
}

}  // extern "C"

// A context from host tables (base null) or on the device tables of base.
// on: the stream of the uploads (nullptr: the setup stream, and the call
// returns when they have completed)
static int ctx_create_impl(const stx_params *par, const stx_tables *tab, const stx_grid *grid, const stx_ctx *base,
                           cudaStream_t on, stx_ctx **out) {
  if (!par || !(tab || base) || !grid || !out) return STX_E_INVALID;
  *out = nullptr;
  const int ns = base ? base->ns : tab->ns, nr = base ? base->d.t.nr : tab->nr;
  if (!ns_supported(ns)) return STX_E_UNSUPPORTED;
  if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || grid->ng < 1 || grid->ng > 4) return STX_E_INVALID;
  if (par->nv_aux < 2 * ns + 13) return STX_E_INVALID;
  if (par->weno_scheme < 1 || par->weno_scheme > 4) return STX_E_INVALID;
  if (par->ep_order < 2 || par->ep_order > 8 || (par->ep_order & 1)) return STX_E_INVALID;
  if (par->visc_order < 2 || par->visc_order > 8 || (par->visc_order & 1)) return STX_E_INVALID;
  if (par->conservative_viscous != 1) return STX_E_UNSUPPORTED;
  // every stencil (central ep_order/2, viscous visc_order/2, WENO weno_scheme) must fit in the ghost layers
  if (par->ep_order / 2 > grid->ng || par->visc_order / 2 > grid->ng || par->weno_scheme > grid->ng) return STX_E_INVALID;
  if (par->nrk < 1 || par->nrk > 4) return STX_E_INVALID;
  for (int q = 0; q < 6; q++) {
    int t = par->bctags[q], nr = par->bctags_nr[q];
    // update_ghost tags of this path (multideal_gpu.F90:1176-1233); 9 (laminar-profile
    // inflow), 10 (recycling), 26/28 (jets) and 46/56 (special walls) are not
    if (t != 0 && t != 1 && t != 2 && t != 4 && t != 5 && t != 6 && t != 7 && t != 8 && t != STX_BC_EXCHANGE)
      return STX_E_UNSUPPORTED;
    if (nr != 0 && nr != 1 && nr != 2 && nr != 3 && nr != 6) return STX_E_UNSUPPORTED;
    if (nr != 0 && (t == 0 || t == STX_BC_EXCHANGE)) return STX_E_INVALID;   // no characteristic face inside the domain
    if (nr == 3 && !par->winf) return STX_E_INVALID;
  }
  // bc_preproc (multideal.F90:5671-5718): a face with a characteristic treatment
  // leaves its boundary cells out of the convective flux divergence
  {
    const int lo[3] = {1, 1, 1}, hi[3] = {grid->nx, grid->ny, grid->nz};
    const int got[6] = {par->eul_imin, par->eul_imax, par->eul_jmin, par->eul_jmax, par->eul_kmin, par->eul_kmax};
    for (int q = 0; q < 6; q++) {
      int want = (q % 2 == 0 ? lo[q / 2] : hi[q / 2]) + (par->bctags_nr[q] != 0 ? (q % 2 == 0 ? 1 : -1) : 0);
      if (got[q] != want) return STX_E_UNSUPPORTED;
    }
  }
  if (!base && (tab->nsetcv < 1 || tab->num_t_tab < 1)) return STX_E_INVALID;
  if (par->enable_chemistry > 0 && nr < 1) return STX_E_INVALID;
  stx_ctx *c = new (std::nothrow) stx_ctx();
  if (!c) return STX_E_NOMEM;
  cudaGetDevice(&c->device);
  c->cs = setup_stream(c->device);
  if (!c->cs) {
    delete c;
    return STX_E_CUDA;
  }
  c->us = on ? on : c->cs;
  c->par = *par;
  c->ns = ns;
  c->nv = ns + 4;
  for (int d = 0; d < 3; d++) c->periodic[d] = par->bctags[2 * d] == 0;
  DevCtx &d = c->d;
  DevTab &t = d.t;
  DevGrid &g = d.g;
  DevPar &p = d.p;
  int rc = STX_OK;
  auto fail = [&](int code) { stx_ctx_destroy(c); return code; };
  // ---- tables (shared: base's device copies, which base keeps)
  if (base) {
    t = base->d.t;
  } else {
  t.ns = ns; t.nr = nr; t.icl = tab->indx_cp_l; t.icr = tab->indx_cp_r; t.nset = tab->nsetcv; t.ntab = tab->num_t_tab;
  t.ncp = t.icr - t.icl + 3; t.tmin = tab->t_min_tab; t.dtab = tab->dt_tab; t.Ru = tab->R_univ;
  const size_t ntab1 = (size_t)tab->num_t_tab + 1;
  if ((rc = upload(c, tab->mw, ns, &t.mw))) return fail(rc);
  if ((rc = upload(c, tab->mwinv, ns, &t.mwinv))) return fail(rc);
  if ((rc = upload(c, tab->rgas, ns, &t.rgas))) return fail(rc);
  if ((rc = upload(c, tab->trange, (size_t)ns * (t.nset + 1), &t.trange))) return fail(rc);
  if ((rc = upload(c, tab->cp_coeff, (size_t)t.ncp * ns * t.nset, &t.cp))) return fail(rc);
  if ((rc = upload(c, tab->cv_coeff, (size_t)t.ncp * ns * t.nset, &t.cv))) return fail(rc);
  {
    // integrated tables: coef_l / (l + 1) for the terms l >= 0 of h(T) and e(T)
    // (the quotient the reference forms per evaluation, get_species_h_from_temperature_dev)
    const size_t ncoef = (size_t)t.ncp * ns * t.nset;
    std::vector<double> hi(tab->cp_coeff, tab->cp_coeff + ncoef), ei(tab->cv_coeff, tab->cv_coeff + ncoef);
    for (size_t q = 0; q < ncoef; q++) {
      const int l = t.icl + (int)(q % (size_t)t.ncp);
      if (l >= 0 && l <= t.icr) {
        hi[q] = tab->cp_coeff[q] / (l + 1.0);
        ei[q] = tab->cv_coeff[q] / (l + 1.0);
      }
    }
    if ((rc = upload(c, hi.data(), ncoef, &t.cpi))) return fail(rc);
    if ((rc = upload(c, ei.data(), ncoef, &t.cvi))) return fail(rc);
  }
  {
    // repack the 1-K tables row-major in temperature so one point reads two contiguous rows
    std::vector<double> vr(ntab1 * ns), lr(ntab1 * ns), dr(ntab1 * ns * ns);
    for (size_t it = 0; it < ntab1; it++)
      for (int k = 0; k < ns; k++) {
        vr[it * ns + k] = tab->visc[(size_t)k * ntab1 + it];
        lr[it * ns + k] = tab->lambda[(size_t)k * ntab1 + it];
        for (int m = 0; m < ns; m++) dr[(it * ns + k) * ns + m] = tab->diffbin[((size_t)m * ns + k) * ntab1 + it];
      }
    if ((rc = upload(c, vr.data(), vr.size(), &t.visc_r))) return fail(rc);
    if ((rc = upload(c, lr.data(), lr.size(), &t.lam_r))) return fail(rc);
    if ((rc = upload(c, dr.data(), dr.size(), &t.diff_r))) return fail(rc);
    std::vector<double> wa((size_t)ns * ns), wb((size_t)ns * ns);
    for (int l = 0; l < ns; l++)
      for (int m = 0; m < ns; m++) {
        wa[l * ns + m] = 1.0 / std::sqrt(1.0 + tab->mw[l] * tab->mwinv[m]);
        wb[l * ns + m] = std::pow(tab->mw[m] * tab->mwinv[l], 0.25);
      }
    if ((rc = upload(c, wa.data(), wa.size(), &t.wk_a))) return fail(rc);
    if ((rc = upload(c, wb.data(), wb.size(), &t.wk_b))) return fail(rc);
  }
  if (nr > 0) {
    if ((rc = upload(c, tab->reac_ty, nr, &t.reac_ty))) return fail(rc);
    if ((rc = upload(c, tab->is_rev, nr, &t.is_rev))) return fail(rc);
    if ((rc = upload(c, tab->arr_a, (size_t)nr * 2, &t.arr_a))) return fail(rc);
    if ((rc = upload(c, tab->arr_b, (size_t)nr * 2, &t.arr_b))) return fail(rc);
    if ((rc = upload(c, tab->arr_ea, (size_t)nr * 2, &t.arr_ea))) return fail(rc);
    if ((rc = upload(c, tab->falloff, (size_t)nr * 5, &t.falloff))) return fail(rc);
    if ((rc = upload(c, tab->tb_eff, (size_t)nr * ns, &t.tb_eff))) return fail(rc);
    if ((rc = upload(c, tab->r_coeffs, (size_t)nr * ns, &t.r_coeffs))) return fail(rc);
    if ((rc = upload(c, tab->p_coeffs, (size_t)nr * ns, &t.p_coeffs))) return fail(rc);
    {
      // sparse stoichiometry: the species with nonzero nu' / nu'' of each
      // reaction, ascending, so the rate kernels visit exactly the terms the
      // dense species loops would, in the same order
      std::vector<int> cnt(nr);
      std::vector<unsigned char> idx((size_t)nr * STX_SPW, 0);
      std::vector<double> coef((size_t)nr * STX_SPW, 0.0);
      for (int r = 0; r < nr; r++) {
        int nR = 0, nP = 0, nU = 0;
        for (int k = 0; k < ns; k++) {
          double rr = tab->r_coeffs[(size_t)k * nr + r], pp = tab->p_coeffs[(size_t)k * nr + r];
          if (rr != 0.0) {
            if (nR == STX_SPR) return fail(STX_E_UNSUPPORTED);
            idx[(size_t)r * STX_SPW + nR] = (unsigned char)k;
            coef[(size_t)r * STX_SPW + nR++] = rr;
          }
          if (pp != 0.0) {
            if (nP == STX_SPR) return fail(STX_E_UNSUPPORTED);
            idx[(size_t)r * STX_SPW + STX_SPR + nP] = (unsigned char)k;
            coef[(size_t)r * STX_SPW + STX_SPR + nP++] = pp;
          }
          if (rr != 0.0 || pp != 0.0) {
            idx[(size_t)r * STX_SPW + 2 * STX_SPR + nU] = (unsigned char)k;
            coef[(size_t)r * STX_SPW + 2 * STX_SPR + nU++] = pp - rr;
          }
        }
        cnt[r] = nR | (nP << 8) | (nU << 16);
      }
      if ((rc = upload(c, cnt.data(), cnt.size(), &t.sp_cnt))) return fail(rc);
      if ((rc = upload(c, idx.data(), idx.size(), &t.sp_idx))) return fail(rc);
      if ((rc = upload(c, coef.data(), coef.size(), &t.sp_coef))) return fail(rc);
      // by species: the reactions a species takes part in (rr or pp nonzero), ascending
      std::vector<int> kptr(ns + 1, 0), kr;
      std::vector<double> kc;
      for (int k = 0; k < ns; k++) {
        for (int r = 0; r < nr; r++) {
          double rr = tab->r_coeffs[(size_t)k * nr + r], pp = tab->p_coeffs[(size_t)k * nr + r];
          if (rr != 0.0 || pp != 0.0) {
            kr.push_back(r);
            kc.push_back(pp - rr);
          }
        }
        kptr[k + 1] = (int)kr.size();
      }
      if ((rc = upload(c, kptr.data(), kptr.size(), &t.sk_ptr))) return fail(rc);
      if ((rc = upload(c, kr.data(), kr.size(), &t.sk_r))) return fail(rc);
      if ((rc = upload(c, kc.data(), kc.size(), &t.sk_c))) return fail(rc);
    }
    std::vector<double> kr(ntab1 * nr);
    for (size_t it = 0; it < ntab1; it++)
      for (int r = 0; r < nr; r++) kr[it * nr + r] = tab->kc_tab[(size_t)r * ntab1 + it];
    if ((rc = upload(c, kr.data(), kr.size(), &t.kc_r))) return fail(rc);
  }
  t.n_eoi = tab->n_eoi;
  if (t.n_eoi != 1) {
    if (t.n_eoi < 1 || !tab->aw_eoi || !tab->coeff_eoi || !tab->beta0 || !tab->nainsp) return fail(STX_E_INVALID);
    if ((rc = upload(c, tab->aw_eoi, t.n_eoi, &t.aw_eoi))) return fail(rc);
    if ((rc = upload(c, tab->coeff_eoi, t.n_eoi, &t.coeff_eoi))) return fail(rc);
    if ((rc = upload(c, tab->beta0, 2, &t.beta0))) return fail(rc);
    if ((rc = upload(c, tab->nainsp, (size_t)ns * t.n_eoi, &t.nainsp))) return fail(rc);
  }
  }  // host tables
  // ---- grid: the nine coordinate and metric arrays in one upload
  g.nx = grid->nx; g.ny = grid->ny; g.nz = grid->nz; g.ng = grid->ng;
  g.nxg = g.nx + 2 * g.ng; g.nyg = g.ny + 2 * g.ng; g.nzg = g.nz + 2 * g.ng;
  g.npg = (long long)g.nxg * g.nyg * g.nzg;
  g.npi = (long long)g.nx * g.ny * g.nz;
  {
    const double *src[9] = {grid->x, grid->y, grid->z, grid->dcsidx, grid->detady, grid->dzitdz,
                            grid->dcsidxs, grid->detadys, grid->dzitdzs};
    const size_t len[9] = {(size_t)g.nxg, (size_t)g.nyg, (size_t)g.nzg, (size_t)g.nx, (size_t)g.ny,
                           (size_t)g.nz, (size_t)g.nx, (size_t)g.ny, (size_t)g.nz};
    size_t off[9], tot = 0;
    for (int q = 0; q < 9; q++) {
      off[q] = tot;
      tot += len[q];
    }
    std::vector<double> gb(tot, 0.0);            // an absent array reads as zeros
    for (int q = 0; q < 9; q++)
      if (src[q]) std::memcpy(gb.data() + off[q], src[q], len[q] * sizeof(double));
    const double *gd = nullptr;
    if ((rc = upload(c, gb.data(), tot, &gd))) return fail(rc);
    const double **dst[9] = {&g.x, &g.y, &g.z, &g.dcsidx, &g.detady, &g.dzitdz, &g.dcsidxs, &g.detadys, &g.dzitdzs};
    for (int q = 0; q < 9; q++) *dst[q] = gd + off[q];
  }
  // ---- numerics
  p.p0 = par->p0; p.rho0 = par->rho0; p.u0 = par->u0; p.eps_sensor = par->eps_sensor; p.tol = par->tol_iter_nr;
  p.sensor_threshold = par->sensor_threshold; p.ros_eps = par->ros_eps;
  p.ep_order = par->ep_order; p.nkeep = par->nkeep; p.weno_scheme = par->weno_scheme; p.weno_version = par->weno_version;
  p.flux_splitting = par->flux_splitting; p.sensor_type = par->sensor_type; p.visc_order = par->visc_order;
  p.nv_aux = par->nv_aux;
  for (int q = 0; q < 6; q++) p.fzf[q] = par->force_zero_flux[q];
  p.ros_maxsteps = par->ros_maxsteps; p.ros_maxtry = par->ros_maxtry;
  p.T_wall = par->T_wall;
  std::memset(p.cd1, 0, sizeof(p.cd1));
  // coeff_deriv1 (src/grid.F90:135-160), column lmax = order/2
  p.cd1[1][1] = 0.5;
  p.cd1[1][2] = 2.0 / 3.0;  p.cd1[2][2] = -1.0 / 12.0;
  p.cd1[1][3] = 0.75;       p.cd1[2][3] = -0.15;      p.cd1[3][3] = 1.0 / 60.0;
  p.cd1[1][4] = 4.0 / 5.0;  p.cd1[2][4] = -1.0 / 5.0; p.cd1[3][4] = 4.0 / 105.0; p.cd1[4][4] = -1.0 / 280.0;
  // ---- device scratch
  const unsigned int *st = nullptr, *cn = nullptr;
  const unsigned long long *dtp = nullptr;
  if ((rc = upload<unsigned int>(c, nullptr, 1, &st))) return fail(rc);
  if ((rc = upload<unsigned int>(c, nullptr, 1, &cn))) return fail(rc);
  if ((rc = upload<unsigned long long>(c, nullptr, 9, &dtp))) return fail(rc);
  const double *tm = nullptr;
  if ((rc = upload<double>(c, nullptr, 2, &tm))) return fail(rc);   // time, dt of captured steps
  const double *rp = nullptr;
  const unsigned long long *mmp = nullptr;
  if ((rc = upload<double>(c, nullptr, STX_RES_BLOCKS, &rp))) return fail(rc);
  if ((rc = upload<unsigned long long>(c, nullptr, 6, &mmp))) return fail(rc);
  c->res_d = (double *)rp;
  c->mm_d = (unsigned long long *)mmp;
  c->status_d = (unsigned int *)st;
  c->counter_d = (unsigned int *)cn;
  c->dt_d = (unsigned long long *)dtp;
  c->time_d = (double *)tm;
  c->dtv_d = (double *)tm + 1;
  p.status = c->status_d;
  if (base) p.mixed = base->d.p.mixed;   // a context like base takes its precision form
  {
    const char *ek = std::getenv("STX_EULER_KERNEL");
    int face = ek && std::strcmp(ek, "face") == 0;
    for (int q = 0; q < 3; q++) p.sweep_kind[q] = face;
  }
  c->winf_d = nullptr;
  if (par->winf) {
    const double *wf = nullptr;
    if ((rc = upload(c, par->winf, (size_t)c->nv, &wf))) return fail(rc);
    c->winf_d = (double *)wf;
  }
  c->par.winf = nullptr;
  if ((rc = launch_euler_setup(ns))) return fail(rc);
  if ((rc = launch_batch0d_setup(ns))) return fail(rc);
  for (int q = 0; q < 3; q++) c->weno_list[q] = 1;
  c->weno = WenoScratch{nullptr, nullptr, nullptr, 0};
  const char *wl_env = std::getenv("STX_WENO_LIST");
  if (ns <= 14 && !(wl_env && std::strcmp(wl_env, "0") == 0)) {
    // the staged sweeps (ns <= 14) read the listed WENO faces' fluxes (STX_WENO_LIST=0: computed in line)
    const long long cap = weno_scratch_faces(g);
    const unsigned int *wc = nullptr;
    const int *wl = nullptr;
    const double *wf = nullptr;
    // the scratch is an optimisation: a grid whose face buffers would take more
    // than a quarter of the free device memory runs without it (WENO in line)
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const double need = (double)cap * (sizeof(int) + sizeof(double) * c->nv);
    if (cap < 0x7fffffffLL && need <= 0.25 * (double)free_b) {
      if ((rc = upload<unsigned int>(c, nullptr, 1, &wc))) return fail(rc);
      if ((rc = upload<int>(c, (const int *)nullptr, (size_t)cap, &wl))) return fail(rc);
      if ((rc = upload<double>(c, nullptr, (size_t)cap * c->nv, &wf))) return fail(rc);
      c->weno = WenoScratch{(unsigned int *)wc, (int *)wl, (double *)wf, cap};
    }
  }
  if ((rc = upload<DevCtx>(c, &c->d, 1, &c->dctx_d))) return fail(rc);
  if (!on && cudaStreamSynchronize(c->cs) != cudaSuccess) return fail(STX_E_CUDA);
  c->us = c->cs;
  *out = c;
  return STX_OK;
}

extern "C" {

int stx_ctx_create(const stx_params *par, const stx_tables *tab, const stx_grid *grid, stx_ctx **out) {
  if (!tab) return STX_E_INVALID;
  return ctx_create_impl(par, tab, grid, nullptr, nullptr, out);
}

int stx_ctx_create_like(const stx_ctx *base, const stx_params *par, const stx_grid *grid, stx_ctx **out) {
  if (!base) return STX_E_INVALID;
  return ctx_create_impl(par, nullptr, grid, base, nullptr, out);
}

int stx_ctx_create_like_on(const stx_ctx *base, const stx_params *par, const stx_grid *grid, void *stream,
                           stx_ctx **out) {
  if (!base || !stream) return STX_E_INVALID;
  return ctx_create_impl(par, nullptr, grid, base, S(stream), out);
}

// ------------------------------------------------------------------ aux
int stx_eval_aux(stx_ctx *c, void *s, double *w, double *wa, int i0, int i1, int j0, int j1, int k0, int k1) {
  if (!c || !w || !wa) return STX_E_INVALID;
  const DevGrid &g = c->d.g;
  if (i0 < 1 - g.ng || i1 > g.nx + g.ng || j0 < 1 - g.ng || j1 > g.ny + g.ng || k0 < 1 - g.ng || k1 > g.nz + g.ng)
    return STX_E_INVALID;
  // reads w (nv) and the T guess; writes Y, u, v, w, h, T, p, c, rho, Z, mu, lambda, rho*D
  Prof pf(c, S(s), STX_K_EVAL_AUX, 1,
          (double)(i1 - i0 + 1) * (j1 - j0 + 1) * (k1 - k0 + 1) * B8(3 * c->ns + 16));
  return launch_eval_aux(c->d, S(s), w, wa, i0, i1, j0, j1, k0, k1);
}

int stx_eval_aux2(stx_ctx *c, void *s, double *wa) {
  if (!c || !wa) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_DUCROS, 1, (double)c->d.g.npi * B8(5));
  return launch_eval_aux2(c->d, S(s), wa);
}

int stx_compute_aux(stx_ctx *c, void *s, double *w, double *wa, int central, int ghost) {
  if (!c || !w || !wa) return STX_E_INVALID;
  const DevGrid &g = c->d.g;
  int nx = g.nx, ny = g.ny, nz = g.nz, ng = g.ng;
  if (central == 1 && ghost == 1) {
    TRY(stx_eval_aux(c, s, w, wa, 1 - ng, nx + ng, 1 - ng, ny + ng, 1 - ng, nz + ng));
  } else if (central == 1 && ghost == 0) {
    TRY(stx_eval_aux(c, s, w, wa, 1, nx, 1, ny, 1, nz));
  } else if (central == 0 && ghost == 1) {
    TRY(stx_eval_aux(c, s, w, wa, 1 - ng, 0, 1 - ng, ny + ng, 1 - ng, nz + ng));
    TRY(stx_eval_aux(c, s, w, wa, nx + 1, nx + ng, 1 - ng, ny + ng, 1 - ng, nz + ng));
    TRY(stx_eval_aux(c, s, w, wa, 1 - ng, nx + ng, 1 - ng, 0, 1 - ng, nz + ng));
    TRY(stx_eval_aux(c, s, w, wa, 1 - ng, nx + ng, ny + 1, ny + ng, 1 - ng, nz + ng));
    TRY(stx_eval_aux(c, s, w, wa, 1 - ng, nx + ng, 1 - ng, ny + ng, 1 - ng, 0));
    TRY(stx_eval_aux(c, s, w, wa, 1 - ng, nx + ng, 1 - ng, ny + ng, nz + 1, nz + ng));
  }
  if (ghost == 1) TRY(stx_eval_aux2(c, s, wa));
  return STX_OK;
}

int stx_bcextr_var(stx_ctx *c, void *s, double *v) {
  if (!c || !v) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_GHOST, 1);
  return launch_bcextr_var(c->d, S(s), v);
}

int stx_bcswap(stx_ctx *c, void *s, double *f, int nvar) {
  if (!c || !f || nvar < 1) return STX_E_INVALID;
  {
    Prof pf(c, S(s), STX_K_GHOST, (c->periodic[0] || c->periodic[1] || c->periodic[2]) ? 1 : 0);
    TRY(launch_bcswap(c->d, S(s), f, nvar, c->periodic));
  }
  if (c->xfn) {
    int rc = c->xfn(c->xuser, s, f, nvar);
    if (rc != 0) return rc < 0 ? rc : STX_E_INVALID;
  }
  return STX_OK;
}

int stx_set_exchange(stx_ctx *c, stx_exchange_fn fn, void *user) {
  if (!c) return STX_E_INVALID;
  c->xfn = fn;
  c->xuser = fn ? user : nullptr;
  return STX_OK;
}

int stx_update_ghost_aux(stx_ctx *c, void *s, double *w, double *w_aux, int do_swap) {
  if (!c || !w) return STX_E_INVALID;
  for (int ilat = 1; ilat <= 6; ilat++) {
    int tag = c->par.bctags[ilat - 1];
    if (tag == 1 || tag == 2 || tag == 5 || tag == 7 || tag == 8) {
      Prof pf(c, S(s), STX_K_GHOST, 1);
      TRY(launch_bc_face(c->d, S(s), w, ilat, tag, c->winf_d));
    } else if (tag == 4 || tag == 6) {
      if (!w_aux) return STX_E_INVALID;              // these fills read and write w_aux
      Prof pf(c, S(s), STX_K_GHOST, 1);
      TRY(launch_bc_face_thermo(c->d, S(s), w, w_aux, ilat, tag));
    }
  }
  if (do_swap == 1) TRY(stx_bcswap(c, s, w, c->nv));
  return STX_OK;
}
int stx_update_ghost(stx_ctx *c, void *s, double *w, int do_swap) {
  return stx_update_ghost_aux(c, s, w, nullptr, do_swap);
}

int stx_bc_nr(stx_ctx *c, void *s, const double *w_aux, const double *w, double *fl) {
  if (!c || !w_aux || !w || !fl) return STX_E_INVALID;
  for (int ilat = 1; ilat <= 6; ilat++) {
    int nr = c->par.bctags_nr[ilat - 1];
    if (nr <= 0) continue;
    Prof pf(c, S(s), STX_K_EULER, 1);
    TRY(launch_bc_nr(c->d, S(s), w_aux, w, fl, c->winf_d, ilat, nr));
  }
  return STX_OK;
}

// ------------------------------------------------------------------ fluxes
int stx_euler_x(stx_ctx *c, void *s, const double *wa, double *fl, int a, int b, int ow) {
  if (!c || !wa || !fl || a < 1 || b > c->d.g.nx) return STX_E_INVALID;
  // reads Y, rho, u, v, w, h, p, c, Ducros (ns+8) and fl (unless overwritten); writes fl
  Prof pf(c, S(s), STX_K_EULER, 1, (double)(b - a + 1) * c->d.g.ny * c->d.g.nz * B8(c->ns + 8 + (ow ? 1 : 2) * c->nv));
  return launch_euler(c->d, c->dctx_d, S(s), 0, wa, fl, a, b, ow, c->weno_list[0] ? &c->weno : nullptr);
}
int stx_euler_y(stx_ctx *c, void *s, const double *wa, double *fl, int a, int b, int ow) {
  if (!c || !wa || !fl || a < 1 || b > c->d.g.ny) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_EULER, 1, (double)(b - a + 1) * c->d.g.nx * c->d.g.nz * B8(c->ns + 8 + (ow ? 1 : 2) * c->nv));
  return launch_euler(c->d, c->dctx_d, S(s), 1, wa, fl, a, b, ow, c->weno_list[1] ? &c->weno : nullptr);
}
int stx_euler_z(stx_ctx *c, void *s, const double *wa, double *fl, int a, int b, int ow) {
  if (!c || !wa || !fl || a < 1 || b > c->d.g.nz) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_EULER, 1, (double)(b - a + 1) * c->d.g.nx * c->d.g.ny * B8(c->ns + 8 + (ow ? 1 : 2) * c->nv));
  return launch_euler(c->d, c->dctx_d, S(s), 2, wa, fl, a, b, ow, c->weno_list[2] ? &c->weno : nullptr);
}

int stx_visflx(stx_ctx *c, void *s, const double *wa, double *fl, int mode) {
  if (!c || !wa || !fl) return STX_E_INVALID;
  const DevGrid &g = c->d.g;
  const int ndir = (g.nx > 1) + (g.ny > 1) + (g.nz > 1);
  // mode 1, per direction: u, v, w, T, mu, lambda, Y, rho*D read and fl read+written;
  // mode 2: u, v, w, mu, div read and four fl components read+written
  Prof pf(c, S(s), STX_K_VISC, mode == 1 ? ndir : 1,
          mode == 1 ? (double)g.npi * ndir * B8(4 * c->ns + 14) : (double)g.npi * B8(13));
  if (mode == 1) {
    if (g.nx > 1) TRY(launch_visflx(c->d, S(s), 0, wa, fl));
    if (g.ny > 1) TRY(launch_visflx(c->d, S(s), 1, wa, fl));
    if (g.nz > 1) TRY(launch_visflx(c->d, S(s), 2, wa, fl));
    return STX_OK;
  }
  if (mode == 2) return launch_visflx_reduced(c->d, S(s), wa, fl);
  return STX_E_UNSUPPORTED;
}

// ------------------------------------------------------------------ RK
int stx_init_flux(stx_ctx *c, void *s, double *fl, double *fln, double rhodt) {
  if (!c || !fl || !fln) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_RK, 1, (double)c->d.g.npi * B8(3 * c->nv));
  return launch_init_flux(c->d, S(s), fl, fln, nullptr, rhodt);
}
int stx_init_flux_simpler(stx_ctx *c, void *s, double *fl, double *fln, const double *fl_sav, double rhodt) {
  if (!c || !fl || !fln || !fl_sav) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_RK, 1);
  return launch_init_flux(c->d, S(s), fl, fln, fl_sav, rhodt);
}
int stx_sav_flx(stx_ctx *c, void *s, const double *fl, double *fl_sav) {
  if (!c || !fl || !fl_sav) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_RK, 1);
  return launch_copy(c->d, S(s), fl, fl_sav);
}
int stx_update_flux(stx_ctx *c, void *s, const double *fl, double *fln, double gamdt) {
  if (!c || !fl || !fln) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_RK, 1);
  return launch_update_flux(c->d, S(s), fl, fln, nullptr, gamdt);
}
int stx_update_simpler_flux(stx_ctx *c, void *s, const double *fl, double *fln, const double *fl_sav, double gamdt) {
  if (!c || !fl || !fln || !fl_sav) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_RK, 1);
  return launch_update_flux(c->d, S(s), fl, fln, fl_sav, gamdt);
}
int stx_update_field(stx_ctx *c, void *s, double *w, const double *fln, const int32_t *mask) {
  if (!c || !w || !fln) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_RK, 1);
  return launch_update_field(c->d, S(s), w, nullptr, (double *)fln, nullptr, mask, 0.0, 0);
}
int stx_rk_finish(stx_ctx *c, void *s, double *w, const double *fl, double *fln, const double *fl_sav,
                  const int32_t *mask, double gamdt, int simpler) {
  if (!c || !w || !fl || !fln || (simpler == 1 && !fl_sav)) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_RK, 1, (double)c->d.g.npi * B8((simpler == 1 ? 6 : 5) * c->nv));
  return launch_update_field(c->d, S(s), w, fl, fln, simpler == 1 ? fl_sav : nullptr, mask, gamdt, 1);
}

int stx_compute_dt(stx_ctx *c, void *s, const double *wa, const int32_t *mask, double out9[9]) {
  if (!c || !wa || !out9) return STX_E_INVALID;
  {
    Prof pf(c, S(s), STX_K_DT, 1, (double)c->d.g.npi * B8(c->ns + 8));
    TRY(launch_compute_dt(c->d, S(s), wa, mask, c->dt_d));
  }
  unsigned long long h[9];
  STX_CUDA_TRY(cudaMemcpyAsync(h, c->dt_d, sizeof(h), cudaMemcpyDeviceToHost, S(s)));
  STX_CUDA_TRY(cudaStreamSynchronize(S(s)));
  for (int q = 0; q < 9; q++) {
    double v;
    std::memcpy(&v, &h[q], sizeof(double));
    out9[q] = v;
  }
  return STX_OK;
}

int stx_compute_residual(stx_ctx *c, void *s, const double *fln, const double *wa, const int32_t *mask, double dt,
                         double out7[7]) {
  if (!c || !fln || !wa || !out7 || !(dt != 0.0)) return STX_E_INVALID;
  {
    Prof pf(c, S(s), STX_K_DT, 1, (double)c->d.g.npi * B8(4));
    TRY(launch_residual_minmax(c->d, S(s), fln, wa, mask, dt, c->res_d, c->mm_d));
  }
  double part[STX_RES_BLOCKS];
  unsigned long long h[6];
  STX_CUDA_TRY(cudaMemcpyAsync(part, c->res_d, sizeof(part), cudaMemcpyDeviceToHost, S(s)));
  STX_CUDA_TRY(cudaMemcpyAsync(h, c->mm_d, sizeof(h), cudaMemcpyDeviceToHost, S(s)));
  STX_CUDA_TRY(cudaStreamSynchronize(S(s)));
  double sum = 0.0;
  for (int b = 0; b < STX_RES_BLOCKS; b++) sum = sum + part[b];
  // residual_rhou = sqrt(sum / (nx ny nz nprocs)) (multideal_gpu.F90:1603-1606, one process)
  out7[0] = std::sqrt(sum / ((double)c->d.g.nx * (double)c->d.g.ny * (double)c->d.g.nz));
  const int order[6] = {0, 3, 1, 4, 2, 5};     // rhomin, rhomax, tmin, tmax, pmin, pmax
  for (int q = 0; q < 6; q++) std::memcpy(&out7[1 + q], &h[order[q]], sizeof(double));
  return STX_OK;
}

// ------------------------------------------------------------------ chemistry
int stx_rosenbrock(stx_ctx *c, void *s, double *w, double *wa, double dttry, double t0, double t1) {
  if (!c || !w || !wa) return STX_E_INVALID;
  if (c->d.t.nr < 1) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_CHEM, 1);
  return launch_rosenbrock(c->d, S(s), w, wa, dttry, t0, t1, c->counter_d);
}
int stx_rosenbrock_krylov(stx_ctx *c, void *s, double *w, const double *wa, const double *fl_sav, double dttry,
                          double t0, double t1, int simpler) {
  if (!c || !w || !wa || (simpler == 1 && !fl_sav)) return STX_E_INVALID;
  if (c->d.t.nr < 1) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_CHEM, 1, (double)c->d.g.npi * B8(2 * c->nv + 2));
  return launch_rok4(c->d, c->dctx_d, S(s), w, wa, fl_sav, dttry, t0, t1, simpler, c->counter_d);
}
int stx_batch0d_integrate(stx_ctx *c, void *s, int n, const double *T0, const double *p0, const double *Y0,
                          double t_max, double dttry, double ign_factor, double end_factor, int max_steps, double *Y,
                          double *T, double *t_ign, double *t_end, int32_t *nsteps) {
  if (!c || n < 0 || (n > 0 && (!T0 || !p0 || !Y0 || !Y || !T || !t_ign || !t_end || !nsteps))) return STX_E_INVALID;
  if (c->d.t.nr < 1 || !(t_max > 0.0) || !(dttry > 0.0) || max_steps < 1) return STX_E_INVALID;
  if (n == 0) return STX_OK;
  DevCtx d = c->d;
  d.p.ros_maxsteps = max_steps;
  Prof pf(c, S(s), STX_K_CHEM, 1, (double)n * 8.0 * (2 * c->d.t.ns + 6));
  // One warp per reactor where the mechanism fits (ns <= 32, nr <= 64) and every
  // reactor gets a resident warp at once: a warp integrates one reactor several
  // times faster than a thread, so a small batch (a served one) ends sooner.
  // Larger batches run a thread per reactor (more reactors at once).
  // STX_BATCH0D_KERNEL=thread / warp forces either kernel.  In the mixed
  // precision form (stx_set_precision) the reactors run the thread kernel's
  // FP32/FP64-split form: the Krylov basis and stage vectors in FP32, the state,
  // every right-hand side and the error control in FP64.
  const char *kind = std::getenv("STX_BATCH0D_KERNEL");
  if (!(kind && std::strcmp(kind, "thread") == 0) && !c->d.p.mixed) {
    int force = kind && std::strcmp(kind, "warp") == 0;
    int rc = launch_batch0d_warp(d, S(s), n, T0, p0, Y0, t_max, dttry, ign_factor, end_factor, Y, T, t_ign, t_end,
                                 nsteps, c->counter_d, force);
    if (rc != STX_E_UNSUPPORTED) return rc;
  }
  return launch_batch0d(d, c->dctx_d, S(s), n, T0, p0, Y0, t_max, dttry, ign_factor, end_factor, Y, T, t_ign, t_end,
                        nsteps, c->counter_d);
}
int stx_compute_chemistry(stx_ctx *c, void *s, double *w, double *wa, double *fl) {
  if (!c || !w || !wa || !fl) return STX_E_INVALID;
  if (c->d.t.nr < 1) return STX_E_INVALID;
  Prof pf(c, S(s), STX_K_CHEM, 1);
  return launch_chem_explicit(c->d, S(s), w, wa, fl);
}

// ------------------------------------------------------------------ steps
static int rhs_pass(stx_ctx *c, void *s, const stx_fields *f) {
  const int ns = c->ns;
  const DevGrid &g = c->d.g;
  double *div = f->w_aux + (size_t)(ns + 9) * g.npg;   // J_DIV (1-based ns+10)
  double *duc = f->w_aux + (size_t)(ns + 8) * g.npg;   // J_DUC
  TRY(stx_bcswap(c, s, f->w, c->nv));
  TRY(stx_compute_aux(c, s, f->w, f->w_aux, 1, 1));
  TRY(stx_bcextr_var(c, s, div));
  TRY(stx_bcswap(c, s, duc, 1));
  TRY(stx_bcswap(c, s, div, 1));
  TRY(stx_euler_x(c, s, f->w_aux, f->fl, c->par.eul_imin, c->par.eul_imax, 0));
  if (g.ny > 1) TRY(stx_euler_y(c, s, f->w_aux, f->fl, c->par.eul_jmin, c->par.eul_jmax, 0));
  if (g.nz > 1) TRY(stx_euler_z(c, s, f->w_aux, f->fl, c->par.eul_kmin, c->par.eul_kmax, 0));
  TRY(stx_visflx(c, s, f->w_aux, f->fl, 1));
  TRY(stx_visflx(c, s, f->w_aux, f->fl, 2));
  TRY(stx_bc_nr(c, s, f->w_aux, f->w, f->fl));
  if (c->par.enable_chemistry == 1) TRY(stx_compute_chemistry(c, s, f->w, f->w_aux, f->fl));
  return STX_OK;
}

// rk_sync (multideal_gpu.F90:548-621).  scale: the factor of dt that the
// splitting hands this call (1, or 0.5 for the simpler splitting's RK half);
// used only while a CFL-driven step is captured (c->d.p.dt_d set), where the
// kernels form the RK scalars from the device dt.
static int rk_sync_impl(stx_ctx *c, void *s, const stx_fields *f, double dt, int simpler, double scale) {
  const bool dev = c->d.p.dt_d != nullptr;
  for (int istep = 0; istep < c->par.nrk; istep++) {
    double rhodt = dev ? c->par.rhork[istep] : c->par.rhork[istep] * dt;
    double gamdt = dev ? c->par.gamrk[istep] : c->par.gamrk[istep] * dt;
    {
      Prof pf(c, S(s), STX_K_RK, 1, simpler == 1 ? 0.0 : (double)c->d.g.npi * B8(3 * c->nv));
      TRY(launch_init_flux(c->d, S(s), f->fl, f->fln, simpler == 1 ? f->fl_sav : nullptr, rhodt, scale));
    }
    TRY(rhs_pass(c, s, f));
    {
      Prof pf(c, S(s), STX_K_RK, 1, (double)c->d.g.npi * B8((simpler == 1 ? 6 : 5) * c->nv));
      TRY(launch_update_field(c->d, S(s), f->w, f->fl, f->fln, simpler == 1 ? f->fl_sav : nullptr, f->fluid_mask,
                              gamdt, 1, scale));
    }
    TRY(stx_update_ghost_aux(c, s, f->w, f->w_aux, 0));
  }
  return STX_OK;
}

int stx_rk_sync(stx_ctx *c, void *s, const stx_fields *f, double dt, int simpler) {
  if (!c || !f || !f->w || !f->w_aux || !f->fl || !f->fln || (simpler == 1 && !f->fl_sav)) return STX_E_INVALID;
  return rk_sync_impl(c, s, f, dt, simpler, 1.0);
}

// advance_solution (multideal_gpu.F90:1605-1642).  While a CFL-driven step is
// captured, dt is not known on the host: the chemistry receives the splitting's
// factor of dt as its dttry (the kernels scale it by the device dt) and the RK
// half its scale.
int stx_advance_solution(stx_ctx *c, void *s, const stx_fields *f, double dt, double time) {
  if (!c || !f || !f->w || !f->w_aux || !f->fl || !f->fln) return STX_E_INVALID;
  const stx_params &p = c->par;
  const bool dev = c->d.p.dt_d != nullptr;
  if (p.enable_chemistry == 2) {
    if (p.operator_splitting == 1) {
      if (p.rosenbrock_version != 2 || !f->fl_sav) return STX_E_INVALID;
      double dt_chem = dt;
      // sav_flx (multideal_gpu.F90:623-692): fl = 0, one right-hand side, fl_sav = fl
      STX_CUDA_TRY(cudaMemsetAsync(f->fl, 0, sizeof(double) * c->d.g.npi * c->nv, S(s)));
      TRY(rhs_pass(c, s, f));
      TRY(stx_update_ghost_aux(c, s, f->w, f->w_aux, 0));
      TRY(stx_sav_flx(c, s, f->fl, f->fl_sav));
      TRY(stx_compute_aux(c, s, f->w, f->w_aux, 1, 0));
      TRY(stx_rosenbrock_krylov(c, s, f->w, f->w_aux, f->fl_sav, dev ? 1.0 : dt_chem, time, time + dt_chem, 1));
      TRY(rk_sync_impl(c, s, f, 0.5 * dt, 1, 0.5));
    } else {
      double dt_chem = 0.5 * dt;
      const double tr = dev ? 0.5 : dt_chem;
      if (p.rosenbrock_version == 1) TRY(stx_rosenbrock(c, s, f->w, f->w_aux, tr, time, time + dt_chem));
      else TRY(stx_rosenbrock_krylov(c, s, f->w, f->w_aux, nullptr, tr, time, time + dt_chem, 0));
      TRY(rk_sync_impl(c, s, f, dt, 0, 1.0));
      TRY(stx_compute_aux(c, s, f->w, f->w_aux, 1, 0));
      if (p.rosenbrock_version == 1) TRY(stx_rosenbrock(c, s, f->w, f->w_aux, tr, time, time + dt_chem));
      else TRY(stx_rosenbrock_krylov(c, s, f->w, f->w_aux, nullptr, tr, time, time + dt_chem, 0));
    }
  } else {
    TRY(rk_sync_impl(c, s, f, dt, 0, 1.0));
  }
  return STX_OK;
}

int stx_set_precision(stx_ctx *c, int mode) {
  if (!c || (mode != STX_PREC_FP64 && mode != STX_PREC_MIXED)) return STX_E_INVALID;
  c->d.p.mixed = mode;
  STX_CUDA_TRY(cudaMemcpyAsync((void *)c->dctx_d, &c->d, sizeof(DevCtx), cudaMemcpyHostToDevice, c->cs));
  STX_CUDA_TRY(cudaStreamSynchronize(c->cs));
  return STX_OK;
}

// ------------------------------------------------------------------ captured steps
// A run at fixed dt (cfl < 0 in multideal.ini) repeats the same kernel sequence
// every step; only the simulation time changes, and only the chemistry reads
// it.  nsteps steps of the reference's integration loop
// (multideal_gpu.F90:1745-1806: compute_aux, advance_solution, compute_aux;
// the time advance) are captured once into a CUDA graph whose chemistry
// kernels read the time from c->time_d and whose last node advances it, so
// one graph launch replaces ~50 launches per step with the same arithmetic.
//
// A CFL-driven run (cfl > 0, dt recomputed every step) is captured the same
// way with the step size in device memory as well: each step forms the nine
// CFL maxima (compute_dt_cuf) and dt = cfl / max on the device, and the
// kernels that take a dt-derived scalar form it from there (DevPar::dt_d), so
// nothing returns to the host between steps; stx_graph_state reads the time
// and the last dt back after a launch.
struct stx_graph {
  stx_ctx *c;
  cudaGraphExec_t exec;
  double dt;          // fixed dt, or 0 for a CFL-driven graph
  double cfl;
  int nsteps;
};

namespace {
__global__ void k_time_add(double *t, double dt) { *t = *t + dt; }
__global__ void k_time_set(double *t, double v) { *t = v; }

// dt > 0: fixed step; otherwise cfl > 0 and the step comes from the CFL maxima
int graph_create_impl(stx_ctx *c, const stx_fields *f, double dt, double cfl, int nsteps, stx_graph **out) {
  *out = nullptr;
  if (c->xfn) return STX_E_UNSUPPORTED;   // the exchange runs host code at every swap
  const bool dev = !(dt > 0.0);
  cudaStream_t cs;
  STX_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  const int prof = c->prof_on;
  c->prof_on = 0;
  c->d.p.time_d = c->time_d;
  if (dev) c->d.p.dt_d = c->dtv_d;
  int rc = STX_OK;
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) rc = STX_E_CUDA;
  for (int n = 0; n < nsteps && rc == STX_OK; n++) {
    if ((rc = stx_compute_aux(c, cs, f->w, f->w_aux, 1, 0))) break;
    if (dev) {
      if ((rc = launch_compute_dt(c->d, cs, f->w_aux, f->fluid_mask, c->dt_d))) break;
      if ((rc = launch_dt_from_max(cs, c->dt_d, cfl, c->dtv_d))) break;
    }
    if ((rc = stx_advance_solution(c, cs, f, dt, 0.0))) break;
    if ((rc = stx_compute_aux(c, cs, f->w, f->w_aux, 1, 0))) break;
    if (dev) {
      if ((rc = launch_time_advance(cs, c->time_d, c->dtv_d))) break;
    } else {
      k_time_add<<<1, 1, 0, cs>>>(c->time_d, dt);
      if (cudaGetLastError() != cudaSuccess) rc = STX_E_CUDA;
    }
  }
  if (e == cudaSuccess) {
    cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
    if (e2 != cudaSuccess && rc == STX_OK) rc = STX_E_CUDA;
  }
  c->d.p.time_d = nullptr;
  c->d.p.dt_d = nullptr;
  c->prof_on = prof;
  stx_graph *g = nullptr;
  if (rc == STX_OK) {
    g = new (std::nothrow) stx_graph();
    if (!g) rc = STX_E_NOMEM;
  }
  if (rc == STX_OK && cudaGraphInstantiate(&g->exec, graph, 0) != cudaSuccess) rc = STX_E_CUDA;
  if (graph) cudaGraphDestroy(graph);
  cudaStreamDestroy(cs);
  if (rc != STX_OK) {
    delete g;
    return rc;
  }
  g->c = c;
  g->dt = dev ? 0.0 : dt;
  g->cfl = dev ? cfl : 0.0;
  g->nsteps = nsteps;
  *out = g;
  return STX_OK;
}
}  // namespace

int stx_graph_create(stx_ctx *c, const stx_fields *f, double dt, int nsteps, stx_graph **out) {
  if (!c || !f || !out || nsteps < 1 || !(dt > 0.0)) return STX_E_INVALID;
  return graph_create_impl(c, f, dt, 0.0, nsteps, out);
}

int stx_graph_create_cfl(stx_ctx *c, const stx_fields *f, double cfl, int nsteps, stx_graph **out) {
  if (!c || !f || !out || nsteps < 1 || !(cfl > 0.0)) return STX_E_INVALID;
  return graph_create_impl(c, f, 0.0, cfl, nsteps, out);
}

int stx_graph_launch(stx_graph *g, void *s, double time) {
  if (!g) return STX_E_INVALID;
  k_time_set<<<1, 1, 0, S(s)>>>(g->c->time_d, time);
  STX_CUDA_TRY(cudaGetLastError());
  STX_CUDA_TRY(cudaGraphLaunch(g->exec, S(s)));
  return STX_OK;
}

int stx_graph_state(stx_graph *g, void *s, double *time, double *dt) {
  if (!g || !time || !dt) return STX_E_INVALID;
  double h[2];
  STX_CUDA_TRY(cudaMemcpyAsync(h, g->c->time_d, sizeof(h), cudaMemcpyDeviceToHost, S(s)));
  STX_CUDA_TRY(cudaStreamSynchronize(S(s)));
  *time = h[0];
  *dt = g->dt > 0.0 ? g->dt : h[1];
  return STX_OK;
}

int stx_graph_destroy(stx_graph *g) {
  if (!g) return STX_OK;
  cudaGraphExecDestroy(g->exec);
  delete g;
  return STX_OK;
}

int stx_profile_enable(stx_ctx *c, int on) {
  if (!c) return STX_E_INVALID;
  c->prof_on = on ? 1 : 0;
  for (int k = 0; k < STX_NK; k++) {
    c->launches[k] = 0;
    c->ev_used[k] = 0;
    c->bytes[k] = 0.0;
  }
  return STX_OK;
}

int stx_profile_read(stx_ctx *c, stx_kprof *out) {
  if (!c || !out) return STX_E_INVALID;
  STX_CUDA_TRY(cudaDeviceSynchronize());
  for (int k = 0; k < STX_NK; k++) {
    out[k].launches = c->launches[k];
    out[k].timed = (int64_t)(c->ev_used[k] / 2);
    double ms = 0.0;
    for (size_t q = 0; q + 1 < c->ev_used[k]; q += 2) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, c->ev[k][q], c->ev[k][q + 1]) == cudaSuccess) ms += t;
    }
    out[k].ms = ms;
    out[k].bytes = c->bytes[k];
  }
  return STX_OK;
}

int stx_status(stx_ctx *c, void *s, uint32_t *bits, int reset) {
  if (!c || !bits) return STX_E_INVALID;
  unsigned int h = 0;
  STX_CUDA_TRY(cudaMemcpyAsync(&h, c->status_d, sizeof(h), cudaMemcpyDeviceToHost, S(s)));
  STX_CUDA_TRY(cudaStreamSynchronize(S(s)));
  *bits = h;
  if (reset) STX_CUDA_TRY(cudaMemsetAsync(c->status_d, 0, sizeof(unsigned int), S(s)));
  return STX_OK;
}

// ------------------------------------------------------------------ tuning
int stx_get_tuning(stx_ctx *c, stx_tuning *out) {
  if (!c || !out) return STX_E_INVALID;
  std::memset(out, 0, sizeof(*out));
  for (int q = 0; q < 3; q++) {
    out->sweep_kind[q] = c->d.p.sweep_kind[q];
    out->weno_list[q] = c->weno_list[q];
  }
  out->chem_ctas_per_sm = c->d.p.chem_ctas_per_sm;
  out->chem_ctas_max = chem_ctas_limit(c->ns);
  out->batch_ctas_max = c->d.p.batch_ctas_max;
  return STX_OK;
}

int stx_set_tuning(stx_ctx *c, const stx_tuning *t) {
  if (!c || !t) return STX_E_INVALID;
  for (int q = 0; q < 3; q++)
    if ((t->sweep_kind[q] != 0 && t->sweep_kind[q] != 1) || (t->weno_list[q] != 0 && t->weno_list[q] != 1))
      return STX_E_INVALID;
  if (t->chem_ctas_per_sm < -1 || t->batch_ctas_max < 0) return STX_E_INVALID;
  for (int q = 0; q < 3; q++) {
    c->d.p.sweep_kind[q] = t->sweep_kind[q];
    c->weno_list[q] = t->weno_list[q];
  }
  c->d.p.chem_ctas_per_sm = t->chem_ctas_per_sm;
  c->d.p.batch_ctas_max = t->batch_ctas_max;
  STX_CUDA_TRY(cudaMemcpyAsync((void *)c->dctx_d, &c->d, sizeof(DevCtx), cudaMemcpyHostToDevice, c->cs));
  STX_CUDA_TRY(cudaStreamSynchronize(c->cs));
  return STX_OK;
}

int stx_autotune(stx_ctx *c, void *sv, const stx_fields *f, double dt_chem, stx_tuning *out) {
  if (!c || !f || !f->w || !f->w_aux) return STX_E_INVALID;
  cudaStream_t s = S(sv);
  const DevGrid &g = c->d.g;
  const size_t nfl = (size_t)g.npi * c->nv, nw = (size_t)g.npg * c->nv;
  cudaMemPool_t pool = ctx_pool(c->device);
  double *fls = nullptr, *w2 = nullptr;
  unsigned int *st_save = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = STX_OK;
  float sweep_ms[3] = {0.f, 0.f, 0.f}, chem_ms = 0.f;
  if (!pool || cudaMallocFromPoolAsync((void **)&fls, nfl * sizeof(double), pool, s) != cudaSuccess ||
      cudaMallocFromPoolAsync((void **)&st_save, sizeof(unsigned int), pool, s) != cudaSuccess)
    return STX_E_NOMEM;
  // the status bits the trial launches raise are not the caller's: saved here, restored at the end
  cudaMemcpyAsync(st_save, c->status_d, sizeof(unsigned int), cudaMemcpyDeviceToDevice, s);
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // ---- convective sweeps: staged tiles with listed WENO faces, staged tiles
  // with WENO in line, one face per thread (a scratch residual, overwritten)
  const int nsw[3] = {g.nx, g.ny, g.nz};
  for (int d = 0; d < 3 && rc == STX_OK; d++) {
    if (d > 0 && nsw[d] == 1) continue;     // the step skips a sweep over one cell
    struct Cand { int kind, list; };
    const Cand cands[3] = {{0, 1}, {0, 0}, {1, 0}};
    float best = -1.f;
    Cand pick = cands[0];
    for (const Cand &k : cands) {
      if (k.list && c->weno.cap == 0) continue;
      c->d.p.sweep_kind[d] = k.kind;
      const WenoScratch *wsc = k.list ? &c->weno : nullptr;
      float ms = time_launches(s, e0, e1, 3, [&] {
        return launch_euler(c->d, c->dctx_d, s, d, f->w_aux, fls, 1, nsw[d], 1, wsc);
      });
      if (ms < 0.f) { rc = STX_E_CUDA; break; }
      // the default (first) stays unless another is clearly faster: the Ducros
      // sensor marks more faces as the flow develops, which favours the default
      if (best < 0.f || ms < 0.9f * best) { best = ms; pick = k; }
    }
    c->d.p.sweep_kind[d] = pick.kind;
    c->weno_list[d] = pick.list;
    sweep_ms[d] = best;
  }
  // ---- cell chemistry (ROK4), on a scratch copy of w: persistent CTAs per SM
  // (work stealing), then the plain launch (one thread per cell, -1), which the
  // hardware's block scheduler balances instead
  const stx_params &p = c->par;
  if (rc == STX_OK && p.enable_chemistry == 2 && p.rosenbrock_version == 2 && dt_chem > 0.0) {
    if (cudaMallocFromPoolAsync((void **)&w2, nw * sizeof(double), pool, s) != cudaSuccess) {
      rc = STX_E_NOMEM;
    } else {
      const int lim = chem_ctas_limit(c->ns);
      float best = -1.f;
      int pick = 0;
      for (int k = lim; k >= -1 && rc == STX_OK; k--) {    // the default (the limit) first
        if (k == 0) continue;
        c->d.p.chem_ctas_per_sm = k;
        float ms = time_launches(s, e0, e1, 1, [&] {
          if (cudaMemcpyAsync(w2, f->w, nw * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            return (int)STX_E_CUDA;
          return launch_rok4(c->d, c->dctx_d, s, w2, f->w_aux, nullptr, dt_chem, 0.0, dt_chem, 0, c->counter_d);
        });
        if (ms < 0.f) { rc = STX_E_CUDA; break; }
        if (best < 0.f || ms < 0.95f * best) { best = ms; pick = k; }
      }
      c->d.p.chem_ctas_per_sm = pick == lim ? 0 : pick;
      chem_ms = best;
    }
  }
  cudaMemcpyAsync(c->status_d, st_save, sizeof(unsigned int), cudaMemcpyDeviceToDevice, s);
  if (w2) cudaFreeAsync(w2, s);
  cudaFreeAsync(fls, s);
  cudaFreeAsync(st_save, s);
  if (cudaStreamSynchronize(s) != cudaSuccess && rc == STX_OK) rc = STX_E_CUDA;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != STX_OK) return rc;
  STX_CUDA_TRY(cudaMemcpyAsync((void *)c->dctx_d, &c->d, sizeof(DevCtx), cudaMemcpyHostToDevice, c->cs));
  STX_CUDA_TRY(cudaStreamSynchronize(c->cs));
  if (out) {
    TRY(stx_get_tuning(c, out));
    for (int d = 0; d < 3; d++) out->sweep_ms[d] = sweep_ms[d];
    out->chem_ms = chem_ms;
  }
  return STX_OK;
}

int stx_status_enqueue(stx_ctx *c, void *s, uint32_t *bits, int reset) {
  if (!c || !bits) return STX_E_INVALID;
  STX_CUDA_TRY(cudaMemcpyAsync(bits, c->status_d, sizeof(unsigned int), cudaMemcpyDefault, S(s)));
  if (reset) STX_CUDA_TRY(cudaMemsetAsync(c->status_d, 0, sizeof(unsigned int), S(s)));
  return STX_OK;
}

}  // extern "C"
