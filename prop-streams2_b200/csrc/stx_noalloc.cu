// stx_noalloc.cu -- allocation-free entry point for the ROK4 chemistry update.
//
// Some callers cannot call cudaMalloc: a host code whose device memory is owned
// by another runtime or a fixed arena (a Fortran host that uploaded its tables
// itself, a pre-sized memory pool), or a code path that must not allocate
// while other work is in flight.  stx_rosenbrock_krylov_noalloc() serves them:
// it needs no context, reads the caller's own device tables in the reference's
// Fortran layouts, and allocates nothing.  Its only scratch -- the cell counter
// of the work-stealing schedule -- is the file-scope device array below.
#include <cstdint>
#include <mutex>

#include "stx_chem.cuh"

// Work-stealing cell counter: 4 bytes of device scratch, allocated when the
// library is loaded on a device and kept until the process exits.  Every call
// on that device shares it; it is cleared at the start of each call, and two
// calls that overlap on the GPU (different streams, no ordering) race on it.
static __device__ __align__(256) unsigned int g_noalloc_counter[1];

// Largest cell count one call accepts: every resident thread may claim once past
// the end, so the 32-bit counter must stay below 2^32 with that overshoot.
#define STX_NOALLOC_MAX_CELLS (1LL << 31)

template <int NS>
__global__ void __launch_bounds__(128) k_rok4_noalloc(DevCtx c, double *__restrict__ w, const double *__restrict__ wa,
                                                      const double *__restrict__ fl_sav, double dttry, double t0,
                                                      double t1, int simpler, unsigned int *counter) {
  const DevGrid &g = c.g;
  const int NV = NS + 4;
  const double eps_Z = 5e-4;
  for (;;) {
    long long cell = claim(counter);
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
    rok4_cell<NS, true>(c, VEC, FG(wa, p, NS + 5), simpler == 1 ? fl_sav + cell : nullptr, g.npi, dttry, t0, t1,
                        simpler);
#pragma unroll
    for (int m = 0; m < NV; m++) FG(w, p, m + 1) = VEC[m];
  }
}

namespace {

// Device address of g_noalloc_counter, looked up once per device with that
// device current (the host-side symbol is not a device address).  The cache
// holds for the life of the device's primary context: after cudaDeviceReset the
// library's module is loaded anew and the cached address is stale, so a caller
// that resets a device must not call this entry point on it again.
std::mutex g_mu;
unsigned int *g_addr[64];
bool g_ready[64];

int counter_address(int dev, unsigned int **out) {
  if (dev < 0 || dev >= 64) return STX_E_CUDA;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ready[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_counter) != cudaSuccess || p == nullptr) return STX_E_CUDA;
    g_addr[dev] = (unsigned int *)p;
    g_ready[dev] = true;
  }
  *out = g_addr[dev];
  return STX_OK;
}

// The kernel keeps its per-thread working set (Krylov basis, stage vectors, the
// frame of the out-of-line right-hand side) in local memory.  The driver backs
// local memory with a reservation of cudaLimitStackSize bytes for every thread
// the device can hold, and grows it -- a device allocation of (frame x resident
// threads), about 1 GB for 9 species on a B200 -- when a launch needs more than
// the current limit.  That growth would break this entry point's promise, so a
// launch that would trigger it is refused with STX_E_LOCAL_MEM instead; the
// caller raises the limit once at initialisation (cudaDeviceSetLimit).
template <int NS>
int local_memory_ok() {
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, (const void *)k_rok4_noalloc<NS>) != cudaSuccess) return STX_E_CUDA;
  size_t lim = 0;
  if (cudaDeviceGetLimit(&lim, cudaLimitStackSize) != cudaSuccess) return STX_E_CUDA;
  return fa.localSizeBytes <= lim ? STX_OK : STX_E_LOCAL_MEM;
}

template <int NS>
int launch(const DevCtx &c, cudaStream_t s, int dev, double *w, const double *wa, const double *fl_sav, double dttry,
           double t0, double t1, int simpler, unsigned int *counter) {
  int rc = local_memory_ok<NS>();
  if (rc != STX_OK) return rc;
  int nsm = 148, per = 1;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void *)k_rok4_noalloc<NS>, 128, 0);
  long long nb = (long long)nsm * (per < 1 ? 1 : per);
  long long need = (c.g.npi + 127) / 128;
  if (nb > need) nb = need;
  if (cudaMemsetAsync(counter, 0, sizeof(unsigned int), s) != cudaSuccess) return STX_E_CUDA;
  k_rok4_noalloc<NS><<<(int)nb, 128, 0, s>>>(c, w, wa, fl_sav, dttry, t0, t1, simpler, counter);
  return cudaGetLastError() == cudaSuccess ? STX_OK : STX_E_CUDA;
}

}  // namespace

extern "C" int stx_rosenbrock_krylov_noalloc(const stx_params *par, const stx_tables *tab, const stx_grid *grid,
                                             void *stream, double *w, const double *w_aux, const double *fl_sav,
                                             double dttry, double time_start, double time_end, int simpler,
                                             uint32_t *status) {
  if (!par || !tab || !grid || !w || !w_aux || (simpler == 1 && !fl_sav)) return STX_E_INVALID;
  if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || grid->ng < 1) return STX_E_INVALID;
  if (tab->nr < 1 || tab->nsetcv < 1 || tab->num_t_tab < 1) return STX_E_INVALID;
  if (!tab->mw || !tab->trange || !tab->cv_coeff || !tab->reac_ty || !tab->is_rev || !tab->arr_a || !tab->arr_b ||
      !tab->arr_ea || !tab->falloff || !tab->tb_eff || !tab->r_coeffs || !tab->p_coeffs || !tab->kc_tab)
    return STX_E_INVALID;
  const long long ncell = (long long)grid->nx * grid->ny * grid->nz;
  if (ncell > STX_NOALLOC_MAX_CELLS) return STX_E_TOO_LARGE;
  DevCtx c;
  DevTab &t = c.t;
  DevGrid &g = c.g;
  DevPar &p = c.p;
  t = DevTab{};
  t.ns = tab->ns; t.nr = tab->nr; t.icl = tab->indx_cp_l; t.icr = tab->indx_cp_r; t.nset = tab->nsetcv;
  t.ntab = tab->num_t_tab; t.ncp = t.icr - t.icl + 3; t.tmin = tab->t_min_tab; t.dtab = tab->dt_tab; t.Ru = tab->R_univ;
  t.mw = tab->mw; t.mwinv = tab->mwinv; t.rgas = tab->rgas; t.trange = tab->trange;
  t.cp = tab->cp_coeff; t.cv = tab->cv_coeff;
  t.reac_ty = tab->reac_ty; t.is_rev = tab->is_rev;
  t.arr_a = tab->arr_a; t.arr_b = tab->arr_b; t.arr_ea = tab->arr_ea; t.falloff = tab->falloff;
  t.tb_eff = tab->tb_eff; t.r_coeffs = tab->r_coeffs; t.p_coeffs = tab->p_coeffs;
  t.kc_r = tab->kc_tab;                        // reference layout, read with KCF = true
  t.n_eoi = 1;
  g = DevGrid{};
  g.nx = grid->nx; g.ny = grid->ny; g.nz = grid->nz; g.ng = grid->ng;
  g.nxg = g.nx + 2 * g.ng; g.nyg = g.ny + 2 * g.ng; g.nzg = g.nz + 2 * g.ng;
  g.npg = (long long)g.nxg * g.nyg * g.nzg;
  g.npi = ncell;
  p = DevPar{};
  p.tol = par->tol_iter_nr;
  p.ros_maxsteps = par->ros_maxsteps;
  p.ros_eps = par->ros_eps;
  p.status = status;
  cudaStream_t s = (cudaStream_t)stream;
  // the scratch and the launch belong to the current device; a stream of
  // another device would pair it with the wrong device's counter
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return STX_E_CUDA;
  int sdev = dev;
  if (s != nullptr && cudaStreamGetDevice(s, &sdev) != cudaSuccess) return STX_E_CUDA;
  if (sdev != dev) return STX_E_INVALID;
  unsigned int *counter = nullptr;
  int rc = counter_address(dev, &counter);
  if (rc != STX_OK) return rc;
  switch (t.ns) {
#define X(N) case N: return launch<N>(c, s, dev, w, w_aux, fl_sav, dttry, time_start, time_end, simpler, counter);
    STX_FOR_NS(X)
#undef X
    default: return STX_E_UNSUPPORTED;
  }
}
