"""GPU parity tests: every libstx.so kernel against the FP64 oracle on the same
inputs (through the C ABI).  Tolerances are relative to each field's scale and
stated per test; chemistry is compiled without FMA contraction and matches the
oracle except for the rounding of exp/pow/log10."""
import ctypes as C

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from driver import OracleSolver  # noqa: E402
from stx.solver import Solver  # noqa: E402


def vp(a):
    return C.c_void_p(a.ctypes.data) if isinstance(a, np.ndarray) else C.c_void_p(a.data_ptr())


def pair(case, threads=8):
    g = Solver(case)
    o = OracleSolver(case, threads=threads)
    return g, o


def to_gpu(g, o):
    """Copy the oracle's state into the device fields."""
    g.w.copy_(torch.from_numpy(o.w))
    g.w_aux.copy_(torch.from_numpy(o.w_aux))
    g.fl.copy_(torch.from_numpy(o.fl))
    g.fln.copy_(torch.from_numpy(o.fln))
    g.fl_sav.copy_(torch.from_numpy(o.fl_sav))
    torch.cuda.synchronize()


def prime(case):
    """Both sides after update_ghost + compute_aux on identical inputs."""
    g, o = pair(case)
    o.update_ghost(1)
    o.compute_aux(1, 1)
    to_gpu(g, o)
    return g, o


def S(g):
    return g.stream


# ------------------------------------------------------------------ aux / ghosts
@pytest.mark.parametrize("n,bc,order,st", [((16, 12, 10), (0, 0, 0, 0, 0, 0), 6, 1), ((20, 6, 5), (8, 2, 0, 0, 2, 8), 6, 1),
                                         ((16, 12, 10), (0, 0, 0, 0, 0, 0), 2, 0),
                                         ((16, 12, 10), (0, 0, 0, 0, 0, 0), 4, 1),
                                         ((16, 12, 10), (8, 2, 0, 0, 2, 8), 8, 0)])
def test_update_ghost_and_compute_aux(n, bc, order, st):
    """Ghost fills and eval_aux / eval_aux2; the derivatives of eval_aux2 at every
    visc_order (= ep_order) the ABI accepts, with both Ducros sensor types."""
    case = H.synthetic_case(n=n, bc=bc, seed=1, ep_order=order, ng=max(3, order // 2), sensor_type=st)
    g, o = pair(case)
    o.update_ghost(1)
    g.update_ghost(1)
    assert np.array_equal(g.host_w(), o.w)           # ghost fills are copies: bit-exact
    o.compute_aux(1, 1)
    g.compute_aux(1, 1)
    wa_g, wa_o = g.host_w_aux(), o.w_aux
    ns = case.ns
    assert np.array_equal(g.host_w(), o.w)
    # species, velocities, h, T, p, c, mu, rho, Z, lambda, rho*D: rounding-level agreement
    for m in list(range(0, ns + 8)) + [ns + 10, ns + 11, ns + 12] + list(range(ns + 13, 2 * ns + 13)):
        H.assert_close(wa_g[m], wa_o[m], 1e-12, f"w_aux[{m}]")
    # Ducros sensor and div/3 (interior; derivatives of the above)
    H.assert_close(case.interior(wa_g[case.J("DIV")]), case.interior(wa_o[case.J("DIV")]), 1e-9, "div")
    H.assert_close(case.interior(wa_g[case.J("DUC")]), case.interior(wa_o[case.J("DUC")]), 1e-9, "ducros",
                   floor=1e-12)


def test_bcswap_small_extent_matches_pack_then_unpack():
    """ny = 1 < ng: the periodic exchange reads ghost cells it also writes."""
    case = H.synthetic_case(n=(12, 1, 2), seed=2)
    g, o = pair(case)
    rng = np.random.default_rng(0)
    o.w[:] = rng.standard_normal(o.w.shape)
    to_gpu(g, o)
    for _ in range(2):
        o.lib.ox_bcswap(o.ctx, vp(o.w), case.nv)
        g.lib.stx_bcswap(g.ctx, S(g), vp(g.w), case.nv)
    assert np.array_equal(g.host_w(), o.w)
    v = o.w_aux[case.J("DIV")]
    v[:] = rng.standard_normal(v.shape)
    to_gpu(g, o)
    o.lib.ox_bcextr_var(o.ctx, vp(v))
    g.lib.stx_bcextr_var(g.ctx, S(g), g.aux_slot(case.J("DIV")))
    assert np.array_equal(g.host_w_aux(), o.w_aux)


# ------------------------------------------------------------------ convective fluxes
EULER_CASES = [
    dict(sensor_threshold=1e9, nkeep=0),                 # central, KEEP(0)
    dict(sensor_threshold=1e9, nkeep=2),                 # central, KEEP(2)
    dict(sensor_threshold=1e9, nkeep=-1),                # classical central
    dict(sensor_threshold=-1.0, weno_version=1),         # WENO5-Z characteristic everywhere
    dict(sensor_threshold=-1.0, weno_version=0),         # WENO5-JS characteristic
    dict(sensor_threshold=-1.0, flux_splitting=1),       # WENO5 Rusanov
    dict(sensor_threshold=0.02, sensor_type=0),          # hybrid: both branches present
    # every other scheme option the ABI accepts (stx_ctx_create: weno_scheme 1..4,
    # ep_order 2..8 even, nkeep -1..2; ng >= max(ep_order/2, weno_scheme))
    dict(sensor_threshold=1e9, nkeep=1),                 # central, KEEP(1)
    dict(sensor_threshold=1e9, nkeep=2, ep_order=2),     # 2nd-order central
    dict(sensor_threshold=1e9, nkeep=2, ep_order=4),     # 4th-order central
    dict(sensor_threshold=1e9, nkeep=2, ep_order=8, ng=4),   # 8th-order central (per-face sweep)
    dict(sensor_threshold=-1.0, weno_scheme=1),          # WENO1 (first-order upwind)
    dict(sensor_threshold=-1.0, weno_scheme=2),          # WENO3
    dict(sensor_threshold=-1.0, weno_scheme=4, ng=4),    # WENO7 (per-face sweep)
    dict(sensor_threshold=-1.0, weno_scheme=2, flux_splitting=1),    # WENO3 Rusanov
    dict(sensor_threshold=-1.0, weno_scheme=4, flux_splitting=1, ng=4),  # WENO7 Rusanov
    dict(sensor_threshold=0.02, sensor_type=1, weno_scheme=4, ep_order=8, ng=4),  # hybrid WENO7 / 8th order
]


@pytest.mark.parametrize("kw", EULER_CASES)
@pytest.mark.parametrize("dirn", [0, 1, 2])
def test_euler_flux_divergence(kw, dirn):
    case = H.synthetic_case(n=(140, 10, 9), seed=3, **kw)
    g, o = prime(case)
    rng = np.random.default_rng(5)
    fl0 = rng.standard_normal(o.fl.shape)
    o.fl[:] = fl0
    to_gpu(g, o)
    n = (case.nx, case.ny, case.nz)[dirn]
    o.lib.ox_euler(o.ctx, dirn, vp(o.w_aux), vp(o.fhat), vp(o.fl), 1, n)
    fn = (g.lib.stx_euler_x, g.lib.stx_euler_y, g.lib.stx_euler_z)[dirn]
    assert fn(g.ctx, S(g), vp(g.w_aux), vp(g.fl), 1, n, 0) == 0
    dg = g.fl.cpu().numpy() - fl0
    do = o.fl - fl0
    for m in range(case.nv):
        H.assert_close(dg[m], do[m], 1e-9, f"euler dir {dirn} var {m}")


def test_euler_overwrite_equals_zero_then_accumulate():
    case = H.synthetic_case(n=(30, 8, 6), seed=4, sensor_threshold=0.02, sensor_type=0)
    g, _ = prime(case)
    g.fl.fill_(123.0)
    assert g.lib.stx_euler_x(g.ctx, S(g), vp(g.w_aux), vp(g.fl), 1, case.nx, 1) == 0
    a = g.fl.clone()
    g.fl.zero_()
    assert g.lib.stx_euler_x(g.ctx, S(g), vp(g.w_aux), vp(g.fl), 1, case.nx, 0) == 0
    assert torch.equal(a, g.fl)


# ------------------------------------------------------------------ viscous fluxes
@pytest.mark.parametrize("n,order", [((150, 10, 9), 6), ((9, 12, 14), 6), ((40, 10, 9), 2), ((40, 10, 9), 4),
                                     ((40, 10, 9), 8)])
def test_visflx(n, order):
    """Both viscous modes at every visc_order the ABI accepts (visc_order =
    ep_order, multideal.F90:683-686; ng = 4 for the 8th-order stencil)."""
    case = H.synthetic_case(n=n, seed=6, ep_order=order, ng=max(3, order // 2))
    g, o = prime(case)
    rng = np.random.default_rng(7)
    fl0 = rng.standard_normal(o.fl.shape)
    for mode in (1, 2):
        o.fl[:] = fl0
        to_gpu(g, o)
        o.lib.ox_visflx(o.ctx, vp(o.w_aux), vp(o.fl), vp(o.fhat), mode)
        assert g.lib.stx_visflx(g.ctx, S(g), vp(g.w_aux), vp(g.fl), mode) == 0
        dg, do = g.fl.cpu().numpy() - fl0, o.fl - fl0
        for m in range(case.nv):
            H.assert_close(dg[m], do[m], 1e-9, f"visflx mode {mode} var {m}")


# ------------------------------------------------------------------ RK and dt
def test_rk_bookkeeping_and_compute_dt():
    case = H.synthetic_case(n=(16, 12, 10), seed=8)
    g, o = prime(case)
    rng = np.random.default_rng(9)
    o.fl[:] = rng.standard_normal(o.fl.shape)
    o.fln[:] = rng.standard_normal(o.fl.shape)
    to_gpu(g, o)
    o.lib.ox_init_flux(o.ctx, vp(o.fl), vp(o.fln), -17.0 / 60.0 * 1e-7)
    g.lib.stx_init_flux(g.ctx, S(g), vp(g.fl), vp(g.fln), -17.0 / 60.0 * 1e-7)
    assert np.array_equal(g.fln.cpu().numpy(), o.fln) and np.array_equal(g.fl.cpu().numpy(), o.fl)
    o.fl[:] = rng.standard_normal(o.fl.shape)
    to_gpu(g, o)
    o.lib.ox_update_flux(o.ctx, vp(o.fl), vp(o.fln), 5.0 / 12.0 * 1e-7)
    o.lib.ox_update_field(o.ctx, vp(o.w), vp(o.fln), None)
    g.lib.stx_rk_finish(g.ctx, S(g), vp(g.w), vp(g.fl), vp(g.fln), None, None, 5.0 / 12.0 * 1e-7, 0)
    # fln -= gamdt*fl contracts to one FMA on the GPU: rounding-level differences
    H.assert_close(g.fln.cpu().numpy(), o.fln, 1e-12, "fln")
    H.assert_close(g.host_w(), o.w, 1e-14, "w")
    out_o = (C.c_double * 9)()
    out_g = (C.c_double * 9)()
    o.lib.ox_compute_dt(o.ctx, vp(o.w_aux), None, out_o)
    assert g.lib.stx_compute_dt(g.ctx, S(g), vp(g.w_aux), None, out_g) == 0
    for q in range(9):
        assert abs(out_g[q] - out_o[q]) <= 1e-13 * abs(out_o[q]), (q, out_g[q], out_o[q])


# ------------------------------------------------------------------ chemistry
def hot_case(seed=10, n=(10, 8, 6), **kw):
    """A pre-ignition state hot enough for active chemistry."""
    return H.synthetic_case(n=n, seed=seed, T0=1300.0, amp_T=200.0, **kw)


def oracle_spread(case, run):
    """How far the oracle itself moves when its input state is perturbed by one
    ulp: the conditioning of an adaptive, error-controlled integration (accept /
    reject and Krylov-dimension decisions are discrete)."""
    res = []
    for pert in (0, 1):
        o = OracleSolver(case, threads=8)
        o.update_ghost(1)
        o.compute_aux(1, 1)
        if pert:
            o.w[:] = np.nextafter(o.w, np.inf)
        run(o)
        res.append(case.interior(o.w).copy())
        o.close()
    return np.abs(res[0] - res[1])


def test_rosenbrock_krylov_short_window():
    """One or two ROK4 sub-steps: GPU and oracle agree to 1e-9 relative."""
    case = hot_case()
    g, o = prime(case)
    dt_chem = 2e-7
    o.lib.ox_rosenbrock_krylov(o.ctx, vp(o.w), vp(o.w_aux), None, dt_chem, 0.0, dt_chem, 0)
    assert g.lib.stx_rosenbrock_krylov(g.ctx, S(g), vp(g.w), vp(g.w_aux), None, dt_chem, 0.0, dt_chem, 0) == 0
    wg, wo = case.interior(g.host_w()), case.interior(o.w)
    for m in range(case.nv):
        H.assert_close(wg[m], wo[m], 1e-9, f"rok4 w[{m}]", floor=1e-9 * np.abs(wo[:case.ns]).max() if m < case.ns else None)
    assert g.status() & ~0x1 == 0


def test_rosenbrock_krylov_long_window_within_method_conditioning():
    """Over 5 us the ROK4 result is sensitive at the 1e-5 level to last-bit changes
    (exp/pow of CUDA and libm differ by an ulp); the GPU must stay within 20x the
    oracle's own one-ulp spread, and within 1e-4 relative (the integrator's
    tolerance) everywhere."""
    case = hot_case()
    dt_chem = 5e-6
    run = lambda o: o.lib.ox_rosenbrock_krylov(o.ctx, vp(o.w), vp(o.w_aux), None, dt_chem, 0.0, dt_chem, 0)
    spread = oracle_spread(case, run)
    g, o = prime(case)
    run(o)
    assert g.lib.stx_rosenbrock_krylov(g.ctx, S(g), vp(g.w), vp(g.w_aux), None, dt_chem, 0.0, dt_chem, 0) == 0
    wg, wo = case.interior(g.host_w()), case.interior(o.w)
    d = np.abs(wg - wo)
    scale = np.abs(wo).reshape(case.nv, -1).max(axis=1)[:, None, None, None]
    assert np.all(d <= 20.0 * spread.max(axis=(1, 2, 3), keepdims=True) + 1e-12 * scale), d.max()
    assert np.all(d <= 1e-4 * np.maximum(np.abs(wo), 1e-6 * scale))
    assert np.median(d / np.maximum(np.abs(wo), 1e-6 * scale)) < 1e-8


def test_rosenbrock_krylov_simpler_splitting():
    case = hot_case(seed=11)
    g, o = prime(case)
    rng = np.random.default_rng(12)
    o.fl_sav[:] = 1e-3 * rng.standard_normal(o.fl_sav.shape)
    to_gpu(g, o)
    dt_chem = 1e-6
    o.lib.ox_rosenbrock_krylov(o.ctx, vp(o.w), vp(o.w_aux), vp(o.fl_sav), dt_chem, 0.0, dt_chem, 1)
    g.lib.stx_rosenbrock_krylov(g.ctx, S(g), vp(g.w), vp(g.w_aux), vp(g.fl_sav), dt_chem, 0.0, dt_chem, 1)
    wg, wo = case.interior(g.host_w()), case.interior(o.w)
    for m in range(case.nv):
        H.assert_close(wg[m], wo[m], 1e-9, f"rok4 simpler w[{m}]", floor=1e-9 * np.abs(wo[:case.ns]).max() if m < case.ns else None)


def test_rosenbrock_full_jacobian():
    """The central-difference Jacobian (h = 1e-6 w, kernels_gpu.F90:9169-9191)
    amplifies the ulp-level exp/pow differences by ~1/h, so the full-Jacobian
    result agrees to ~1e-9 relative (1e-8 stated)."""
    case = hot_case(seed=13, n=(6, 5, 4), rosenbrock_version=1)
    g, o = prime(case)
    dt_chem = 2e-6
    o.lib.ox_rosenbrock(o.ctx, vp(o.w), vp(o.w_aux), dt_chem, 0.0, dt_chem)
    assert g.lib.stx_rosenbrock(g.ctx, S(g), vp(g.w), vp(g.w_aux), dt_chem, 0.0, dt_chem) == 0
    wg, wo = case.interior(g.host_w()), case.interior(o.w)
    for m in range(case.nv):
        H.assert_close(wg[m], wo[m], 1e-8, f"ros w[{m}]", floor=1e-8 * np.abs(wo[:case.ns]).max() if m < case.ns else None)
    H.assert_close(case.interior(g.host_w_aux()[case.J("T")]), case.interior(o.w_aux[case.J("T")]), 1e-8, "ros T")


def test_explicit_chemistry_source():
    case = hot_case(seed=14, chemistry=1)
    g, o = prime(case)
    o.lib.ox_compute_chemistry(o.ctx, vp(o.w), vp(o.w_aux), vp(o.fl))
    assert g.lib.stx_compute_chemistry(g.ctx, S(g), vp(g.w), vp(g.w_aux), vp(g.fl)) == 0
    for m in range(case.ns):
        H.assert_close(g.fl.cpu().numpy()[m], o.fl[m], 1e-11, f"wdot[{m}]", floor=1e-11 * np.abs(o.fl[:case.ns]).max())


def test_status_bits_report_caps_without_faulting():
    """ros_maxsteps = 1 makes every cell hit the step cap: the kernel sets a status
    bit and returns; the context stays usable."""
    case = hot_case(seed=15, n=(4, 4, 4))
    case.ros_maxsteps = 1
    g, o = prime(case)
    g.status(reset=True)
    assert g.lib.stx_rosenbrock_krylov(g.ctx, S(g), vp(g.w), vp(g.w_aux), None, 1e-9, 0.0, 1e-5, 0) == 0
    bits = g.status(reset=True)
    assert bits & 0x2
    assert g.status() == 0
    g.compute_aux(1, 1)
    torch.cuda.synchronize()


# ------------------------------------------------------------------ whole steps
@pytest.mark.parametrize("splitting,version", [(2, 2), (1, 2), (2, 1)])
def test_advance_solution_3d(splitting, version):
    case = hot_case(seed=16, n=(16, 12, 10), splitting=splitting, rosenbrock_version=version,
                    sensor_threshold=0.02, sensor_type=0)
    g, o = pair(case)
    o.prepare()
    to_gpu(g, o)
    g.dt = o.dt
    for _ in range(2):
        o.step()
        g.step()
    # dt after one step inherits the state's parity (the "simpler" split runs a
    # 1 us ROK4 window, conditioned at the 1e-8 level)
    assert abs(g.dt - o.dt) <= 1e-7 * o.dt
    wg, wo = case.interior(g.host_w()), case.interior(o.w)
    if splitting == 1 and version == 2:
        # Strang + ROK4 integrates two half-step windows per step with adaptive
        # accept/reject: the oracle itself moves by ~5e-7 relative (species) and
        # ~3e-4 of the small momenta when its start state is perturbed by one ulp.
        # The GPU must stay within 20x that spread.
        res = []
        for pert in (0, 1):
            op = OracleSolver(case, threads=8)
            op.prepare()
            if pert:
                op.w[:] = np.nextafter(op.w, np.inf)
            for _ in range(2):
                op.step()
            res.append(case.interior(op.w).copy())
            op.close()
        spread = np.abs(res[0] - res[1]).reshape(case.nv, -1).max(axis=1)[:, None, None, None]
        scale = np.abs(wo).reshape(case.nv, -1).max(axis=1)[:, None, None, None]
        d = np.abs(wg - wo)
        assert np.all(d <= 20.0 * spread + 1e-12 * scale), (d.reshape(case.nv, -1).max(axis=1), spread.ravel())
        assert np.median(d / np.maximum(np.abs(wo), 1e-6 * scale)) < 1e-5   # the spread's own median is 3e-7
        return
    for m in range(case.nv):
        H.assert_close(wg[m], wo[m], 1e-8, f"step w[{m}]", floor=1e-8 * np.abs(wo[:case.ns]).max() if m < case.ns else None)


def test_reactive_shock_tube_steps():
    """examples/reactive_shock_tube inputs (reflecting wall, extrapolation, WENO
    everywhere, Strang + ROK4) on 400 cells: 30 steps against the oracle."""
    case = H.shock_tube_case(nx=400)
    g, o = pair(case)
    o.prepare()
    g.prepare()
    assert np.array_equal(g.host_w(), o.w)
    for _ in range(30):
        o.step()
        g.step()
    wg, wo = case.interior(g.host_w()), case.interior(o.w)
    for m in range(case.nv):
        H.assert_close(wg[m], wo[m], 1e-8, f"shock tube w[{m}]", floor=1e-8 * np.abs(wo[:case.ns]).max() if m < case.ns else None)


def test_batch_reactor_on_gpu_matches_reference_output():
    """The 0-D reactor of examples/batch_reactor replicated on 64 identical cells:
    every cell follows the reference's own FP64 trajectory through ignition."""
    case, gold = H.batch_case(4, 4, 4)
    ref = np.array(gold["reference"])
    g = Solver(case)
    g.prepare()
    out = []
    for n in range(1, 3001):
        g.step()
        if n % 10 == 0:
            out.append(case.interior(g.w_aux[case.J("T")].cpu().numpy()).ravel())
    out = np.array(out)
    assert np.ptp(out, axis=1).max() == 0.0          # identical cells, identical results
    dT = np.abs(out[:, 0] - ref[:300, 2])
    assert dT.max() < 0.02, dT.max()


# ------------------------------------------------------------------ remaining ghost tags, bc_nr
@pytest.mark.parametrize("bc", [(4, 4, 4, 4, 4, 4), (7, 7, 7, 7, 7, 7), (2, 2, 5, 5, 0, 0), (2, 8, 6, 6, 0, 0)])
def test_update_ghost_remaining_tags(bc):
    """bcextr_sub (4), bcsym (5, y sides), bcwall (6, isothermal, y sides) and
    bcoutopenfoam (7) against the oracle, on a field whose velocity has both
    signs at every face (the outflow fill's switch)."""
    case = H.synthetic_case(n=(14, 10, 8), bc=bc, seed=11, T_wall=950.0)
    g, o = pair(case)
    o.compute_aux(1, 1)            # w_aux (the Newton guesses and mass fractions the fills read)
    to_gpu(g, o)
    o.update_ghost(0)
    g.update_ghost(0)
    wg, wag = g.host_w(), g.host_w_aux()
    if 4 in bc or 6 in bc:
        for m in range(case.nv):
            H.assert_close(wg[m], o.w[m], 1e-12, f"ghost w[{m}] tags {bc}")
        for m in range(case.ns):
            H.assert_close(wag[m], o.w_aux[m], 1e-14, f"w_aux[{m}] tags {bc}")
    else:
        assert np.array_equal(wg, o.w)        # copies and sign flips: bit-exact
    assert not np.array_equal(wg, case.w)    # the fills wrote something


NR_CASES = [
    # (bc tags, bc_nr tags): every treatment on every side
    ((2, 2, 0, 0, 0, 0), (1, 1, 0, 0, 0, 0)),
    ((2, 2, 2, 2, 0, 0), (2, 3, 1, 6, 0, 0)),
    ((0, 0, 2, 2, 2, 2), (0, 0, 3, 2, 6, 1)),
    ((7, 4, 0, 0, 2, 2), (6, 2, 0, 0, 3, 1)),
]


@pytest.mark.parametrize("bc,nr", NR_CASES)
def test_bc_nr_matches_oracle(bc, nr):
    """bc_nr_lat_{x,y,z}: the characteristic treatment added to fl at the
    boundary cells of each face, against the oracle's dense eigenvector products."""
    case = H.synthetic_case(n=(14, 10, 8), bc=bc, bc_nr=nr, seed=12)
    g, o = pair(case)
    o.update_ghost(1)
    o.compute_aux(1, 1)
    to_gpu(g, o)
    rng = np.random.default_rng(13)
    fl0 = rng.standard_normal(o.fl.shape)
    o.fl[:] = fl0
    g.fl.copy_(torch.from_numpy(fl0))
    o.lib.ox_bc_nr(o.ctx, vp(o.w_aux), vp(o.w), vp(o.fl))
    assert g.lib.stx_bc_nr(g.ctx, S(g), vp(g.w_aux), vp(g.w), vp(g.fl)) == 0
    dg, do = g.fl.cpu().numpy() - fl0, o.fl - fl0
    assert np.abs(do).max() > 0
    for m in range(case.nv):
        H.assert_close(dg[m], do[m], 1e-10, f"bc_nr var {m}", floor=1e-10 * np.abs(do).max())


@pytest.mark.parametrize("bc,nr", NR_CASES[1:3])
def test_steps_with_characteristic_boundaries(bc, nr):
    """Whole steps (Strang + ROK4, hybrid fluxes, viscous fluxes) with the
    characteristic boundaries and the convective sweeps cut to eul_*."""
    case = H.synthetic_case(n=(16, 10, 8), bc=bc, bc_nr=nr, seed=14, cfl=-5e-9)
    assert case.eul != [1, case.nx, 1, case.ny, 1, case.nz]
    g, o = pair(case)
    o.prepare()
    g.prepare()
    for _ in range(2):
        o.step()
        g.step()
    wg, wo = case.interior(g.host_w()), case.interior(o.w)
    for m in range(case.nv):
        H.assert_close(wg[m], wo[m], 1e-8, f"nr steps w[{m}]",
                       floor=1e-8 * np.abs(wo[:case.ns]).max() if m < case.ns else None)
