"""ctypes mirror of ``include/stx.h`` and loaders for the native libraries.

``load_stx()`` loads the product library ``csrc/libstx.so`` (CUDA, sm_100a) and
fails loudly when it is missing.  ``load_oracle()`` loads the CPU oracle used by
the tests and by the bench's CPU baseline; the solver never calls it.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)                    # prop-streams2_b200/
REPO_ROOT = os.path.dirname(PKG_ROOT)
STX_SO = os.path.join(PKG_ROOT, "csrc", "libstx.so")
ORACLE_SO = os.path.join(REPO_ROOT, "oracle", "liboracle.so")

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int32)


class StxTables(C.Structure):
    _fields_ = [
        ("ns", C.c_int32), ("nr", C.c_int32),
        ("indx_cp_l", C.c_int32), ("indx_cp_r", C.c_int32), ("nsetcv", C.c_int32), ("num_t_tab", C.c_int32),
        ("t_min_tab", C.c_double), ("dt_tab", C.c_double), ("R_univ", C.c_double),
        ("mw", dp), ("mwinv", dp), ("rgas", dp), ("trange", dp), ("cp_coeff", dp), ("cv_coeff", dp),
        ("visc", dp), ("lam", dp), ("diffbin", dp),
        ("reac_ty", ip), ("is_rev", ip),
        ("arr_a", dp), ("arr_b", dp), ("arr_ea", dp), ("falloff", dp),
        ("tb_eff", dp), ("r_coeffs", dp), ("p_coeffs", dp), ("kc_tab", dp),
        ("n_eoi", C.c_int32), ("aw_eoi", dp), ("coeff_eoi", dp), ("nainsp", ip), ("beta0", dp),
    ]


class StxGrid(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("ng", C.c_int32),
        ("x", dp), ("y", dp), ("z", dp),
        ("dcsidx", dp), ("detady", dp), ("dzitdz", dp),
        ("dcsidxs", dp), ("detadys", dp), ("dzitdzs", dp),
    ]


class StxParams(C.Structure):
    _fields_ = [
        ("nv_aux", C.c_int32),
        ("p0", C.c_double), ("rho0", C.c_double), ("u0", C.c_double), ("eps_sensor", C.c_double),
        ("tol_iter_nr", C.c_double),
        ("ep_order", C.c_int32), ("nkeep", C.c_int32), ("weno_scheme", C.c_int32), ("weno_version", C.c_int32),
        ("flux_splitting", C.c_int32),
        ("sensor_type", C.c_int32), ("visc_order", C.c_int32), ("conservative_viscous", C.c_int32),
        ("sensor_threshold", C.c_double),
        ("bctags", C.c_int32 * 6), ("bctags_nr", C.c_int32 * 6), ("force_zero_flux", C.c_int32 * 6),
        ("eul_imin", C.c_int32), ("eul_imax", C.c_int32), ("eul_jmin", C.c_int32), ("eul_jmax", C.c_int32),
        ("eul_kmin", C.c_int32), ("eul_kmax", C.c_int32),
        ("enable_chemistry", C.c_int32), ("rosenbrock_version", C.c_int32), ("operator_splitting", C.c_int32),
        ("ros_maxsteps", C.c_int32), ("ros_maxtry", C.c_int32),
        ("ros_eps", C.c_double),
        ("nrk", C.c_int32),
        ("rhork", C.c_double * 4), ("gamrk", C.c_double * 4),
        ("winf", dp),
        ("T_wall", C.c_double),
    ]


class StxFields(C.Structure):
    _fields_ = [("w", C.c_void_p), ("w_aux", C.c_void_p), ("fl", C.c_void_p), ("fln", C.c_void_p),
                ("fl_sav", C.c_void_p), ("fluid_mask", C.c_void_p)]


class StxKprof(C.Structure):
    _fields_ = [("launches", C.c_int64), ("timed", C.c_int64), ("ms", C.c_double), ("bytes", C.c_double)]


class StxTuning(C.Structure):
    _fields_ = [("sweep_kind", C.c_int32 * 3), ("weno_list", C.c_int32 * 3), ("chem_ctas_per_sm", C.c_int32),
                ("chem_ctas_max", C.c_int32), ("batch_ctas_max", C.c_int32), ("sweep_ms", C.c_float * 3),
                ("chem_ms", C.c_float)]


_VP = C.c_void_p
_I = C.c_int
_D = C.c_double

# stx_exchange_fn: int (*)(void *user, void *stream, double *field, int nvar)
EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int)

# (name, restype, argtypes) of every entry point declared in include/stx.h
STX_SIGNATURES = [
    ("stx_abi_version", C.c_int, []),
    ("stx_strerror", C.c_char_p, [_I]),
    ("stx_ctx_create", _I, [C.POINTER(StxParams), C.POINTER(StxTables), C.POINTER(StxGrid), C.POINTER(_VP)]),
    ("stx_ctx_create_like", _I, [_VP, C.POINTER(StxParams), C.POINTER(StxGrid), C.POINTER(_VP)]),
    ("stx_ctx_create_like_on", _I, [_VP, C.POINTER(StxParams), C.POINTER(StxGrid), _VP, C.POINTER(_VP)]),
    ("stx_set_exchange", _I, [_VP, EXCHANGE_FN, _VP]),
    ("stx_ctx_destroy", _I, [_VP]),
    ("stx_eval_aux", _I, [_VP, _VP, _VP, _VP, _I, _I, _I, _I, _I, _I]),
    ("stx_compute_aux", _I, [_VP, _VP, _VP, _VP, _I, _I]),
    ("stx_eval_aux2", _I, [_VP, _VP, _VP]),
    ("stx_bcextr_var", _I, [_VP, _VP, _VP]),
    ("stx_bcswap", _I, [_VP, _VP, _VP, _I]),
    ("stx_update_ghost", _I, [_VP, _VP, _VP, _I]),
    ("stx_update_ghost_aux", _I, [_VP, _VP, _VP, _VP, _I]),
    ("stx_bc_nr", _I, [_VP, _VP, _VP, _VP, _VP]),
    ("stx_euler_x", _I, [_VP, _VP, _VP, _VP, _I, _I, _I]),
    ("stx_euler_y", _I, [_VP, _VP, _VP, _VP, _I, _I, _I]),
    ("stx_euler_z", _I, [_VP, _VP, _VP, _VP, _I, _I, _I]),
    ("stx_visflx", _I, [_VP, _VP, _VP, _VP, _I]),
    ("stx_init_flux", _I, [_VP, _VP, _VP, _VP, _D]),
    ("stx_init_flux_simpler", _I, [_VP, _VP, _VP, _VP, _VP, _D]),
    ("stx_sav_flx", _I, [_VP, _VP, _VP, _VP]),
    ("stx_update_flux", _I, [_VP, _VP, _VP, _VP, _D]),
    ("stx_update_simpler_flux", _I, [_VP, _VP, _VP, _VP, _VP, _D]),
    ("stx_update_field", _I, [_VP, _VP, _VP, _VP, _VP]),
    ("stx_rk_finish", _I, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _D, _I]),
    ("stx_compute_dt", _I, [_VP, _VP, _VP, _VP, C.POINTER(C.c_double)]),
    ("stx_compute_residual", _I, [_VP, _VP, _VP, _VP, _VP, _D, C.POINTER(C.c_double)]),
    ("stx_rosenbrock", _I, [_VP, _VP, _VP, _VP, _D, _D, _D]),
    ("stx_rosenbrock_krylov", _I, [_VP, _VP, _VP, _VP, _VP, _D, _D, _D, _I]),
    ("stx_compute_chemistry", _I, [_VP, _VP, _VP, _VP, _VP]),
    ("stx_batch0d_integrate", _I, [_VP, _VP, _I, _VP, _VP, _VP, _D, _D, _D, _D, _I, _VP, _VP, _VP, _VP, _VP]),
    ("stx_set_precision", _I, [_VP, _I]),
    ("stx_graph_create", _I, [_VP, C.POINTER(StxFields), _D, _I, C.POINTER(_VP)]),
    ("stx_graph_create_cfl", _I, [_VP, C.POINTER(StxFields), _D, _I, C.POINTER(_VP)]),
    ("stx_graph_launch", _I, [_VP, _VP, _D]),
    ("stx_graph_state", _I, [_VP, _VP, C.POINTER(_D), C.POINTER(_D)]),
    ("stx_graph_destroy", _I, [_VP]),
    ("stx_rk_sync", _I, [_VP, _VP, C.POINTER(StxFields), _D, _I]),
    ("stx_advance_solution", _I, [_VP, _VP, C.POINTER(StxFields), _D, _D]),
    ("stx_status", _I, [_VP, _VP, C.POINTER(C.c_uint32), _I]),
    ("stx_status_enqueue", _I, [_VP, _VP, _VP, _I]),
    ("stx_get_tuning", _I, [_VP, C.POINTER(StxTuning)]),
    ("stx_set_tuning", _I, [_VP, C.POINTER(StxTuning)]),
    ("stx_autotune", _I, [_VP, _VP, C.POINTER(StxFields), _D, C.POINTER(StxTuning)]),
    ("stx_profile_enable", _I, [_VP, _I]),
    ("stx_profile_read", _I, [_VP, C.POINTER(StxKprof)]),
]

ORACLE_SIGNATURES = [
    ("ox_ctx_create", _VP, [C.POINTER(StxParams), C.POINTER(StxTables), C.POINTER(StxGrid)]),
    ("ox_ctx_destroy", None, [_VP]),
    ("ox_set_threads", None, [_I]),
    ("ox_status", C.c_uint32, [_VP, _I]),
    ("ox_eval_aux", None, [_VP, _VP, _VP, _I, _I, _I, _I, _I, _I]),
    ("ox_compute_aux", None, [_VP, _VP, _VP, _I, _I]),
    ("ox_eval_aux2", None, [_VP, _VP]),
    ("ox_bcextr_var", None, [_VP, _VP]),
    ("ox_bcswap", None, [_VP, _VP, _I]),
    ("ox_update_ghost", None, [_VP, _VP, _I]),
    ("ox_update_ghost_aux", None, [_VP, _VP, _VP, _I]),
    ("ox_bc_nr", None, [_VP, _VP, _VP, _VP]),
    ("ox_euler", None, [_VP, _I, _VP, _VP, _VP, _I, _I]),
    ("ox_visflx", None, [_VP, _VP, _VP, _VP, _I]),
    ("ox_init_flux", None, [_VP, _VP, _VP, _D]),
    ("ox_update_flux", None, [_VP, _VP, _VP, _D]),
    ("ox_update_field", None, [_VP, _VP, _VP, _VP]),
    ("ox_compute_dt", None, [_VP, _VP, _VP, C.POINTER(C.c_double)]),
    ("ox_compute_residual", None, [_VP, _VP, _VP, _VP, _D, C.POINTER(C.c_double)]),
    ("ox_rosenbrock", None, [_VP, _VP, _VP, _D, _D, _D]),
    ("ox_rosenbrock_krylov", None, [_VP, _VP, _VP, _VP, _D, _D, _D, _I]),
    ("ox_compute_chemistry", None, [_VP, _VP, _VP, _VP]),
    ("ox_rk_sync", None, [_VP, C.POINTER(StxFields), _VP, _D, _I]),
    ("ox_advance_solution", None, [_VP, C.POINTER(StxFields), _VP, _D, _D]),
    ("ox_krylov_cell", None, [_VP, _VP, _D, _D, _VP, _D, _D, _D, _I]),
    ("ox_rosenbrock_cell", None, [_VP, _VP, _VP, _VP, _D, _D, _D]),
    ("ox_temperature_from_e", _D, [_VP, _D, _D, _VP]),
    ("ox_batch0d_cp", None, [_VP, _I, _VP, _VP, _VP, _D, _D, _D, _D, _I, _VP, _VP, _VP, _VP, _VP]),
]


def _bind(lib, sigs):
    for name, res, args in sigs:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_stx = None
_oracle = None


def load_stx(path: str = STX_SO):
    """Load libstx.so.  Raises if the CUDA extension has not been built: there is
    no CPU fallback for the solver."""
    global _stx
    if _stx is None:
        if not os.path.exists(path):
            raise RuntimeError(f"libstx.so not found at {path}; build it with "
                               f"`python __graft_entry__.py build` (or make -C prop-streams2_b200/csrc)")
        _stx = _bind(C.CDLL(path), STX_SIGNATURES)
    return _stx


def load_oracle(path: str = ORACLE_SO):
    """Load the CPU oracle (test infrastructure only)."""
    global _oracle
    if _oracle is None:
        if not os.path.exists(path):
            raise RuntimeError(f"liboracle.so not found at {path}; run make -C oracle")
        _oracle = _bind(C.CDLL(path), ORACLE_SIGNATURES)
    return _oracle


def check(rc: int, what: str = ""):
    if rc != 0:
        lib = load_stx()
        raise RuntimeError(f"{what} failed: {lib.stx_strerror(rc).decode()} ({rc})")
