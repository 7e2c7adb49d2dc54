"""CPU tests: the oracle and the table generator pinned against the reference's
own outputs and constants (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import helpers as H
from stx import case as CS
from stx import mech as M


def test_thermo_constants_match_reference_run_log():
    """examples/laminar_premix_flame/data.dat:10-29 prints R_mix, cp0, cv0, gamma,
    rho0, mu0, c0 and h(298.15) of every species for its multideal.ini."""
    pins = H.golden("flame_log_pins.json")
    mech = H.mechanism("flame_11sp")
    tb = M.build_tables(mech, 101325.0)
    Y = np.array([float(pins["ini"]["ref_state"][f"init_Y_{k + 1:02d}"]) for k in range(mech.ns)])
    T0 = float(pins["ini"]["ref_state"]["t0"])
    rm = float(np.dot(tb.rgas, Y))
    cp = M.mixture_cp(tb, T0, Y)
    assert abs(rm / pins["rmixt0"] - 1) < 1e-14
    assert abs(cp / pins["cp0"] - 1) < 1e-14
    assert abs((cp - rm) / pins["cv0"] - 1) < 1e-14
    assert abs(cp / (cp - rm) / pins["gam"] - 1) < 1e-14
    assert abs(101325.0 / rm / T0 / pins["rho0"] - 1) < 1e-14
    assert abs(np.sqrt(cp / (cp - rm) * rm * T0) / pins["c0"] - 1) < 1e-14
    for k, h in enumerate(pins["h298"]):
        assert abs(tb.h298[k] - h) <= 1e-9 * max(abs(h), 1e3), (mech.names[k], tb.h298[k], h)
    # viscosity comes from the project's kinetic-theory tables (Cantera absent): loose pin
    mu = M.mixture_viscosity(tb, T0, Y)
    assert abs(mu / pins["mu0"] - 1) < 0.02


def test_mechanism_parser_counts():
    assert H.mechanism("shock_tube_9sp").nr == 18
    assert H.mechanism("flame_11sp").nr == 21
    h2air = H.mechanism("h2air_9sp")
    assert h2air.ns == 9 and h2air.nr == 21 and "N2" in h2air.names
    kero = H.mechanism("keromnes_14sp")
    assert kero.ns == 14 and kero.nr == 37
    types = [r.rtype for r in kero.reactions]
    assert types.count(M.RT_TROE) == 5 and types.count(M.RT_LINDEMANN) == 1 and types.count(M.RT_THREEBODY) == 5


def test_equilibrium_constant_consistency():
    """K_c of a reaction and of its reverse multiply to one (NASA Gibbs data)."""
    mech = H.mechanism("h2air_9sp")
    tb = M.build_tables(mech, 101325.0, with_transport=False)
    r = mech.reactions[0]
    rev = M.Reaction("rev", r.products, r.reactants, True, 0, [1.0, 0.0, 0.0])
    tb2 = M.build_tables(M.Mechanism(mech.species, [r, rev]), 101325.0, with_transport=False)
    prod = tb2.kc_tab[:, 0] * tb2.kc_tab[:, 1]
    assert np.allclose(prod, 1.0, rtol=1e-10)
    assert np.all(tb.kc_tab > 0)


def test_fluid_prop_bin_round_trip(tmp_path):
    mech = H.mechanism("shock_tube_9sp")
    tb = M.build_tables(mech, 7173.0, 200.0, 1200.0, 1.0)
    fn = str(tmp_path / "fluid_prop.bin")
    M.write_fluid_prop(fn, tb, 7173.0)
    rd = M.read_fluid_prop(fn, 7173.0, 9)
    for name in ("mw", "rgas", "h298", "trange", "cp_coeff", "cv_coeff", "visc", "lam", "diffbin", "arr_a", "arr_b",
                 "arr_ea", "falloff", "tb_eff", "r_coeffs", "p_coeffs", "kc_tab"):
        a, b = getattr(tb, name), getattr(rd, name)
        assert np.allclose(a, b, rtol=1e-15, atol=0), name
    assert rd.num_t_tab == tb.num_t_tab and rd.names == tb.names
    with pytest.raises(ValueError):
        M.read_fluid_prop(fn, 7173.0, 11)


def test_oracle_temperature_inverts_energy():
    mech = H.mechanism("h2air_9sp")
    Y = H.h2air_Y(0.7, mech)
    case = H.synthetic_case(n=(4, 4, 4))
    from driver import OracleSolver
    o = OracleSolver(case, threads=1)
    for T in (250.0, 800.0, 999.0, 1000.0, 1001.0, 2400.0, 3400.0):
        e = M.mixture_e(case.tb, T, Y)
        Tn = o.lib.ox_temperature_from_e(o.ctx, e, 1000.0, Y.ctypes.data_as(C.c_void_p))
        assert abs(Tn - T) < 1e-9 * T
    o.close()


@pytest.mark.slow
def test_oracle_batch_reactor_matches_reference_output():
    """examples/syngas_mech_eval/OUTPUT/output_Keromnes2013.dat is the reference's own
    FP64 0-D run of examples/batch_reactor; the oracle replays its run loop
    (Strang splitting, ROK4, Wray RK3 on a periodic 1x1x1 cell) for 3000 steps,
    through ignition.  Cantera tolerances of result_comp.py:7-9 apply on top."""
    from driver import OracleSolver
    case, g = H.batch_case()
    ref = np.array(g["reference"])
    cant = np.array(g["cantera"])
    o = OracleSolver(case, threads=1)
    o.prepare()
    assert o.dt == 2e-7
    J_T, J_R = case.J("T"), case.J("R")
    n_out = 300
    out = []
    for n in range(1, 10 * n_out + 1):
        o.step()
        if n % 10 == 0:
            out.append((o.time, case.interior(o.w_aux)[J_R].item(), case.interior(o.w_aux)[J_T].item()))
    out = np.array(out)
    assert np.allclose(out[:, 0], ref[:n_out, 0], rtol=1e-12)
    dT = np.abs(out[:, 2] - ref[:n_out, 2])
    assert dT.max() < 0.02, dT.max()
    assert out[-1, 2] > 2400.0                      # ignited
    assert np.abs(out[:, 2] - cant[:n_out, 2]).max() < 1.0
    assert np.abs(out[:, 1] - cant[:n_out, 1]).max() < 1e-5
    o.close()


def test_oracle_constant_pressure_reactor_conserves_h_and_ignites():
    """The constant-pressure 0-D reactor of the oracle (the checker of
    stx_batch0d_integrate): h and sum Y_k stay constant through ignition,
    ignition is detected at T > 1.05 T0 and the run ends at 2 t_ign, and a
    hotter start ignites earlier."""
    from stx import configs, native
    from stx.reactors import sample_h2air
    mech = configs.mechanism("h2air_9sp")
    tb = M.build_tables(mech, 101325.0, 200.0, 5500.0, 1.0)
    cfg = CS.default_ini(1, 1, 1, L=(1e-3,) * 3, Y=np.full(mech.ns, 1.0 / mech.ns), ns=mech.ns)
    case = CS.Case(cfg, tb, alloc_fields=False)
    lib = native.load_oracle()
    par, tab, grid = case.params_struct(), case.tables_struct(), case.grid_struct()
    ctx = lib.ox_ctx_create(C.byref(par), C.byref(tab), C.byref(grid))
    lib.ox_set_threads(4)
    T0 = np.array([1300.0, 1400.0, 1500.0, 1450.0])
    p0 = np.array([1.0, 1.0, 1.0, 5.0]) * 101325.0
    Y0 = np.ascontiguousarray(np.stack([configs.h2air_Y(1.0, mech)] * 4, axis=1))
    n = 4
    Y = np.empty_like(Y0); T = np.empty(n); ti = np.empty(n); te = np.empty(n); ns = np.empty(n, dtype=np.int32)
    vp = lambda a: C.c_void_p(a.ctypes.data)
    lib.ox_batch0d_cp(ctx, n, vp(T0), vp(p0), vp(Y0), 1e-3, 1e-8, 1.05, 2.0, 100000, vp(Y), vp(T), vp(ti), vp(te),
                      vp(ns))
    assert lib.ox_status(ctx, 1) & 0x2 == 0
    lib.ox_ctx_destroy(ctx)
    assert np.all(ti > 0) and np.allclose(te, 2.0 * ti, rtol=1e-12)
    assert ti[0] > ti[1] > ti[2]
    assert np.max(np.abs(Y.sum(axis=0) - 1.0)) < 1e-12
    for r in range(n):
        h0 = M.mixture_h(tb, T0[r], Y0[:, r])
        assert abs(M.mixture_h(tb, T[r], np.maximum(Y[:, r], 0.0)) - h0) < 1e-9 * abs(h0) + 1e-6
        assert T[r] > 2000.0                        # burnt (at 2 t_ign, near but below T_ad)
    # the sampler of the batched workload is seeded and in range
    a, b, c = sample_h2air(16, 3, mech)
    assert np.all((a >= 900) & (a <= 1500)) and np.all((b >= 101325.0) & (b <= 40 * 101325.0 + 1e-6))
    assert np.allclose(c.sum(axis=0), 1.0)


def _declared_symbols():
    hdr = open(os.path.join(H.REPO, "include", "stx.h")).read()
    return sorted(set(re.findall(r"\b(stx_[a-z0-9_]+)\s*\(", hdr)))


def test_libstx_exports_every_declared_symbol():
    so = os.path.join(H.REPO, "prop-streams2_b200", "csrc", "libstx.so")
    if not os.path.exists(so):
        pytest.skip("libstx.so not built (run __graft_entry__.build())")
    out = subprocess.run(["nm", "-D", "--defined-only", so], capture_output=True, text=True, check=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if " T " in l)
    missing = [s for s in _declared_symbols() if s not in exported]
    assert not missing, missing
    lib = C.CDLL(so)          # loads without a GPU (cudart is linked statically)
    lib.stx_abi_version.restype = C.c_int
    assert lib.stx_abi_version() == 1


def test_every_declared_entry_point_has_a_python_binding():
    """Every stx_* function of include/stx.h carries a ctypes signature in
    stx/native.py (the allocation-free entry point is bound by its own test)."""
    from stx import native
    have = {s[0] for s in native.STX_SIGNATURES} | {"stx_rosenbrock_krylov_noalloc"}
    missing = [s for s in _declared_symbols() if s not in have]
    assert not missing, missing


def test_ctx_create_rejects_unsupported_options_without_touching_the_gpu():
    so = os.path.join(H.REPO, "prop-streams2_b200", "csrc", "libstx.so")
    if not os.path.exists(so):
        pytest.skip("libstx.so not built")
    from stx.native import load_stx
    lib = load_stx()
    case = H.synthetic_case(n=(4, 4, 4))
    par, tab, grid = case.params_struct(), case.tables_struct(), case.grid_struct()
    ctx = C.c_void_p()
    par.bctags[0] = 10                     # recycling-rescaling inflow: not on this path
    assert lib.stx_ctx_create(C.byref(par), C.byref(tab), C.byref(grid), C.byref(ctx)) == -4
    par.bctags[0] = 0
    par.bctags_nr[1] = 1                   # characteristic treatment of a periodic face
    assert lib.stx_ctx_create(C.byref(par), C.byref(tab), C.byref(grid), C.byref(ctx)) == -1
    par.bctags[0], par.bctags[1] = 2, 2
    par.bctags_nr[1] = 4                   # not a treatment bc_nr knows
    assert lib.stx_ctx_create(C.byref(par), C.byref(tab), C.byref(grid), C.byref(ctx)) == -4
    par.bctags_nr[1] = 1                   # eul_imax not moved off the face as bc_preproc does
    assert lib.stx_ctx_create(C.byref(par), C.byref(tab), C.byref(grid), C.byref(ctx)) == -4
    par.bctags[0], par.bctags[1], par.bctags_nr[1] = 0, 0, 0
    tab.ns = 7                             # species count not compiled in
    assert lib.stx_ctx_create(C.byref(par), C.byref(tab), C.byref(grid), C.byref(ctx)) == -4
    assert lib.stx_ctx_create(None, C.byref(tab), C.byref(grid), C.byref(ctx)) == -1
    assert lib.stx_strerror(-4) == b"option outside the supported hot path"


def test_case_rejects_out_of_scope_inputs():
    cfg = CS.default_ini(4, 4, 4, Y=H.h2air_Y(0.7, H.mechanism("h2air_9sp")))
    cfg.set("bc", "xmin", 10)               # recycling-rescaling inflow
    cfg.set("bc", "xmax", 2)
    with pytest.raises(ValueError):
        CS.Case(cfg, H.tables("h2air_9sp", 101325.0))


def _c_struct_fields(hdr, name):
    """Field names of `typedef struct name { ... } name;` in declaration order."""
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), hdr, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        # "const double *a, *b" / "int32_t bctags[6]" -> a, b / bctags
        rest = re.sub(r"^(const\s+)?(unsigned\s+)?[A-Za-z_0-9]+\s*", "", decl)
        for part in rest.split(","):
            names.append(re.sub(r"[\s*]|\[.*?\]", "", part))
    return names


def _f_type_fields(src, name):
    body = re.search(r"type, bind\(c\) :: %s\n(.*?)end type %s" % (name, name), src, re.S).group(1)
    names = []
    for line in body.splitlines():
        line = line.split("!", 1)[0].strip()
        if "::" in line:
            for part in line.split("::", 1)[1].split(","):
                names.append(re.sub(r"\(.*?\)|\s", "", part))
    return [n for n in names if n]


def test_fortran_interface_module_matches_the_header():
    """include/stx_interface.F90 (the iso_c_binding module a Fortran host uses)
    binds every entry point of include/stx.h, and its derived types list the C
    structs' fields in the same order (no Fortran compiler here, so this is the
    check that keeps the two in step)."""
    hdr = open(os.path.join(H.REPO, "include", "stx.h")).read()
    src = open(os.path.join(H.REPO, "include", "stx_interface.F90")).read()
    bound = set(re.findall(r'bind\(c, name="(stx_[a-z0-9_]+)"\)', src))
    missing = [s for s in _declared_symbols() if s not in bound]
    assert not missing, missing
    assert not bound - set(_declared_symbols()), bound - set(_declared_symbols())
    for st in ("stx_tables", "stx_grid", "stx_params", "stx_fields", "stx_tuning", "stx_kprof"):
        assert _f_type_fields(src, st) == _c_struct_fields(hdr, st), st
    for code in re.findall(r"#define (STX_E_[A-Z_]+)\s+(-?\d+)", hdr):
        assert re.search(r"\b%s = %s\b" % code, src), code
