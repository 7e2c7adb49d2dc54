"""CPU tests of the output and restart files (stx/output.py) against the
reference's formats: the progress lines of its own flame run log, the byte
layout of its serial and MPI-IO restart files, and the field_info file."""
import os
import struct

import numpy as np

import helpers as H
from stx import output as O


def test_progress_lines_reproduce_the_reference_run_log():
    """print_progress '(1I10,F18.10,20ES20.10)': every progress line of
    examples/laminar_premix_flame/data.dat, rebuilt from its parsed values,
    equals the reference's text character for character."""
    g = H.golden("flame_progress.json")
    for row, line in zip(g["rows"], g["lines"]):
        icyc, step_time, dt, time = row[:4]
        assert O.progress_line(icyc, step_time, dt, time, row[4:]) == line


def test_fortran_es_edge_cases():
    assert O.fortran_es(0.0) == "    0.0000000000E+00"
    assert O.fortran_es(-1.5e-300) == "   -1.5000000000-300"
    assert O.fortran_es(9.99999999999e99) == "    1.0000000000+100"
    assert len(O.fortran_es(-2.9798695615e2)) == 20


def _small_case():
    return H.synthetic_case(n=(5, 4, 3), seed=30)


def test_serial_restart_layout_and_round_trip(tmp_path):
    """write_field_serial: one unformatted record of w(1:nv,1:nx,1:ny,1:nz) with
    4-byte length markers, the variable index fastest."""
    case = _small_case()
    w = np.random.default_rng(1).standard_normal(case.w.shape)
    p = str(tmp_path / O.restart_serial_name())
    O.write_restart_serial(p, case, w)
    raw = open(p, "rb").read()
    n = case.nv * case.nx * case.ny * case.nz * 8
    assert len(raw) == n + 8
    assert struct.unpack("=i", raw[:4])[0] == n and struct.unpack("=i", raw[-4:])[0] == n
    vals = np.frombuffer(raw[4:-4], dtype=np.float64)
    ng = case.ng
    # Fortran w(l, i, j, k) at offset (l-1) + nv*((i-1) + nx*((j-1) + ny*(k-1)))
    for (l, i, j, k) in [(1, 1, 1, 1), (2, 1, 1, 1), (1, 2, 1, 1), (3, 4, 2, 3), (case.nv, case.nx, case.ny, case.nz)]:
        off = (l - 1) + case.nv * ((i - 1) + case.nx * ((j - 1) + case.ny * (k - 1)))
        assert vals[off] == w[l - 1, k + ng - 1, j + ng - 1, i + ng - 1]
    os.rename(p, str(tmp_path / O.restart_serial_name(prefix="rst0")))
    back = O.read_restart_serial(str(tmp_path / O.restart_serial_name(prefix="rst0")), case)
    assert np.array_equal(back, case.interior(w))


def test_mpiio_restart_layout_and_round_trip(tmp_path):
    """write_field: nv consecutive blocks w(l,1:nx,1:ny,1:nz), i fastest."""
    case = _small_case()
    w = np.random.default_rng(2).standard_normal(case.w.shape)
    p = str(tmp_path / "rst.bin")
    O.write_restart_mpiio(p, case, w)
    vals = np.fromfile(p, dtype=np.float64)
    ng, ntot = case.ng, case.nx * case.ny * case.nz
    for (l, i, j, k) in [(1, 1, 1, 1), (1, 2, 1, 1), (2, 1, 1, 1), (case.nv, 3, 4, 2)]:
        off = (l - 1) * ntot + (i - 1) + case.nx * ((j - 1) + case.ny * (k - 1))
        assert vals[off] == w[l - 1, k + ng - 1, j + ng - 1, i + ng - 1]
    assert np.array_equal(O.read_restart_mpiio(p, case), case.interior(w))


def test_field_info_round_trip(tmp_path):
    st = O.RunState()
    st.time_from_last_rst = 1.25e-7
    st.istore = 4
    info = st.info(icyc=1234, time=2.3e-4)
    p = str(tmp_path / "field_info1.dat")
    O.write_field_info(p, info)
    text = open(p).read()
    assert text.startswith("[field_info]\nicyc0 = 1234\n")
    back = O.read_field_info(p)
    assert back["icyc0"] == 1234 and back["time0"] == 2.3e-4 and back["istore"] == 4
    assert back["time_from_last_rst"] == 1.25e-7
    assert back["time_from_last_slice_vtr"] == 0.0
