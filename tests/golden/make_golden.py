"""Generate the golden fixtures in this folder from the reference's example data.

Run once in a checkout where the reference tree is available:

    python tests/golden/make_golden.py /path/to/Prop-STREAmS2

It writes small JSON files only (mechanism parameters parsed from the examples'
Cantera YAML inputs, the reference's own output trajectories subsampled, and
the constants printed in a reference run log).  Nothing under tests/ reads the
reference tree at test time.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "prop-streams2_b200"))

from stx import case as CS  # noqa: E402
from stx import mech as M  # noqa: E402


def dump(name, obj):
    with open(os.path.join(HERE, name), "w") as fh:
        json.dump(obj, fh, indent=1)
    print("wrote", name)


def ini_keys(cfg: CS.Config, keep):
    return {sec: {k: v for k, v in cfg.data.get(sec, {}).items()} for sec in keep}


def main(ref):
    ex = os.path.join(ref, "examples")
    # --- mechanisms
    shock = M.load_yaml_mechanism(os.path.join(ex, "reactive_shock_tube", "input_cantera.yaml"))
    dump("mech_shock_tube_9sp.json", M.mechanism_to_dict(shock))
    flame = M.load_yaml_mechanism(os.path.join(ex, "laminar_premix_flame", "input_cantera.yaml"))
    dump("mech_flame_11sp.json", M.mechanism_to_dict(flame))
    h2air = M.restrict_species(flame, ["H2", "H", "O2", "O", "OH", "HO2", "H2O2", "H2O", "N2"])
    dump("mech_h2air_9sp.json", M.mechanism_to_dict(h2air))
    kero = M.load_yaml_mechanism(os.path.join(ex, "batch_reactor", "input_cantera.yaml"))
    dump("mech_keromnes_14sp.json", M.mechanism_to_dict(kero))
    # --- batch reactor: the reference's own FP64 0-D output and Cantera's answer
    ref_out = np.loadtxt(os.path.join(ex, "syngas_mech_eval", "OUTPUT", "output_Keromnes2013.dat"))
    cantera = np.loadtxt(os.path.join(ex, "batch_reactor", "OUTPUT", "cantera_results.dat"))
    cfg = CS.Config.from_file(os.path.join(ex, "batch_reactor", "multideal.ini"))
    dump("batch_reactor_keromnes.json", {
        "source": "examples/syngas_mech_eval/OUTPUT/output_Keromnes2013.dat (reference FP64 GPU run of "
                  "examples/batch_reactor) and examples/batch_reactor/OUTPUT/cantera_results.dat",
        "ini": ini_keys(cfg, ["ref_state", "grid", "bc", "controls", "numerics", "flow", "fluid"]),
        "reference": ref_out.tolist(),
        "cantera": cantera.tolist(),
    })
    # --- shock tube and flame inputs (keys only)
    cfg = CS.Config.from_file(os.path.join(ex, "reactive_shock_tube", "multideal.ini"))
    dump("shock_tube_ini.json", ini_keys(cfg, ["ref_state", "grid", "bc", "controls", "numerics", "flow", "fluid"]))
    cfg = CS.Config.from_file(os.path.join(ex, "laminar_premix_flame", "multideal.ini"))
    flame_ini = ini_keys(cfg, ["ref_state", "grid", "bc", "controls", "numerics", "flow", "fluid"])
    # --- constants printed by the reference's flame run (examples/laminar_premix_flame/data.dat:10-29)
    pins = {"h298": [], "source": "examples/laminar_premix_flame/data.dat"}
    with open(os.path.join(ex, "laminar_premix_flame", "data.dat")) as fh:
        for line in fh:
            if "h(298.15)" in line:
                pins["h298"].append(float(line.split()[-1]))
            for key, name in (("Mixture gas constant", "rmixt0"), ("Mixture cp0", "cp0"), ("Mixture cv0", "cv0"),
                              ("Mixture Gamma", "gam"), ("Mixture density", "rho0"), ("Mixture viscosity", "mu0"),
                              ("Speed of sound", "c0")):
                if key in line:
                    pins[name] = float(line.split()[-1].replace("D", "E"))
    pins["ini"] = flame_ini
    dump("flame_log_pins.json", pins)
    # --- the flame's initial profile (examples/laminar_premix_flame/premix.dat: x, u, T, Y_1..Y_ns per
    #     cell, read by init_premix, multideal.F90:5534-5606), kept with the package's input data, and the
    #     run log's progress rows (data.dat:32-131: icyc, step time, dt, time, residual, rho/T/p min/max)
    pm = np.loadtxt(os.path.join(ex, "laminar_premix_flame", "premix.dat"))
    out = os.path.join(HERE, "..", "..", "prop-streams2_b200", "stx", "data", "premix_flame_11sp.npz")
    np.savez_compressed(out, x=pm[:, 0], u=pm[:, 1], T=pm[:, 2], Y=pm[:, 3:].T.copy())
    print("wrote", os.path.relpath(out, HERE))
    rows, lines = [], []
    with open(os.path.join(ex, "laminar_premix_flame", "data.dat")) as fh:
        for line in fh:
            f = line.split()
            if len(f) == 11 and f[0].isdigit():
                rows.append([int(f[0])] + [float(v) for v in f[1:]])
                lines.append(line.rstrip("\n"))
    dump("flame_progress.json", {
        "source": "examples/laminar_premix_flame/data.dat (reference FP64 GPU run from premix.dat, print_control "
                  "1000; columns of print_progress, multideal_gpu.F90:1933-1972)",
        "columns": ["icyc", "step_time", "dt", "time", "residual_rhou", "rhomin", "rhomax", "tmin", "tmax", "pmin",
                    "pmax"],
        "rows": rows, "lines": lines})
    # --- the digitised reference curves of Ferrer et al. that examples/reactive_shock_tube/OUTPUT/result_comp.py
    #     plots against output_1d_{170,190,230}micro_s.dat (x [m] and T [K], u [m/s], Y_H2)
    fer = {"source": "examples/reactive_shock_tube/OUTPUT/Ferrer_{Temp,U,YH2}_{170,190,230}micro_s.dat"}
    for q in ("Temp", "U", "YH2"):
        for t in (170, 190, 230):
            a = np.loadtxt(os.path.join(ex, "reactive_shock_tube", "OUTPUT", f"Ferrer_{q}_{t}micro_s.dat"))
            fer[f"{q}_{t}"] = a.tolist()
    dump("ferrer_shock_tube.json", fer)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference checkout>")
    main(sys.argv[1])
