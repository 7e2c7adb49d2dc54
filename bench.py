#!/usr/bin/env python
"""Benchmark of the multi-species reacting step (cell-steps/s).

Workload: 3-D periodic reacting decaying turbulence on 256^3 cells per GPU,
9-species H2/air (phi = 0.7, 1000 K, 1 atm), hybrid WENO5-Z / KEEP(2) fluxes with
the Ducros sensor, mixture-averaged transport, Strang-split ROK4 chemistry,
Wray RK3, CFL 0.5, FP64 throughout (the reference method).  One step is the
reference's integration-loop iteration: CFL reduction, advance_solution
(Rosenbrock half step, three RK substeps, Rosenbrock half step) and the final
compute_aux.

  python bench.py [--gpus N --steps K --warmup W]     # this implementation
  python bench.py --impl reference [...]              # the CPU reference arm

Multi-GPU (torchrun, one rank per GPU): every rank advances a 256^3 z slab of
a 256 x 256 x (256 N) periodic domain (weak scaling), exchanging its z ghost
layers with the neighbouring ranks over NCCL at every swap of the step (the
MPI half of the reference's bcswap); the CFL maxima are max-reduced over ranks
each step, as the reference's mpi_allreduce does.
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "prop-streams2_b200"))

METRIC = "cell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="stx", choices=["stx", "reference"])
    ap.add_argument("--n", type=int, default=256, help="cells per direction per GPU")
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--cpu-n", type=int, default=64, help="box edge of the CPU sample")
    ap.add_argument("--cpu-budget", type=float, default=60.0, help="most seconds of timed CPU work for the baseline")
    ap.add_argument("--e2e-steps", type=int, default=0, help="steps of the host-buffer leg (default: --steps)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--stiff-n", type=int, default=32, help="box edge of --workload stiff53 (32: the smallest sample that fills the GPU)")
    ap.add_argument("--workload", default="turbulence",
                    choices=["turbulence", "reactors", "flame", "serve", "stiff53", "tube"],
                    help="turbulence: the headline reacting-step benchmark; reactors: batched 0-D reactors; "
                         "flame: the 2000-cell 1-D premixed flame of the reference's published timing; "
                         "serve: a Poisson stream of mixed 0-D / 1-D / 2-D solves")
    ap.add_argument("--graph-steps", type=int, default=10, help="steps per captured graph (--workload flame, tube)")
    ap.add_argument("--form", default="batched", choices=["batched", "plain"],
                    help="batched: persistent work-stealing chemistry, staged sweeps with listed WENO faces, "
                         "autotuned; plain: the reference method's launch structure (a thread per cell for the "
                         "chemistry, a thread per face for the sweeps, no tuning) -- the same arithmetic")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="fp64: the reference method; mixed: FP32 face fluxes and transport, FP64 residual/chemistry")
    ap.add_argument("--requests", type=int, default=600, help="requests of the served mix (--workload serve)")
    ap.add_argument("--rate", type=float, default=10.0, help="Poisson arrival rate [1/s] (--workload serve)")
    ap.add_argument("--reactors", type=int, default=8192, help="reactors per GPU (--workload reactors)")
    ap.add_argument("--t-max", type=float, default=1e-2, help="longest integration of a reactor [s]")
    ap.add_argument("--max-steps", type=int, default=20000, help="ROK4 step cap per reactor")
    ap.add_argument("--ncu-raw", default=None,
                    help="an ncu --page raw --csv export of the dominant kernel class's launch(es) captured on this "
                         "box; its dram__bytes_read.sum + dram__bytes_write.sum per launch, scaled by cells to this "
                         "workload's launch, becomes roofline.traffic (null without it)")
    ap.add_argument("--ncu-cells", type=int, default=0, help="interior cells of the --ncu-raw capture's case")
    return ap.parse_args()


# kernel-name prefixes of the HBM-class kernel classes (for --ncu-raw)
KERNELS_OF_CLASS = {"euler": ("k_euler", "k_weno"), "visc": ("k_visc",), "eval_aux": ("k_eval_aux",),
                    "rk": ("k_update_field", "k_init_flux")}


def fp64_peaks(stream_ptr):
    """The device's FP64 FMA and FP64 tensor-core (DMMA, mma.sync m8n8k4 f64)
    throughput, measured by libstx_peaks.so (TFLOP/s), or None if it is not built."""
    import ctypes as C
    so = os.path.join(ROOT, "prop-streams2_b200", "csrc", "libstx_peaks.so")
    if not os.path.exists(so):
        return None
    lib = C.CDLL(so)
    lib.stx_peak_fp64.restype = C.c_int
    lib.stx_peak_fp64.argtypes = [C.c_int, C.c_void_p, C.POINTER(C.c_double)]
    out = {}
    for name, which in (("fma_tflops", 0), ("dmma_tflops", 1)):
        v = C.c_double()
        out[name] = round(v.value, 2) if lib.stx_peak_fp64(which, C.c_void_p(stream_ptr), C.byref(v)) == 0 else None
    out["how"] = ("persistent grid of 8 x 256-thread CTAs per SM: 8 chains of dependent DFMA per thread / 4 chains "
                  "of mma.sync.m8n8k4.f64 per warp; best of 3 timed launches")
    return out


def ncu_traffic(path, prefixes, cells_captured, cells_here):
    """DRAM bytes per launch of a kernel class from an ncu raw CSV export
    (ncu -i <rep> --page raw --csv): the mean over the captured launches of
    dram__bytes_read.sum + dram__bytes_write.sum, summed over the class's
    kernels, scaled by cells to this workload (traffic grows with the cells
    processed).  None without a capture."""
    if not path or not prefixes or cells_captured <= 0:
        return None
    import csv
    with open(path) as fh:
        rows = list(csv.reader(fh))
    head = rows[0]
    ik = head.index("Kernel Name")
    ir, iw = head.index("dram__bytes_read.sum"), head.index("dram__bytes_write.sum")
    units = rows[1]
    scale = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}
    per_kernel = {}
    for r in rows[2:]:
        if not any(r[ik].startswith(p) for p in prefixes):
            continue
        b = float(r[ir].replace(",", "")) * scale.get(units[ir], 1.0) + \
            float(r[iw].replace(",", "")) * scale.get(units[iw], 1.0)
        per_kernel.setdefault(r[ik].split("(")[0].split("<")[0], []).append(b)
    if not per_kernel:
        return None
    total = sum(sum(v) / len(v) for v in per_kernel.values())
    return total * cells_here / cells_captured


def config_dict(n, world, extra=None):
    d = {"workload": f"3-D periodic reacting decaying turbulence, {n}^3 cells per GPU, 9-species H2/air "
                     f"(21 reactions), phi=0.7, T=1000 K, p=1 atm, u_rms=0.3 c0, E(k)~k^4 exp(-2(k/4)^2); "
                     f"hybrid WENO5-Z/KEEP(2) + Ducros (threshold 0.1), mixture-averaged transport, "
                     f"Strang ROK4, Wray RK3, CFL 0.5",
         "cells_per_gpu": n ** 3, "species": 9, "reactions": 21, "precision_form": "plain FP64",
         "parallelism": (f"z-slab decomposition over {world} ranks of an {n}x{n}x{n * world} periodic domain, "
                         f"NCCL ghost exchange at every swap, global dt") if world > 1 else "1 GPU, periodic box",
         "l2": "inputs larger than L2 (about 15 GB of fields per GPU)"}
    if extra:
        d.update(extra)
    return d


# ------------------------------------------------------------------ clocks
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.fn = None

    def start(self):
        try:
            fd, self.fn = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.fn, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.fn) as fh:
            for line in fh:
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax.append(float(f[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.fn)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU (oracle) leg
def cpu_run(n, steps, seed, warm=1, budget_s=60.0, threads=None):
    """The CPU restatement (oracle) on an n^3 same-resolution sample of the workload,
    with the GPU run's step history: `warm` untimed steps, then `steps` timed steps
    (fewer if they take longer than budget_s): returns (cell-steps/s, cores, sample
    text)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    from stx import configs
    from driver import OracleSolver
    threads = threads or os.cpu_count() or 1
    c = configs.turbulence_case(n, alloc_fields=True)
    W, WA = configs.turbulence_fields(c, seed)
    c.w[...] = W
    c.w_aux[...] = WA
    o = OracleSolver(c, threads=threads)
    o.prepare()
    for _ in range(warm):
        o.step()
    t0 = time.perf_counter()
    k = 0
    while k < steps:
        o.step()
        k += 1
        el = time.perf_counter() - t0
        if el >= budget_s:
            break
    el = time.perf_counter() - t0
    o.close()
    rate = n ** 3 * k / el
    return rate, threads, (f"{n}^3 cells of the same workload (same grid spacing, seed and state statistics), "
                           f"{k} timed steps after {warm} warm-up steps (the GPU run's step history), {el:.1f} s")


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    oracle_so = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(oracle_so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    # W warm-up steps, then K timed steps of the CPU implementation on a bounded sample
    rate, cores, sample = cpu_run(args.cpu_n, args.steps, args.seed, warm=args.warmup, budget_s=90.0)
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": config_dict(args.n, args.gpus, {"reference_impl": "CPU restatement of the reference's FP64 "
                                                      "kernels (oracle/, OpenMP), not the reference binary: the "
                                                      "CUDA-Fortran reference cannot be compiled here"}),
            "cpu_baseline": {"value": rate, "unit": METRIC, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU leg
KNAMES = ["eval_aux", "ducros", "ghost", "euler", "visc", "rk", "chem", "dt"]


def mixed_error(dev, seed, n=48, steps=5):
    """Max relative error in T and Y_k (Y_k > 1e-8) of the mixed form against the
    FP64 form after `steps` reacting steps on an n^3 same-resolution sample."""
    import numpy as np
    import torch
    from stx import configs
    from stx.solver import Solver
    case = configs.turbulence_case(n)
    out = {}
    for form in ("fp64", "mixed"):
        W, WA = configs.turbulence_fields(case, seed, xp=torch, device=dev)
        s = Solver(case, device=str(dev), w=W, w_aux=WA)
        s.set_precision(form)
        s.prepare()
        for _ in range(steps):
            s.step()
        torch.cuda.synchronize()
        out[form] = (case.interior(s.w_aux[case.J("T")]).cpu().numpy(), case.interior(s.w_aux[:case.ns]).cpu().numpy())
        s.close()
    (T0, Y0), (T1, Y1) = out["fp64"], out["mixed"]
    big = Y0 > 1e-8
    return {"T_rel_max": float(np.max(np.abs(T1 - T0) / T0)),
            "Y_rel_max": float(np.max(np.abs(Y1 - Y0)[big] / Y0[big])),
            "sample": f"{n}^3 cells, {steps} steps, GPU FP64 form (= oracle to 1e-8) vs mixed form"}


def run_stx(args):
    import ctypes as C
    import numpy as np
    import torch
    import torch.distributed as dist
    from stx import configs
    from stx.native import check
    from stx.solver import Solver

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    n = args.n
    from stx import dist as D

    case = configs.turbulence_case(n)
    # One rank: a periodic n^3 box.  Several: z slabs of an n x n x (n * world)
    # periodic domain, the z ghosts exchanged with the neighbouring ranks over
    # NCCL at every swap of the step (stx_set_exchange); every slab starts from
    # the same seeded field, so the global field is the periodic continuation of
    # one box and the interfaces carry no jump.
    if world > 1:
        D.make_z_slab(case)
    W, WA = configs.turbulence_fields(case, args.seed, xp=torch, device=dev)
    sol = Solver(case, device=str(dev), w=W, w_aux=WA)
    del W, WA
    exch = D.ZSlabExchange(sol).install() if world > 1 else None
    lib = sol.lib
    if args.precision == "mixed":
        sol.set_precision("mixed")

    def compute_dt_global():
        out = (C.c_double * 9)()
        check(lib.stx_compute_dt(sol.ctx, sol.stream, C.c_void_p(sol.w_aux.data_ptr()), None, out), "compute_dt")
        sol.dt = D.global_dt(list(out), case.cfl, device=dev)
        return sol.dt

    def step():
        sol.icyc += 1
        sol.compute_aux(1, 0)
        compute_dt_global()
        sol.advance_solution()
        sol.compute_aux(1, 0)
        sol.time += sol.dt

    sol.update_ghost(1)
    sol.compute_aux(1, 1)
    check(lib.stx_bcextr_var(sol.ctx, sol.stream, sol.aux_slot(case.J("DIV"))), "bcextr")
    check(lib.stx_bcswap(sol.ctx, sol.stream, sol.aux_slot(case.J("DIV")), 1), "bcswap")
    check(lib.stx_bcswap(sol.ctx, sol.stream, sol.aux_slot(case.J("DUC")), 1), "bcswap")
    sol.fl.zero_()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # launch shapes chosen by the autotuner on the warmed-up fields (the Ducros
    # sensor marks faces by now), timed on this GPU; not part of the timed region
    tuning = None
    if args.form == "plain":
        sol.set_tuning({"sweep_kind": [1, 1, 1], "weno_list": [0, 0, 0], "chem_ctas_per_sm": -1})
        tuning = dict(sol.tuning(), form="plain")
    elif not args.no_autotune:
        compute_dt_global()
        tuning = sol.autotune(dt_chem=0.5 * sol.dt)
        torch.cuda.synchronize()

    # ---------------- timed region: device-resident fields
    from stx.native import StxKprof  # noqa: F401  (declared below if absent)
    check(lib.stx_profile_enable(sol.ctx, 1), "profile")
    clocks = Clocks(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    prof = (StxKprof * 8)()
    check(lib.stx_profile_read(sol.ctx, prof), "profile_read")
    check(lib.stx_profile_enable(sol.ctx, 0), "profile")
    ms_all = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(ms_all, op=dist.ReduceOp.MAX)
    ms_max = float(ms_all.item())
    value = (n ** 3) * world * args.steps / (ms_max / 1e3)
    launches = int(sum(p.launches for p in prof))
    status = sol.status()

    # ---------------- e2e: the same step through the C ABI with host buffers
    K2 = args.e2e_steps or args.steps
    host_w = torch.empty(sol.w.shape, dtype=torch.float64, pin_memory=True)
    host_w.copy_(sol.w)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    # Every step reads its input state from pinned host memory and returns its
    # result there.  The copies go in E2E_CHUNKS pieces on two streams: the read
    # back of a piece of one step's result runs beside the upload of the piece
    # before it for the next step, so the link carries both directions at once.
    main_s = torch.cuda.current_stream(dev)
    down_s, up_s = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    flat_d, flat_h = sol.w.view(-1), host_w.view(-1)
    nel = flat_d.numel()
    cuts = [nel * c // E2E_CHUNKS for c in range(E2E_CHUNKS + 1)]

    def round_trip(down, up):
        ev = torch.cuda.Event()
        ev.record(main_s)
        (down_s if down else up_s).wait_event(ev)
        for a, b in zip(cuts[:-1], cuts[1:]):
            if down:
                with torch.cuda.stream(down_s):
                    flat_h[a:b].copy_(flat_d[a:b], non_blocking=True)
                if up:
                    ev = torch.cuda.Event()
                    ev.record(down_s)
                    up_s.wait_event(ev)
            if up:
                with torch.cuda.stream(up_s):
                    flat_d[a:b].copy_(flat_h[a:b], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(up_s if up else down_s)
        main_s.wait_event(ev)

    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for k in range(K2):
        round_trip(down=k > 0, up=True)       # the previous step's result back, this step's input up
        step()
    round_trip(down=True, up=False)           # the last step's result back
    t1.record()
    torch.cuda.synchronize()
    ms2 = torch.tensor([t0.elapsed_time(t1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(ms2, op=dist.ReduceOp.MAX)
    e2e_value = (n ** 3) * world * K2 / (float(ms2.item()) / 1e3)
    wbytes = sol.w.numel() * 8

    # ---------------- roofline of the dominant HBM-bound kernel class
    cls = {KNAMES[k]: {"launches": int(prof[k].launches), "calls": int(prof[k].timed), "ms": prof[k].ms,
                       "bytes": prof[k].bytes} for k in range(8)}
    tot_ms = sum(v["ms"] for v in cls.values()) or 1.0
    for v in cls.values():
        v["share"] = v["ms"] / tot_ms
        v["gbs"] = (v["bytes"] / (v["ms"] / 1e3) / 1e9) if v["ms"] > 0 and v["bytes"] > 0 else None
    hbm_classes = [k for k in cls if k != "chem" and cls[k]["bytes"] > 0]
    dom = max(hbm_classes, key=lambda k: cls[k]["ms"])
    peaks_fn = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback 6.65 TB/s"
    if os.path.exists(peaks_fn):
        with open(peaks_fn) as fh:
            peak = float(json.load(fh)["hbm_gbs"])
        peak_src = "measured (MEASURED_PEAKS.json hbm_gbs)"
    # one "launch" of a class is one entry-point call: a fused sweep may run up
    # to three kernels (listed WENO faces: mark, list, staged tile)
    traffic = ncu_traffic(args.ncu_raw, KERNELS_OF_CLASS.get(dom, ()), args.ncu_cells, n ** 3)
    ach = cls[dom]["gbs"]
    roofline = {"bound": "hbm", "kernel_class": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak if ach else None, "traffic": traffic, "peak_source": peak_src,
                "calls": cls[dom]["calls"], "kernel_launches": cls[dom]["launches"],
                "bytes_per_launch": cls[dom]["bytes"] / max(1, cls[dom]["calls"]),
                "traffic_source": ("ncu capture " + os.path.basename(args.ncu_raw)) if traffic else
                "null: no ncu capture given (--ncu-raw)"}

    peaks64 = fp64_peaks(torch.cuda.current_stream().cuda_stream) if rank == 0 else None
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32/f64 mixed",
            "data": "synthetic (seeded)",
            "config": config_dict(n, world, {"dt_last": sol.dt, "tuning": tuning,
                                             "precision_form": "FP64 (the reference method)" if args.precision == "fp64"
                                             else "mixed: FP32 central/viscous face fluxes and transport properties, "
                                             "FP64 RK residual, Newton T(e), WENO faces and chemistry",
                                             "launch_form": "plain: a thread per cell (chemistry) and per face "
                                             "(sweeps), no tuning" if args.form == "plain" else
                                             "batched: persistent work-stealing chemistry, staged sweeps with "
                                             "listed WENO faces, autotuned"}),
            "roofline": roofline, "clocks": ck, "gpu_launches": launches,
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": wbytes, "d2h_bytes_per_step": wbytes,
                    "path": "stx_advance_solution et al. through the C ABI, state w copied from pinned host memory "
                            "before and back after every step, in %d pieces on two streams (the read back of one "
                            "step's result overlaps the upload of the next step's input)" % E2E_CHUNKS},
            "kernels": cls, "status_bits": status,
            "fp64_peaks": peaks64,
            "chem_bound": "FP64 arithmetic and the per-thread working set, not HBM: see fp64_peaks and the ncu "
                          "summary of k_rok4 (FP64-pipe utilisation) in profiles/"}
    if args.precision == "mixed" and rank == 0:
        line["error_vs_fp64"] = mixed_error(dev, args.seed)
    if world == 1 and rank == 0 and not args.no_cpu:
        rate, cores, sample = cpu_run(args.cpu_n, args.steps, args.seed, warm=args.warmup, budget_s=args.cpu_budget)
        line["cpu_baseline"] = {"value": rate, "unit": METRIC, "cores": cores, "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sol.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ batched 0-D reactors
R_METRIC = "reactor-solves/s"


def reactors_config(args, world):
    return {"workload": f"{args.reactors} adiabatic constant-pressure H2/air 0-D reactors per GPU (9 species, "
                        f"21 reactions), T0~U(900,1500) K, p~logU(1,40) atm, phi~U(0.3,3), ROK4, each integrated "
                        f"to min(2 t_ign, {args.t_max:g} s) with t_ign the first T > 1.05 T0, at most "
                        f"{args.max_steps} steps, one persistent launch, coldest reactors first",
            "reactors_per_gpu": args.reactors, "species": 9, "reactions": 21, "precision_form": "plain FP64",
            "parallelism": f"dp{world} (independent reactor sets)",
            "l2": "compute bound; inputs are a few hundred KB"}


def cpu_reactors(args, n_sample):
    """The oracle's constant-pressure reactors on a bounded sample (solves/s)."""
    import ctypes as C
    import numpy as np
    from stx import configs, native
    from stx import case as CS
    from stx import mech as M
    from stx.reactors import sample_h2air
    mech = configs.mechanism("h2air_9sp")
    tb = M.build_tables(mech, 101325.0, 200.0, 5500.0, 1.0)
    cfg = CS.default_ini(1, 1, 1, L=(1e-3,) * 3, Y=np.full(mech.ns, 1.0 / mech.ns), ns=mech.ns)
    case = CS.Case(cfg, tb, alloc_fields=False)
    oracle_so = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(oracle_so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    lib = native.load_oracle()
    par, tab, grid = case.params_struct(), case.tables_struct(), case.grid_struct()
    ctx = lib.ox_ctx_create(C.byref(par), C.byref(tab), C.byref(grid))
    cores = os.cpu_count() or 1
    lib.ox_set_threads(cores)
    T0, p0, Y0 = sample_h2air(n_sample, args.seed, mech)
    Y0 = np.ascontiguousarray(Y0)
    Y = np.empty_like(Y0); T = np.empty(n_sample); ti = np.empty(n_sample); te = np.empty(n_sample)
    ns = np.empty(n_sample, dtype=np.int32)
    vp = lambda a: C.c_void_p(a.ctypes.data)
    t0 = time.perf_counter()
    lib.ox_batch0d_cp(ctx, n_sample, vp(T0), vp(p0), vp(Y0), args.t_max, 1e-8, 1.05, 2.0, args.max_steps, vp(Y),
                      vp(T), vp(ti), vp(te), vp(ns))
    el = time.perf_counter() - t0
    lib.ox_ctx_destroy(ctx)
    solved = int((ns <= args.max_steps).sum())
    return solved / el, cores, (f"{n_sample} reactors of the same distribution (seed {args.seed}), {el:.1f} s; "
                                f"{solved} solved, {n_sample - solved} at the step cap (counted out, as on the GPU)")


def run_reactors(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    from stx.reactors import BatchReactors, sample_h2air

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    br = BatchReactors("h2air_9sp", device=str(dev))
    split = args.precision == "mixed"
    if split:
        br.set_form("split")
    T0, p0, Y0 = sample_h2air(args.reactors, args.seed + rank, br.mech)
    dT0, dp0, dY0 = (torch.as_tensor(a, dtype=torch.float64, device=dev).contiguous() for a in (T0, p0, Y0))

    def solve():
        return br.integrate(dT0, dp0, dY0, args.t_max, 1e-8, 1.05, 2.0, args.max_steps, sync=False,
                            order="coldest_first")

    for _ in range(args.warmup):
        out = solve()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        out = solve()
    e1.record()
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms_max = float(ms.item())
    value = args.reactors * world * args.steps / (ms_max / 1e3)
    nsteps = out["nsteps"].cpu().numpy()
    t_ign = out["t_ign"].cpu().numpy()
    status = br.status()

    # e2e: inputs from pinned host memory, all outputs back to pinned host memory, every step
    hT0, hp0, hY0 = (torch.as_tensor(a, dtype=torch.float64).contiguous().pin_memory() for a in (T0, p0, Y0))
    hout = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory() for k, v in out.items()}
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(args.steps):
        dT0.copy_(hT0, non_blocking=True); dp0.copy_(hp0, non_blocking=True); dY0.copy_(hY0, non_blocking=True)
        o = solve()
        for k in hout:
            hout[k].copy_(o[k], non_blocking=True)
    t1.record()
    torch.cuda.synchronize()
    ms2 = torch.tensor([t0.elapsed_time(t1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(ms2, op=dist.ReduceOp.MAX)
    e2e = args.reactors * world * args.steps / (float(ms2.item()) / 1e3)
    h2d = sum(t.numel() * t.element_size() for t in (hT0, hp0, hY0))
    d2h = sum(t.numel() * t.element_size() for t in hout.values())
    # a reactor is solved when it has run to 2 t_ign or to t_max; the others stop
    # at the step cap (the slow-induction states: T0 below ~1100 K at several atm,
    # where ROK4's steps stay small -- the oracle caps the same ones)
    capped = nsteps > args.max_steps
    done = int((~capped).sum())
    err = None
    if split:
        # the same reactors once more in the FP64 form: the split form's difference
        # over the reactors both forms solve
        o_sp = {k: v.clone() for k, v in out.items()}
        br.set_form("fp64")
        o_64 = solve()
        torch.cuda.synchronize()
        br.set_form("split")
        a, b = o_sp["nsteps"].cpu().numpy(), o_64["nsteps"].cpu().numpy()
        both = (a <= args.max_steps) & (b <= args.max_steps)
        Ts, T6 = o_sp["T"].cpu().numpy()[both], o_64["T"].cpu().numpy()[both]
        ts, t6 = o_sp["t_ign"].cpu().numpy()[both], o_64["t_ign"].cpu().numpy()[both]
        ig = (ts > 0) & (t6 > 0)
        Ys, Y6 = o_sp["Y"].cpu().numpy()[:, both], o_64["Y"].cpu().numpy()[:, both]
        big = Y6 > 1e-3
        err = {"reactors_compared": int(both.sum()),
               "T_final_rel_max": float(np.max(np.abs(Ts - T6) / T6)) if both.any() else None,
               "t_ign_rel_median": float(np.median(np.abs(ts[ig] - t6[ig]) / t6[ig])) if ig.any() else None,
               "t_ign_rel_max": float(np.max(np.abs(ts[ig] - t6[ig]) / t6[ig])) if ig.any() else None,
               "Y_gt_1e-3_rel_max": float(np.max(np.abs(Ys[big] - Y6[big]) / Y6[big])) if big.any() else None,
               "steps_ratio_mean": float(np.mean(a[both] / np.maximum(b[both], 1)))}
    line = {"metric": R_METRIC, "value": done * world * args.steps / (ms_max / 1e3), "unit": R_METRIC,
            "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "config": reactors_config(args, world),
            "value_note": "reactors that reached min(2 t_ign, t_max) per second; the launch also carried the capped "
                          "ones (reactors_launched_per_s)",
            "reactors_launched_per_s": value,
            "reactors": {"solved": done, "capped": int(capped.sum()), "per_launch": args.reactors},
            "reactor_steps_per_s": float(nsteps.sum()) * world * args.steps / (ms_max / 1e3),
            "steps_per_reactor": {"mean": float(nsteps.mean()), "max": int(nsteps.max()),
                                  "capped": int(capped.sum())},
            "ignited": int((t_ign > 0).sum()), "clocks": ck, "gpu_launches": args.steps,
            "e2e": {"value": e2e, "unit": R_METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "path": "BatchReactors.integrate -> stx_batch0d_integrate, inputs from and outputs to pinned "
                            "host memory every step"},
            "status_bits": status}
    line["config"]["precision_form"] = ("FP32/FP64 split (ROK4 Krylov basis and stage vectors in FP32; state, "
                                        "right-hand sides and error control in FP64)") if split else "plain FP64"
    if split:
        line["dtype"] = "f32/f64 split"
        line["error_vs_fp64"] = err
    if world == 1 and rank == 0 and not args.no_cpu:
        rate, cores, sample = cpu_reactors(args, 64)
        line["cpu_baseline"] = {"value": rate, "unit": R_METRIC, "cores": cores, "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    br.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ 1-D premixed flame
# The reference's one published timing (examples/laminar_premix_flame/data.dat:132):
# 7.0269314 ms per RK step for 2000 cells on one A100 (sm_80), i.e. 2.846e5 cell-steps/s.
FLAME_PUBLISHED = 2000.0 / 7.0269314e-3


def flame_config(world, graph_steps):
    return {"workload": "1-D laminar premixed H2/air flame, 2000 cells over 0.03 m, 11 species / 21 reactions: "
                        "examples/laminar_premix_flame as the reference runs it (its multideal.ini: inflow xmin, "
                        "extrapolation xmax, WENO5-Z on every face + KEEP(2), simpler splitting, ROK4, Wray RK3, "
                        "fixed dt 1e-8 s; its premix.dat initial profile)",
            "cells_per_gpu": 2000, "species": 11, "reactions": 21, "precision_form": "plain FP64",
            "parallelism": f"dp{world} (independent flames)",
            "launch": f"{graph_steps} steps per CUDA graph launch",
            "published_baseline": "7.0269314 ms/step on one A100 (data.dat:132) = 2.846e5 cell-steps/s",
            "l2": "fields (12 MB) fit in L2; latency bound"}


def cpu_flame(args, budget_s=20.0):
    """The oracle on the same flame, all host cores, for about budget_s seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    oracle_so = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(oracle_so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    from stx import configs
    from driver import OracleSolver
    cores = os.cpu_count() or 1
    o = OracleSolver(configs.premix_flame_case(), threads=cores)
    o.prepare()
    o.step()
    t0 = time.perf_counter()
    k = 0
    while True:
        o.step()
        k += 1
        el = time.perf_counter() - t0
        if el >= budget_s or k >= 2000:
            break
    o.close()
    return 2000 * k / el, cores, f"the same 2000-cell flame, {k} steps after 1 warm-up, {el:.1f} s"


def run_flame(args):
    import torch
    import torch.distributed as dist
    from stx import configs
    from stx.solver import Solver

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    case = configs.premix_flame_case()
    sol = Solver(case, device=str(dev))
    sol.prepare()
    G = max(1, args.graph_steps)
    K = max(G, (args.steps // G) * G)
    g = sol.capture(G)
    for _ in range(max(1, args.warmup // G + (args.warmup % G > 0))):
        sol.replay(g)
    torch.cuda.synchronize()
    check_lib = sol.lib
    check_lib.stx_profile_enable(sol.ctx, 0)
    clocks = Clocks(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(K // G):
        sol.replay(g)
    e1.record()
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms_max = float(ms.item())
    value = 2000 * world * K / (ms_max / 1e3)
    status = sol.status()
    # e2e: step by step through the C ABI, the state from pinned host memory before and back after every step
    host_w = torch.empty(sol.w.shape, dtype=torch.float64, pin_memory=True)
    host_w.copy_(sol.w)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    K2 = min(K, 200)
    t0.record()
    for _ in range(K2):
        sol.w.copy_(host_w, non_blocking=True)
        sol.step()
        host_w.copy_(sol.w, non_blocking=True)
    t1.record()
    torch.cuda.synchronize()
    ms2 = torch.tensor([t0.elapsed_time(t1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(ms2, op=dist.ReduceOp.MAX)
    e2e = 2000 * world * K2 / (float(ms2.item()) / 1e3)
    wbytes = sol.w.numel() * 8
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": K, "warmup": args.warmup,
            "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": value / (FLAME_PUBLISHED * world), "dtype": "f64",
            "data": "the reference's own input (examples/laminar_premix_flame/premix.dat)",
            "config": flame_config(world, G), "clocks": ck, "gpu_launches": K // G,
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": wbytes, "d2h_bytes_per_step": wbytes,
                    "path": "Solver.step (stx_compute_aux / stx_advance_solution through the C ABI, ~50 launches "
                            "per step, no graph), state w from pinned host memory before and back after every step"},
            "status_bits": status}
    if world == 1 and rank == 0 and not args.no_cpu:
        rate, cores, sample = cpu_flame(args)
        line["cpu_baseline"] = {"value": rate, "unit": METRIC, "cores": cores, "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sol.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ config 1: CFL-driven shock tube
TUBE_N = 2400


def tube_config(world, graph_steps):
    return {"workload": f"1-D reactive shock tube, {TUBE_N} cells over 0.12 m, 9 species / 18 reactions "
                        "(examples/reactive_shock_tube's mechanism and initial state, H2:O2:Ar = 2:1:7): reflecting "
                        "wall at x = 0, extrapolation at 0.12 m, WENO5-Z everywhere, Strang + ROK4, Wray RK3, "
                        "CFL 0.5 (dt recomputed every step), from t = 0",
            "cells_per_gpu": TUBE_N, "species": 9, "reactions": 18, "precision_form": "plain FP64",
            "parallelism": f"dp{world} (independent tubes)",
            "launch": f"{graph_steps} CFL-driven steps per CUDA graph launch (dt formed on the device)",
            "l2": "fields fit in L2; latency bound"}


def cpu_tube(budget_s=20.0):
    """The oracle on the same tube, all host cores, for about budget_s seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    oracle_so = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(oracle_so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
    from stx import configs
    from driver import OracleSolver
    cores = os.cpu_count() or 1
    o = OracleSolver(configs.config1_case(TUBE_N, cfl=0.5), threads=cores)
    o.prepare()
    o.step()
    t0 = time.perf_counter()
    k = 0
    while True:
        o.step()
        k += 1
        el = time.perf_counter() - t0
        if el >= budget_s or k >= 5000:
            break
    o.close()
    return TUBE_N * k / el, cores, f"the same {TUBE_N}-cell tube, {k} CFL-driven steps after 1 warm-up, {el:.1f} s"


def run_tube(args):
    import torch
    import torch.distributed as dist
    from stx import configs
    from stx.solver import Solver

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    G = max(1, args.graph_steps)
    K = max(G, (args.steps // G) * G)
    W = max(3, args.warmup)

    def timed(fn, n):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        return float(ms.item())

    # captured: G CFL-driven steps per graph launch (every replay reads the time back)
    sol = Solver(configs.config1_case(TUBE_N, cfl=0.5), device=str(dev))
    sol.prepare()
    for _ in range(W):
        sol.step()
    g = sol.capture(G)
    sol.replay(g)
    clocks = Clocks(local)
    clocks.start()
    ms_graph = timed(lambda: sol.replay(g), K // G)
    ck = clocks.stop()
    value = TUBE_N * world * K / (ms_graph / 1e3)
    t_end, status = sol.time, sol.status()
    # the host loop: the nine CFL maxima read back every step (Solver.step)
    ms_host = timed(sol.step, K)
    host = TUBE_N * world * K / (ms_host / 1e3)
    # e2e: graph replays with the state from pinned host memory before and back after every replay
    host_w = torch.empty(sol.w.shape, dtype=torch.float64, pin_memory=True)
    host_w.copy_(sol.w)

    def e2e_chunk():
        sol.w.copy_(host_w, non_blocking=True)
        sol.replay(g)
        host_w.copy_(sol.w, non_blocking=True)
    ms_e2e = timed(e2e_chunk, K // G)
    e2e = TUBE_N * world * K / (ms_e2e / 1e3)
    wbytes = sol.w.numel() * 8
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_graph / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "the reference example's initial state (synthetic grid of 2400 cells)",
            "config": tube_config(world, G), "clocks": ck, "gpu_launches": K // G,
            "host_loop": {"value": host, "ms_per_step": ms_host / K,
                          "path": "Solver.step: the CFL maxima read back to the host every step"},
            "sim_time_after_timed_steps_s": t_end,
            "e2e": {"value": e2e, "unit": METRIC, "h2d_bytes_per_step": wbytes / G, "d2h_bytes_per_step": wbytes / G,
                    "path": "graph replays through the C ABI, state w from pinned host memory before and back "
                            "after every replay of G steps"},
            "status_bits": status}
    if world == 1 and rank == 0 and not args.no_cpu:
        rate, cores, sample = cpu_tube()
        line["cpu_baseline"] = {"value": rate, "unit": METRIC, "cores": cores, "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sol.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ 53-species stiff mechanism
def stiff_config(n, world):
    return {"workload": f"synthetic stiff-mechanism box, {n}^3 cells per GPU: 53 species / 325 seeded reactions "
                        "(A~logU(1e8,1e16), b~U(-1.5,2), Ea~U(0,50) kcal/mol, 20% third-body), Y~Dirichlet(0.5), "
                        "T smooth in 1200..2000 K, 1 atm, at rest; WENO5-Z/KEEP(2) hybrid, Strang splitting with the "
                        "full-Jacobian Rosenbrock (dense 57x57 finite-difference Jacobian and LU per cell), fixed dt "
                        "1e-10 s",
            "cells_per_gpu": n ** 3, "species": 53, "reactions": 325, "precision_form": "plain FP64",
            "parallelism": f"dp{world} (independent boxes)",
            "size_note": f"{n}^3 stands in for the 128^3 case: at dt 1e-10 s every cell takes thousands of "
                         "adaptive sub-steps, each with 57 right-hand sides of 325 reactions, so a 128^3 step "
                         "runs for hours; the per-cell work does not depend on the box size, but "
                         f"{n ** 3} cells (one thread each) occupy a small part of the GPU, so this rate "
                         "understates what a full box sustains",
            "l2": "compute bound (per-cell Jacobian)"}


def cpu_stiff(budget_s=20.0):
    """The oracle on single cells of the same box (one thread per cell), about budget_s seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from stx import configs
    from driver import OracleSolver
    _, tb = configs.stiff_mechanism_tables(0)
    cores = os.cpu_count() or 1
    n = 1
    while True:                                   # grow the sample until it takes a few seconds
        case = configs.stiff_case(n, seed=3, tables=tb, dt=1e-10)
        o = OracleSolver(case, threads=cores)
        o.prepare()
        t0 = time.perf_counter()
        o.step()
        el = time.perf_counter() - t0
        o.close()
        if el >= budget_s / 4 or n >= 8 or 8 * el > budget_s:     # the next size costs 8x
            return n ** 3 / el, cores, f"{n}^3 cells of the same box (seed 3), one step, {el:.1f} s"
        n *= 2


def run_stiff(args):
    import torch
    import torch.distributed as dist
    from stx import configs
    from stx.solver import Solver

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    from stx.native import StxKprof, check
    n = args.stiff_n
    _, tb = configs.stiff_mechanism_tables(0)
    sol = Solver(configs.stiff_case(n, seed=3 + rank, tables=tb, dt=1e-10), device=str(dev))
    sol.prepare()
    for _ in range(args.warmup):
        sol.step()
    torch.cuda.synchronize()
    check(sol.lib.stx_profile_enable(sol.ctx, 0), "profile")      # zero the launch counters
    clocks = Clocks(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        sol.step()
    e1.record()
    torch.cuda.synchronize()
    ck = clocks.stop()
    prof = (StxKprof * 8)()
    check(sol.lib.stx_profile_read(sol.ctx, prof), "profile_read")
    launches = int(sum(p.launches for p in prof))
    ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms_max = float(ms.item())
    value = n ** 3 * world * args.steps / (ms_max / 1e3)
    # e2e: the state from pinned host memory before and back after every step
    host_w = torch.empty(sol.w.shape, dtype=torch.float64, pin_memory=True)
    host_w.copy_(sol.w)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(args.steps):
        sol.w.copy_(host_w, non_blocking=True)
        sol.step()
        host_w.copy_(sol.w, non_blocking=True)
    t1.record()
    torch.cuda.synchronize()
    ms2 = torch.tensor([t0.elapsed_time(t1)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(ms2, op=dist.ReduceOp.MAX)
    wbytes = sol.w.numel() * 8
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "config": stiff_config(n, world),
            "clocks": ck, "gpu_launches": launches,
            "e2e": {"value": n ** 3 * world * args.steps / (float(ms2.item()) / 1e3), "unit": METRIC,
                    "h2d_bytes_per_step": wbytes, "d2h_bytes_per_step": wbytes,
                    "path": "Solver.step through the C ABI, state w from pinned host memory before and back after "
                            "every step"},
            "status_bits": sol.status()}
    if world == 1 and rank == 0 and not args.no_cpu:
        rate, cores, sample = cpu_stiff()
        line["cpu_baseline"] = {"value": rate, "unit": METRIC, "cores": cores, "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sol.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ served mix
S_METRIC = "solves/s"


# pieces of the headline's end-to-end state copies (see its e2e loop)
E2E_CHUNKS = 16


# The served mix's stated p99 latency target at its stated rate (10 requests/s):
# a request's latency includes its own integration, and a cold 0-D reactor run
# to min(2 t_ign, 10 ms) takes up to the 20 000-step cap of ROK4 steps on its
# warp, seconds on its own; grid solves (flames, tubes) are held to 0.25 s
SERVE_P99_TARGET_S = 4.0
SERVE_GRID_P99_TARGET_S = 0.25


def run_serve(args):
    import torch
    from stx import configs
    from stx.serve import Server, mixed_requests

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    srv = Server(device=f"cuda:{local}", precision=args.precision)
    mech = configs.mechanism("h2air_9sp")
    warm = mixed_requests(max(3, args.warmup * 4), 1e9, args.seed + 97 + rank, mech)
    srv.run(warm, realtime=False)
    reqs = mixed_requests(args.requests, args.rate, args.seed + rank, mech)
    clocks = Clocks(local)
    clocks.start()
    stats = srv.run(reqs, realtime=True)
    ck = clocks.stop()
    srv.close()
    cfg = {"workload": f"served stream of {args.requests} requests per GPU, Poisson arrivals at {args.rate:g}/s: "
                       f"60% 0-D H2/air reactors (the batched-reactor distribution, to min(2 t_ign, 10 ms)), "
                       f"30% 1-D premixed flames (nx~U{{512..4096}}, phi~U(0.5,1.5), Tu~U(300,800) K, 20 steps "
                       f"at dt 1e-8 s), 10% 2-D reactive shock tubes 512x128 (10 steps at dt 2e-8 s); 9 species",
           "parallelism": f"replicas x{world}",
           "admission": f"HBM budget 16 GiB, {srv.max_grid} grid slots, {len(srv.lanes)} reactor lanes "
                        f"(reactors batched per launch, each launch capped at SMs/lanes CTAs)",
           "precision_form": "plain FP64" if args.precision == "fp64" else
                             "mixed (grid solves: FP32 face fluxes and transport; chemistry FP64)",
           "p99_target_s": SERVE_P99_TARGET_S, "grid_p99_target_s": SERVE_GRID_P99_TARGET_S,
           "l2": "mixed; latency-bound small solves"}
    line = {"metric": S_METRIC, "value": stats["solves_per_s"] * world, "unit": S_METRIC, "n_gpus": world,
            "steps": args.requests, "warmup": len(warm), "ms_per_step": 1e3 / stats["solves_per_s"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": cfg, "p50_s": stats["p50_s"], "p99_s": stats["p99_s"],
            "by_kind": {k: stats[k] for k in ("reactor", "flame1d", "tube2d") if k in stats},
            "p99_target_met": stats["p99_s"] <= SERVE_P99_TARGET_S,
            "grid_p99_target_met": all(stats[k]["p99_s"] <= SERVE_GRID_P99_TARGET_S
                                       for k in ("flame1d", "tube2d") if k in stats),
            "max_grid_in_flight": stats["max_grid_in_flight"], "clocks": ck,
            "host_calls": stats.get("host_calls"),
            "e2e": {"value": stats["solves_per_s"] * world, "unit": S_METRIC, "path": "host Request objects in, "
                    "host results out (every request's inputs are copied to and its results from the device)"}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.workload == "serve":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference serves one solve per process; "
                              "there is no served-mix counterpart to time"}), flush=True)
            return 0
        return run_serve(args)
    if args.workload == "flame":
        if args.impl == "reference":
            if int(os.environ.get("RANK", "0")) != 0:
                return 0
            rate, cores, sample = cpu_flame(args)
            print(json.dumps({"impl": "reference", "metric": METRIC, "value": rate, "unit": METRIC,
                              "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                              "higher_is_better": True, "scaling": "weak",
                              "vs_baseline": rate / FLAME_PUBLISHED, "dtype": "f64", "data": "synthetic (seeded)",
                              "config": flame_config(args.gpus, 1),
                              "cpu_baseline": {"value": rate, "unit": METRIC, "cores": cores, "kind": "port",
                                               "sample": sample},
                              "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
            return 0
        return run_flame(args)
    if args.workload == "tube":
        if args.impl == "reference":
            if int(os.environ.get("RANK", "0")) != 0:
                return 0
            rate, cores, sample = cpu_tube()
            print(json.dumps({"impl": "reference", "metric": METRIC, "value": rate, "unit": METRIC,
                              "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                              "data": "the reference example's initial state", "config": tube_config(args.gpus, 1),
                              "cpu_baseline": {"value": rate, "unit": METRIC, "cores": cores, "kind": "port",
                                               "sample": sample},
                              "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
            return 0
        return run_tube(args)
    if args.workload == "stiff53":
        if args.impl == "reference":
            if int(os.environ.get("RANK", "0")) != 0:
                return 0
            rate, cores, sample = cpu_stiff()
            print(json.dumps({"impl": "reference", "metric": METRIC, "value": rate, "unit": METRIC,
                              "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                              "data": "synthetic (seeded)", "config": stiff_config(args.stiff_n, args.gpus),
                              "cpu_baseline": {"value": rate, "unit": METRIC, "cores": cores, "kind": "port",
                                               "sample": sample},
                              "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
            return 0
        return run_stiff(args)
    if args.workload == "reactors":
        if args.impl == "reference":
            if int(os.environ.get("RANK", "0")) != 0:
                return 0
            rate, cores, sample = cpu_reactors(args, 64)
            print(json.dumps({"impl": "reference", "metric": R_METRIC, "value": rate, "unit": R_METRIC,
                              "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                              "data": "synthetic (seeded)", "config": reactors_config(args, args.gpus),
                              "cpu_baseline": {"value": rate, "unit": R_METRIC, "cores": cores, "kind": "port",
                                               "sample": sample},
                              "e2e": {"value": rate, "unit": R_METRIC, "h2d_bytes_per_step": 0,
                                      "d2h_bytes_per_step": 0}}), flush=True)
            return 0
        return run_reactors(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_stx(args)


if __name__ == "__main__":
    sys.exit(main())
