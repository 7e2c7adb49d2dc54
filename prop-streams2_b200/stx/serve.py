"""A request loop that serves 0-D reactor, 1-D flame and 2-D shock-tube solves
on one GPU with continuous batching.

The reference runs one solve per process.  Here solves of different kinds and
sizes arrive over time and share the device:

* reactor requests (one adiabatic constant-pressure 0-D reactor each) are
  coalesced: whenever one of the reactor lanes (each a context with its own
  work counter and stream) is free, every reactor request that has arrived is
  launched in one persistent stx_batch0d_integrate launch on it, so requests
  that arrive while batches run start in the next free lane, concurrently
  with the running ones;
* grid requests (1-D flames, 2-D shock tubes; fixed dt, so no host
  synchronisation inside a step) each get their own solver context, fields in
  HBM and CUDA stream, and are admitted in arrival order while the memory
  budget and the slot count allow; the loop enqueues a few steps at a time on
  every active request's stream, so their kernels overlap on the device, and
  frees the slot as soon as a request has done its steps.

A request's result does not depend on what else runs: every kernel's result
per cell or reactor is independent of the launch's other work (the
work-stealing schedule only changes which thread does a cell), each grid solve
has its own context and counters, and fixed-dt steps involve no reduction.
Latency is completion minus arrival, measured on the host clock.
"""
from __future__ import annotations

import dataclasses
import time
from typing import Dict, List, Optional

import numpy as np
import torch

from . import configs
from . import mech as M
from .reactors import BatchReactors
from .solver import Solver


@dataclasses.dataclass
class Request:
    rid: int
    kind: str                      # "reactor" | "flame1d" | "tube2d"
    arrival: float                 # seconds after the start of the run
    params: dict
    steps: int = 0                 # grid solves: RK steps to take
    admitted: Optional[float] = None
    done: Optional[float] = None
    result: Optional[dict] = None

    @property
    def latency(self) -> Optional[float]:
        return None if self.done is None else self.done - self.arrival


class _GridJob:
    def __init__(self, req: Request, solver: Solver, stream: torch.cuda.Stream, nbytes: int):
        self.req, self.sol, self.stream, self.nbytes = req, solver, stream, nbytes
        self.steps_done = 0
        self.event: Optional[torch.cuda.Event] = None


class Server:
    """Continuous-batching server for one GPU.

    mem_budget: bytes of HBM the grid solves may hold at once; max_grid: most
    grid solves in flight; chunk: steps enqueued per grid solve per pass;
    reactor_batch: most reactors per batched launch."""

    def __init__(self, device: str = "cuda", mem_budget: int = 16 << 30, max_grid: int = 32, chunk: int = 5,
                 reactor_batch: int = 16384, t_max: float = 1e-2, max_steps: int = 20000, reactor_lanes: int = 4):
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        torch.cuda.set_device(self.device)
        rtab = M.build_tables(configs.mechanism("h2air_9sp"), 101325.0, 200.0, 5500.0, 1.0)
        self.lanes = [BatchReactors("h2air_9sp", device=str(self.device), tables=rtab) for _ in range(reactor_lanes)]
        self.lane_streams = [torch.cuda.Stream(self.device) for _ in range(reactor_lanes)]
        self.reactors = self.lanes[0]
        self.tables = {
            "flame1d": M.build_tables(configs.mechanism("h2air_9sp"), 101325.0, 200.0, 5500.0, 1.0),
            "tube2d": M.build_tables(configs.mechanism("shock_tube_9sp"), 7173.0, 200.0, 20000.0, 1.0),
        }
        self.mem_budget, self.max_grid, self.chunk = mem_budget, max_grid, chunk
        self.reactor_batch, self.t_max, self.max_steps = reactor_batch, t_max, max_steps

    # ------------------------------------------------------------------ grid solves
    def _case(self, req: Request):
        p = req.params
        if req.kind == "flame1d":
            return configs.flame_case(p["nx"], phi=p["phi"], Tu=p["Tu"], tables=self.tables["flame1d"],
                                      mech_name="h2air_9sp")
        if req.kind == "tube2d":
            return configs.tube_case(p["nx"], p["ny"], tables=self.tables["tube2d"])
        raise ValueError(req.kind)

    @staticmethod
    def grid_bytes(case) -> int:
        npg = case.nxg * case.nyg * case.nzg
        npi = case.nx * case.ny * case.nz
        return 8 * ((case.nv + case.nv_aux) * npg + 3 * case.nv * npi) + (8 << 20)

    def _admit_grid(self, req: Request, now: float) -> _GridJob:
        case = self._case(req)
        stream = torch.cuda.Stream(self.device)
        with torch.cuda.stream(stream):
            sol = Solver(case, device=str(self.device))
            sol.prepare()
        req.admitted = now
        return _GridJob(req, sol, stream, self.grid_bytes(case))

    def _advance(self, job: _GridJob):
        n = min(self.chunk, job.req.steps - job.steps_done)
        with torch.cuda.stream(job.stream):
            for _ in range(n):
                job.sol.step()
            job.event = torch.cuda.Event()
            job.event.record(job.stream)
        job.steps_done += n

    def _finish_grid(self, job: _GridJob, now: float):
        with torch.cuda.stream(job.stream):
            w = job.sol.w.cpu().numpy()
            T = job.sol.w_aux[job.sol.case.J("T")].cpu().numpy()
        job.req.result = {"w": w, "T": job.sol.case.interior(T), "status": job.sol.status()}
        job.req.done = now
        job.sol.close()

    # ------------------------------------------------------------------ reactors
    def _launch_reactors(self, lane: int, reqs: List[Request], now: float):
        T0 = np.array([r.params["T0"] for r in reqs])
        p0 = np.array([r.params["p0"] for r in reqs])
        Y0 = np.stack([r.params["Y0"] for r in reqs], axis=1)
        st = self.lane_streams[lane]
        with torch.cuda.stream(st):
            out = self.lanes[lane].integrate(T0, p0, Y0, self.t_max, 1e-8, 1.05, 2.0, self.max_steps, sync=False,
                                             order="coldest_first")
            ev = torch.cuda.Event()
            ev.record(st)
        for r in reqs:
            r.admitted = now
        return reqs, out, ev, st

    def _finish_reactors(self, batch, now: float):
        reqs, out, ev, st = batch
        ev.synchronize()
        with torch.cuda.stream(st):      # not the legacy default stream: it would wait for every lane
            host = {k: v.cpu().numpy() for k, v in out.items()}
        for i, r in enumerate(reqs):
            r.result = {"Y": host["Y"][:, i].copy(), "T": float(host["T"][i]), "t_ign": float(host["t_ign"][i]),
                        "t_end": float(host["t_end"][i]), "nsteps": int(host["nsteps"][i])}
            r.done = now

    # ------------------------------------------------------------------ the loop
    def run(self, requests: List[Request], realtime: bool = True, poll_s: float = 2e-4) -> Dict:
        """Serve the requests (arrival times relative to the start) and return
        throughput and latency statistics.  realtime=False admits every request
        at once (arrivals at 0)."""
        todo = sorted(requests, key=lambda r: r.arrival)
        if not realtime:
            for r in todo:
                r.arrival = 0.0
        pending_r: List[Request] = []
        pending_g: List[Request] = []
        active: List[_GridJob] = []
        batches = [None] * len(self.lanes)
        mem_used = 0
        nxt = 0
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0
        n_done = 0
        max_active = 0
        while n_done < len(todo):
            now = clock()
            while nxt < len(todo) and todo[nxt].arrival <= now:
                (pending_r if todo[nxt].kind == "reactor" else pending_g).append(todo[nxt])
                nxt += 1
            progressed = False
            # reactor lanes
            for ln in range(len(self.lanes)):
                if batches[ln] is not None and batches[ln][2].query():
                    self._finish_reactors(batches[ln], clock())
                    n_done += len(batches[ln][0])
                    batches[ln] = None
                    progressed = True
                if batches[ln] is None and pending_r:
                    take, pending_r = pending_r[:self.reactor_batch], pending_r[self.reactor_batch:]
                    batches[ln] = self._launch_reactors(ln, take, clock())
                    progressed = True
            # grid lanes
            still = []
            for job in active:
                if job.event is None or job.event.query():
                    if job.steps_done >= job.req.steps:
                        self._finish_grid(job, clock())
                        mem_used -= job.nbytes
                        n_done += 1
                        progressed = True
                        continue
                    self._advance(job)
                    progressed = True
                still.append(job)
            active = still
            while pending_g and len(active) < self.max_grid:
                est = self.grid_bytes(self._case_shape(pending_g[0]))
                if mem_used + est > self.mem_budget and active:
                    break
                req = pending_g.pop(0)
                job = self._admit_grid(req, clock())
                mem_used += job.nbytes
                self._advance(job)
                active.append(job)
                progressed = True
            max_active = max(max_active, len(active))
            if not progressed:
                time.sleep(poll_s)
        makespan = max(r.done for r in todo) - min(r.arrival for r in todo)
        lat = np.array([r.latency for r in todo])
        stats = {"requests": len(todo), "makespan_s": makespan, "solves_per_s": len(todo) / makespan,
                 "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                 "max_grid_in_flight": max_active}
        for kind in ("reactor", "flame1d", "tube2d"):
            lk = np.array([r.latency for r in todo if r.kind == kind])
            if lk.size:
                stats[kind] = {"n": int(lk.size), "p50_s": float(np.percentile(lk, 50)),
                               "p99_s": float(np.percentile(lk, 99))}
        return stats

    @dataclasses.dataclass
    class _Shape:
        nv: int
        nv_aux: int
        nxg: int
        nyg: int
        nzg: int
        nx: int
        ny: int
        nz: int

    def _case_shape(self, req: Request):
        """Field sizes of a grid request, without building its case."""
        p = req.params
        ng = 3
        if req.kind == "flame1d":
            ns, nx, ny = 9, p["nx"], 1
        else:
            ns, nx, ny = 9, p["nx"], p["ny"]
        nv, nv_aux = ns + 4, 2 * ns + 13 + 2 * (ns + 1)
        return self._Shape(nv, nv_aux, nx + 2 * ng, ny + 2 * ng, 1 + 2 * ng, nx, ny, 1)

    def close(self):
        for br in self.lanes:
            br.close()


def mixed_requests(n: int, rate: float, seed: int, mech: M.Mechanism, flame_steps: int = 20,
                   tube_steps: int = 10, frac=(0.6, 0.3, 0.1), flame_nx=(512, 4096), tube_shape=(512, 128)):
    """The served mix: Poisson arrivals at `rate` per second; 60 % 0-D reactors
    (the batched-reactor distribution), 30 % 1-D flames with nx ~ U{512..4096},
    phi ~ U(0.5, 1.5), Tu ~ U(300, 800) K, 10 % 2-D shock tubes of 512 x 128
    cells; seeded."""
    from .reactors import sample_h2air
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    kinds = rng.choice(3, size=n, p=np.asarray(frac) / np.sum(frac))
    T0, p0, Y0 = sample_h2air(n, seed + 1, mech)
    reqs = []
    for i in range(n):
        if kinds[i] == 0:
            reqs.append(Request(i, "reactor", float(t[i]), {"T0": float(T0[i]), "p0": float(p0[i]),
                                                           "Y0": Y0[:, i].copy()}))
        elif kinds[i] == 1:
            reqs.append(Request(i, "flame1d", float(t[i]),
                                {"nx": int(rng.integers(flame_nx[0], flame_nx[1] + 1)),
                                 "phi": float(rng.uniform(0.5, 1.5)), "Tu": float(rng.uniform(300.0, 800.0))},
                                steps=flame_steps))
        else:
            reqs.append(Request(i, "tube2d", float(t[i]), {"nx": tube_shape[0], "ny": tube_shape[1]},
                                steps=tube_steps))
    return reqs
