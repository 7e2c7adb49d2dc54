"""A request loop that serves 0-D reactor, 1-D flame and 2-D shock-tube solves
on one GPU with continuous batching.

The reference runs one solve per process.  Here solves of different kinds and
sizes arrive over time and share the device:

* reactor requests (one adiabatic constant-pressure 0-D reactor each) are
  coalesced: whenever one of the reactor lanes (each a context with its own
  work counter and stream) is free, every reactor request that has arrived is
  launched in one persistent stx_batch0d_integrate launch on it, so requests
  that arrive while batches run start in the next free lane, concurrently
  with the running ones.  A lane's inputs and outputs live in pinned host
  memory that the kernel reads and writes in place; the kernel publishes each
  reactor's step count last, behind a system-scope fence, so the loop
  completes every reactor as soon as it is done instead of when its batch
  ends;
* grid requests (1-D flames, 2-D shock tubes; fixed dt, so no host
  synchronisation inside a step) each get their own solver context, fields in
  HBM and CUDA stream, and are admitted in arrival order while the memory
  budget and the slot count allow; the loop enqueues a few steps at a time on
  every active request's stream, so their kernels overlap on the device, then
  enqueues the result's copies into pinned host buffers and frees the slot
  when they have landed.  Nothing in the loop waits on the device: it polls
  events (and, for reactors, the step counts in host memory).

A request's result does not depend on what else runs: every kernel's result
per cell or reactor is independent of the launch's other work (the
work-stealing schedule only changes which thread does a cell), each grid solve
has its own context and counters, and fixed-dt steps involve no reduction.
Latency is completion minus arrival, measured on the host clock.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import dataclasses
import os
import time
from typing import Dict, List, Optional

import numpy as np
import torch

# Two process-wide CUDA settings, applied if CUDA has not been initialised in
# this process yet:
#  * the server runs tens of streams; CUDA maps streams onto a few hardware
#    queues (CUDA_DEVICE_MAX_CONNECTIONS, 8 by default), and work queued behind
#    a long-running kernel in one stream then waits in every stream that shares
#    its queue: 32 queues;
#  * with lazy module loading (the default) a kernel's module loads at its first
#    launch or stream capture, in the middle of serving: all kernels load at
#    start instead.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
os.environ.setdefault("CUDA_MODULE_LOADING", "EAGER")

from . import configs
from . import mech as M
from .native import check
from .reactors import BatchReactors
from .requests import Request, mixed_requests  # noqa: F401  (mixed_requests: the served mix, re-exported)
from .solver import Solver


class _GridJob:
    def __init__(self, req: Request, solver: Solver, stream: torch.cuda.Stream, nbytes: int):
        self.req, self.sol, self.stream, self.nbytes = req, solver, stream, nbytes
        self.steps_done = 0
        self.event: Optional[torch.cuda.Event] = None
        self.host: Optional[dict] = None      # pinned result buffers while draining
        self.graph = None                     # captured chunk of steps
        self.staged: List[torch.Tensor] = []  # pinned pool buffers in use by the job


class _PinnedPool:
    """Pinned host buffers in power-of-two size classes, kept for reuse: served
    requests stage their fields through buffers taken from here, so the loop
    does not page-lock new host memory per request (flames of every size would
    each need new buffers); allocations happen only while the pool warms up."""

    def __init__(self):
        self.free: Dict[int, List[torch.Tensor]] = {}

    def take(self, numel: int) -> torch.Tensor:
        size = 1 << max(12, (int(numel) - 1).bit_length())
        lst = self.free.get(size)
        if lst:
            return lst.pop()
        return torch.empty(size, dtype=torch.float64, pin_memory=True)

    def give(self, buf: torch.Tensor):
        self.free.setdefault(buf.numel(), []).append(buf)

    def warm(self, max_numel: int, per_class: int):
        """Allocate per_class buffers of every size class up to max_numel."""
        size = 1 << 12
        while size <= max_numel:
            for _ in range(per_class):
                self.give(torch.empty(size, dtype=torch.float64, pin_memory=True))
            size <<= 1


class _ReactorLane:
    """A reactor lane: a context (its own work counter), a stream, and pinned
    host buffers of `cap` reactors that the kernel reads and writes in place."""

    def __init__(self, br: BatchReactors, stream: torch.cuda.Stream, cap: int):
        self.br, self.stream, self.cap = br, stream, cap
        ns = br.ns
        f64 = dict(dtype=torch.float64, pin_memory=True)
        self.T0, self.p0 = torch.empty(cap, **f64), torch.empty(cap, **f64)
        self.Y0, self.Y = torch.empty(ns * cap, **f64), torch.empty(ns * cap, **f64)
        self.T, self.t_ign, self.t_end = (torch.empty(cap, **f64) for _ in range(3))
        self.nsteps = torch.empty(cap, dtype=torch.int32, pin_memory=True)
        self.reqs: Optional[List[Request]] = None
        self.collected: Optional[np.ndarray] = None

    @property
    def busy(self) -> bool:
        return self.reqs is not None

    def launch(self, reqs: List[Request], t_max: float, max_steps: int):
        """Launch the requests' reactors, coldest first (the longest integrations
        start first)."""
        n, ns = len(reqs), self.br.ns
        T0 = np.array([r.params["T0"] for r in reqs])
        order = np.argsort(T0, kind="stable")
        reqs = [reqs[i] for i in order]
        self.T0.numpy()[:n] = T0[order]
        self.p0.numpy()[:n] = [r.params["p0"] for r in reqs]
        Y0 = self.Y0[:ns * n].view(ns, n)
        Y0.numpy()[:] = np.stack([r.params["Y0"] for r in reqs], axis=1)
        self.nsteps.numpy()[:n] = -1
        out = {"Y": self.Y[:ns * n].view(ns, n), "T": self.T[:n], "t_ign": self.t_ign[:n], "t_end": self.t_end[:n],
               "nsteps": self.nsteps[:n]}
        # No event behind the launch: an operation queued after a kernel that runs
        # for seconds would hold up the hardware queue it shares with other
        # streams.  The lane is free once every reactor has reported (the kernel
        # reads a reactor's inputs before it writes its step count, so the
        # buffers may then be refilled; the next launch follows in stream order).
        with torch.cuda.stream(self.stream):
            self.br.launch(self.T0[:n], self.p0[:n], Y0, out, t_max, 1e-8, 1.05, 2.0, max_steps)
        self.reqs = reqs
        self.collected = np.zeros(n, dtype=bool)

    def poll(self, now: float) -> int:
        """Complete the reactors whose results have arrived; free the lane when the
        launch has ended.  Returns the number completed."""
        n, ns = len(self.reqs), self.br.ns
        fresh = np.nonzero((self.nsteps.numpy()[:n] >= 0) & ~self.collected)[0]
        if fresh.size:
            Y = self.Y.numpy()[:ns * n].reshape(ns, n)
            T, ti, te, st = (a.numpy() for a in (self.T, self.t_ign, self.t_end, self.nsteps))
            for i in fresh:
                self.reqs[i].result = {"Y": Y[:, i].copy(), "T": float(T[i]), "t_ign": float(ti[i]),
                                       "t_end": float(te[i]), "nsteps": int(st[i])}
                self.reqs[i].done = now
            self.collected[fresh] = True
        if self.collected.all():
            self.reqs = None
        return int(fresh.size)


class Server:
    """Continuous-batching server for one GPU.

    mem_budget: bytes of HBM the grid solves may hold at once; max_grid: most
    grid solves in flight; chunk: steps enqueued per grid solve per pass
    (graphs: as one replay of a captured graph of chunk steps);
    reactor_batch: most reactors per batched launch (the default, 1024, stays
    within the reactors the warp-per-reactor kernel runs at once on a B200, so
    every served batch, like a request served alone, takes that kernel).
    precision: the grid solves' form, "fp64" (the reference method) or "mixed"
    (FP32 face fluxes and transport, stx_set_precision); the reactors' chemistry
    is FP64 in both."""

    # torch hands out the streams of a per-device pool of 32 in turn; the
    # lanes' and the grid solves' streams must all be distinct
    STREAM_POOL = 32

    def __init__(self, device: str = "cuda", mem_budget: int = 16 << 30, max_grid: int = 20, chunk: int = 5,
                 reactor_batch: int = 1024, t_max: float = 1e-2, max_steps: int = 20000, reactor_lanes: int = 12,
                 graphs: bool = True, precision: str = "fp64"):
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        torch.cuda.set_device(self.device)
        if reactor_lanes + max_grid > self.STREAM_POOL:
            raise ValueError(f"reactor_lanes + max_grid must be at most {self.STREAM_POOL}: torch's stream pool "
                             "would hand a grid solve the stream of a reactor lane")
        rtab = M.build_tables(configs.mechanism("h2air_9sp"), 101325.0, 200.0, 5500.0, 1.0)
        self.lanes = [_ReactorLane(BatchReactors("h2air_9sp", device=str(self.device), tables=rtab),
                                   torch.cuda.Stream(self.device), reactor_batch) for _ in range(reactor_lanes)]
        self.reactors = self.lanes[0].br
        # the grid solves' streams, created once: every stream created beyond
        # CUDA_DEVICE_MAX_CONNECTIONS shares a hardware queue with an earlier one,
        # and work queued behind a reactor lane's seconds-long launch in a shared
        # queue waits for it, so the loop creates no stream while it serves
        self._streams = [torch.cuda.Stream(self.device) for _ in range(max_grid)]
        conns = int(os.environ.get("CUDA_DEVICE_MAX_CONNECTIONS", "8"))
        self.stream_budget = {"reactor_lanes": reactor_lanes, "grid_streams": max_grid, "connections": conns}
        # the lanes' persistent kernels together hold at most one CTA per SM
        # (half the warp kernel's occupancy), so the grid solves' kernels keep
        # finding room on every SM
        nsm = torch.cuda.get_device_properties(self.device).multi_processor_count
        for lane in self.lanes:
            lane.br.set_launch_cap(max(2, nsm // reactor_lanes))
        self.tables = {
            "flame1d": M.build_tables(configs.mechanism("h2air_9sp"), 101325.0, 200.0, 5500.0, 1.0),
            "tube2d": M.build_tables(configs.mechanism("shock_tube_9sp"), 7173.0, 200.0, 20000.0, 1.0),
        }
        self.mem_budget, self.max_grid, self.chunk = mem_budget, max_grid, chunk
        self.reactor_batch, self.t_max, self.max_steps = reactor_batch, t_max, max_steps
        self._cases: Dict[tuple, object] = {}
        self.graphs = graphs
        self.pinned = _PinnedPool()
        self.pinned.warm(1 << 23, 4)          # up to 64 MB buffers (a 512 x 128 tube's w is 50 MB)
        # one small solver per grid kind holds that mechanism's device tables;
        # every request's context shares them (stx_ctx_create_like): admitting a
        # request uploads its fields and grid only
        self._bases = {
            "flame1d": Solver(configs.flame_case(64, tables=self.tables["flame1d"], mech_name="h2air_9sp"),
                              device=str(self.device)),
            "tube2d": Solver(configs.tube_case(16, 4, tables=self.tables["tube2d"]), device=str(self.device)),
        }
        # every request's context takes its base's precision form (stx_ctx_create_like_on)
        self.precision = precision
        for b in self._bases.values():
            b.set_precision(precision)
        # host time of every call site of the loop: name -> [calls, total s, max s]
        self.trace: Dict[str, list] = {}

    @contextlib.contextmanager
    def _timed(self, name: str):
        t = time.perf_counter()
        try:
            yield
        finally:
            d = time.perf_counter() - t
            e = self.trace.setdefault(name, [0, 0.0, 0.0])
            e[0] += 1
            e[1] += d
            e[2] = max(e[2], d)

    # ------------------------------------------------------------------ grid solves
    def _case(self, req: Request):
        """The request's case (host initial fields and parameters).  Cases are
        read-only once built, so requests with the same parameters share one
        (a small cache: the shock tubes of the mix are all alike)."""
        key = (req.kind, tuple(sorted(req.params.items())))
        case = self._cases.pop(key, None)
        if case is None:
            p = req.params
            if req.kind == "flame1d":
                case = configs.flame_case(p["nx"], phi=p["phi"], Tu=p["Tu"], tables=self.tables["flame1d"],
                                          mech_name="h2air_9sp")
            elif req.kind == "tube2d":
                case = configs.tube_case(p["nx"], p["ny"], tables=self.tables["tube2d"])
            else:
                raise ValueError(req.kind)
        self._cases[key] = case                      # most recently used last
        while len(self._cases) > 8:
            self._cases.pop(next(iter(self._cases)))
        return case

    @staticmethod
    def grid_bytes(case) -> int:
        npg = case.nxg * case.nyg * case.nzg
        npi = case.nx * case.ny * case.nz
        return 8 * ((case.nv + case.nv_aux) * npg + 3 * case.nv * npi) + (8 << 20)

    def _admit_grid(self, req: Request, now: float) -> _GridJob:
        with self._timed("admit.case"):
            case = self._case(req)
        stream = self._streams.pop()
        staged = []
        with torch.cuda.stream(stream):
            # the host fields go up through pinned pool buffers; a fresh case's
            # w_aux holds only the temperature guess (the rest starts at zero)
            def up(a):
                buf = self.pinned.take(a.size)
                staged.append(buf)
                v = buf[:a.size].view(a.shape)
                v.numpy()[...] = a
                return torch.empty(a.shape, dtype=torch.float64, device=self.device).copy_(v, non_blocking=True)
            with self._timed("admit.upload"):
                w = up(case.w)
                w_aux = torch.zeros(case.w_aux.shape, dtype=torch.float64, device=self.device)
                jT = case.J("T")
                w_aux[jT].copy_(up(case.w_aux[jT]))
            with self._timed("admit.context"):
                sol = Solver(case, device=str(self.device), w=w, w_aux=w_aux, tables_from=self._bases[req.kind],
                             stream_ordered=True)
            with self._timed("admit.prepare"):
                sol.prepare()
        req.admitted = now
        job = _GridJob(req, sol, stream, self.grid_bytes(case))
        job.staged = staged                  # released when the job ends (the copies are done by then)
        return job

    def _advance(self, job: _GridJob):
        """Enqueue the job's next chunk of steps: a replay of its captured graph of
        `chunk` steps (fixed dt: bit-identical to the steps one by one), or, for
        a shorter remainder, the steps one by one."""
        n = min(self.chunk, job.req.steps - job.steps_done)
        with torch.cuda.stream(job.stream):
            c = job.sol.case
            if self.graphs and n == self.chunk and c.cfl < 0 and c.iter_dt_recompute == 1:
                if job.graph is None:
                    with self._timed("advance.capture"):
                        job.graph = job.sol.capture(self.chunk)
                with self._timed("advance.replay"):
                    job.sol.replay(job.graph)
            else:
                with self._timed("advance.steps"):
                    for _ in range(n):
                        job.sol.step()
            with self._timed("advance.event"):
                job.event = torch.cuda.Event()
                job.event.record(job.stream)
        job.steps_done += n

    def _drain_grid(self, job: _GridJob):
        """Enqueue the result's copies into pinned host buffers (and the status
        word) on the job's stream; the loop completes the job when they land."""
        with self._timed("drain"):
            self._drain_grid_(job)

    def _drain_grid_(self, job: _GridJob):
        sol = job.sol
        bw, bt, bs = self.pinned.take(sol.w.numel()), self.pinned.take(sol.w_aux[0].numel()), self.pinned.take(1)
        job.staged += [bw, bt, bs]
        h = {"w": bw[:sol.w.numel()].view(sol.w.shape), "T": bt[:sol.w_aux[0].numel()].view(sol.w_aux.shape[1:]),
             "status": bs[:1].view(torch.int32)[:1]}
        h["status"].zero_()
        with torch.cuda.stream(job.stream):
            h["w"].copy_(sol.w, non_blocking=True)
            h["T"].copy_(sol.w_aux[sol.case.J("T")], non_blocking=True)
            check(sol.lib.stx_status_enqueue(sol.ctx, sol.stream, C.c_void_p(h["status"].data_ptr()), 1),
                  "stx_status_enqueue")
            job.event = torch.cuda.Event()
            job.event.record(job.stream)
        job.host = h

    def _finish_grid(self, job: _GridJob, now: float):
        with self._timed("finish"):
            self._finish_grid_(job, now)

    def _finish_grid_(self, job: _GridJob, now: float):
        h = job.host
        job.req.result = {"w": h["w"].numpy().copy(), "T": job.sol.case.interior(h["T"].numpy()).copy(),
                          "status": int(h["status"].numpy()[0]) & 0xffffffff}
        job.req.done = now
        job.sol.close()
        for b in job.staged:
            self.pinned.give(b)
        job.staged = []
        self._streams.append(job.stream)

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
            for lane in self.lanes:
                if lane.busy:
                    with self._timed("reactor.poll"):
                        k = lane.poll(clock())
                    n_done += k
                    progressed |= k > 0
                if not lane.busy and pending_r:
                    take, pending_r = pending_r[:self.reactor_batch], pending_r[self.reactor_batch:]
                    now = clock()
                    for r in take:
                        r.admitted = now
                    with self._timed("reactor.launch"):
                        lane.launch(take, self.t_max, self.max_steps)
                    progressed = True
            # grid lanes
            still = []
            for job in active:
                with self._timed("grid.query"):
                    ready = job.event is None or job.event.query()
                if ready:
                    if job.host is not None:             # results have landed
                        self._finish_grid(job, clock())
                        mem_used -= job.nbytes
                        n_done += 1
                        progressed = True
                        continue
                    if job.steps_done >= job.req.steps:
                        self._drain_grid(job)
                    else:
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
                 "max_grid_in_flight": max_active,
                 "host_calls": {k: {"calls": v[0], "total_s": round(v[1], 4), "max_ms": round(1e3 * v[2], 2)}
                                for k, v in sorted(self.trace.items())}}
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
        for lane in self.lanes:
            lane.br.close()
        for b in self._bases.values():
            b.close()
