"""Serving loop: model runs of different grids, condition points and lengths, arriving over
time, advanced together on one GPU by continuous batching.

A request is one run: a grid, a condition point (ensemble.draw_condition) and a number of
model iterations.  The server keeps every admitted run's state resident on the device (one
mixed-precision GpuAtmosphere each) and advances all of them by one iteration per step
through one GpuBatch: each run's column physics at its own cadence, the RK4 stages of all
runs in one persistent launch per stage.  Between steps it
  * retires runs that have done their iterations (download of the requested fields, the
    context's memory freed),
  * admits waiting requests in arrival order while a slot is free and the run's device
    footprint (athad_footprint_bytes_params) fits in what is left of the HBM budget,
so requests that arrive while others are on the GPU join as slots and memory free up, and
their work overlaps on the device.  A run's result does not depend on what else is in the
batch: every run executes the same per-cell code on its own fields.

Latency per simulated day = wall latency / (iterations x dt_phys / 86400 s), with
dt_phys = dt * metricShellLength / u_0 (cAtmosphereModel.h:465-470, RHS_Atm_Turb.cpp:445):
0.60 s for the configuration's dt = 4e-5.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .context import GpuAtmosphere, GpuBatch
from .ensemble import Condition, condition_params, draw_condition, init_config

GRIDS = [(21, 91, 181), (41, 181, 361), (41, 91, 181)]


def dt_phys_seconds(dt: float = 4e-5, im: int = 41, L_atm: float = 6287.5, zeta: float = 3.0,
                    u_0: float = 8.0) -> float:
    """Physical length of one iteration: dt * metricShellLength() / u_0."""
    span = 1.0   # rad runs from 1 to 2 in steps of 1/(im-1)
    shell = (math.exp(zeta * span) - 1.0) * L_atm / span
    return dt * shell / u_0


@dataclass
class Request:
    rid: int
    arrival: float                  # seconds after the start of the loop
    grid: tuple
    cond: Condition
    steps: int
    seed: int
    admitted: float = -1.0
    finished: float = -1.0
    result: dict = field(default_factory=dict)

    @property
    def points(self) -> int:
        return self.grid[0] * self.grid[1] * self.grid[2]


def poisson_requests(rate: float = 2.0, duration: float = 600.0, seed: int = 20261203,
                     grids=GRIDS, steps=(200, 2000)) -> list:
    """Arrivals of a Poisson process of the given rate over [0, duration): exponential gaps;
    grid uniform over `grids`, condition point as the ensemble's, iterations uniform."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration:
            break
        grid = tuple(grids[int(rng.integers(0, len(grids)))])
        out.append(Request(len(out), t, grid, draw_condition(rng), int(rng.integers(steps[0], steps[1] + 1)),
                           seed + 7919 * (len(out) + 1)))
    return out


class _Run:
    def __init__(self, req: Request, ctx: GpuAtmosphere, footprint: int):
        self.req = req
        self.ctx = ctx
        self.footprint = footprint
        self.next_iter = 1


class Server:
    """Continuous batching of runs on the current CUDA device."""

    def __init__(self, hbm_budget_bytes: int | None = None, max_slots: int = 64, dt: float = 4e-5,
                 use_graph: bool = True, shape: int | None = None, keep_fields=("t",),
                 stream=None, graph_after: int = 0, rebuild_every: int = 1):
        """graph_after: iterations a batch runs without CUDA graphs before it captures them
        (a batch that changes members every few iterations would capture every cadence
        pattern anew each time).  rebuild_every: fewest iterations between two rebuilds of
        the batch; runs that finish in between are set inactive and leave, and waiting
        requests join, at the next rebuild."""
        import torch
        self.torch = torch
        self.lib = _abi.load_library()
        if hbm_budget_bytes is None:
            free, _total = torch.cuda.mem_get_info()
            hbm_budget_bytes = int(free * 0.85)
        self.budget = int(hbm_budget_bytes)
        self.max_slots = max_slots
        self.dt = dt
        self.use_graph = use_graph
        self.shape = shape
        self.keep_fields = tuple(keep_fields)
        self.stream = stream if stream is not None else torch.cuda.Stream()
        self.used = 0
        self.runs: list = []
        self.batch: GpuBatch | None = None
        self.iterations = 0
        self.rebuilds = 0
        self.graph_after = int(graph_after)
        self.rebuild_every = max(1, int(rebuild_every))
        self.since_rebuild = 0
        self.host_s = {"admit": 0.0, "retire": 0.0, "rebuild": 0.0, "iteration": 0.0}

    # ---- admission ----
    def footprint(self, req: Request) -> int:
        p = condition_params(req.cond)
        g = _abi.Grid(*req.grid)
        return int(self.lib.athad_footprint_bytes_params(ctypes.byref(g), ctypes.byref(p)))

    def _admit(self, req: Request, now: float) -> bool:
        if len(self.runs) >= self.max_slots:
            return False
        fp = self.footprint(req)
        if self.used + fp > self.budget:
            return False
        ctx = GpuAtmosphere(*req.grid, condition_params(req.cond))
        ctx.set_stream(self.stream.cuda_stream)
        ctx.initial_state(init_config(req.cond))   # the reference's deterministic initial state
        self.used += fp
        req.admitted = now
        self.runs.append(_Run(req, ctx, fp))
        return True

    def _retire(self, run: _Run, now: float):
        if not run.req.result:
            run.req.result = {n: run.ctx.download(n) for n in self.keep_fields}
        run.req.finished = now
        run.ctx.close()
        self.used -= run.footprint
        self.runs.remove(run)

    def _rebuild(self):
        self.since_rebuild = 0
        if self.batch is not None:
            self.batch.close()
            self.batch = None
        if not self.runs:
            return
        self.batch = GpuBatch([r.ctx for r in self.runs], dt=self.dt,
                              first_iter=[r.next_iter for r in self.runs])
        self.batch.set_stream(self.stream.cuda_stream)
        if self.shape is not None:
            self.batch.set_shape(self.shape)
        self.rebuilds += 1

    # ---- the loop ----
    def run(self, requests: list, clock=None) -> dict:
        """Serve `requests` (sorted by arrival); returns the report.  `clock` returns the
        loop's time in seconds (default: wall time since the call)."""
        t0 = time.perf_counter()
        now_fn = clock or (lambda: time.perf_counter() - t0)
        pending = sorted(requests, key=lambda r: r.arrival)
        waiting: list = []
        pi = 0
        done = []
        leaving: list = []     # finished, inactive in the batch until the next rebuild
        clk = time.perf_counter
        while pi < len(pending) or waiting or self.runs:
            now = now_fn()
            while pi < len(pending) and pending[pi].arrival <= now:
                waiting.append(pending[pi])
                pi += 1
            active = len(self.runs) - len(leaving)
            may_rebuild = self.batch is None or active == 0 or self.since_rebuild >= self.rebuild_every
            changed = False
            if may_rebuild:
                if leaving:
                    t = clk()
                    if self.batch is not None:
                        self.batch.close()
                        self.batch = None
                    for r in leaving:
                        self._retire(r, r.req.finished)
                    leaving = []
                    changed = True
                    self.host_s["retire"] += clk() - t
                t = clk()
                while waiting and self._admit(waiting[0], now):
                    waiting.pop(0)
                    changed = True
                self.host_s["admit"] += clk() - t
            if not self.runs:
                if waiting:
                    raise RuntimeError(f"request {waiting[0].rid} does not fit the HBM budget alone")
                if pi < len(pending):   # idle until the next arrival
                    time.sleep(max(0.0, min(0.05, pending[pi].arrival - now)))
                continue
            if changed or self.batch is None:
                t = clk()
                self._rebuild()
                self.host_s["rebuild"] += clk() - t
            t = clk()
            self.batch.iteration(graph=self.use_graph and self.since_rebuild >= self.graph_after)
            self.host_s["iteration"] += clk() - t
            self.iterations += 1
            self.since_rebuild += 1
            for r in self.runs:
                if r not in leaving:
                    r.next_iter += 1
            finished = [r for r in self.runs if r not in leaving and r.next_iter > r.req.steps]
            if finished:
                t = clk()
                self.batch.synchronize()
                now = now_fn()
                for r in finished:
                    r.req.result = {n: r.ctx.download(n) for n in self.keep_fields}
                    r.req.finished = now
                    self.batch.set_active(self.runs.index(r), False)
                    leaving.append(r)
                    done.append(r.req)
                self.host_s["retire"] += clk() - t
        if self.batch is not None:
            self.batch.close()
            self.batch = None
        for r in leaving:
            self._retire(r, r.req.finished)
        rep = report(done, now_fn(), self.dt)
        rep["host_seconds"] = dict(self.host_s)
        return rep


def report(done: list, wall: float, dt: float = 4e-5) -> dict:
    """p50/p99 of latency per simulated day, aggregate grid-point steps per second."""
    if not done:
        return {"requests": 0}
    dtp = dt_phys_seconds(dt)
    lat = np.array([r.finished - r.arrival for r in done])
    per_day = np.array([(r.finished - r.arrival) / (r.steps * dtp / 86400.0) for r in done])
    work = float(sum(r.points * r.steps for r in done))
    first = min(r.arrival for r in done)
    last = max(r.finished for r in done)
    return {"requests": len(done), "gp_steps": work, "wall_s": last - first,
            "gp_steps_per_s": work / max(last - first, 1e-9),
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "latency_per_sim_day_s": {"p50": float(np.percentile(per_day, 50)),
                                      "p99": float(np.percentile(per_day, 99))},
            "dt_phys_s": dtp}
