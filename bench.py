#!/usr/bin/env python
"""Benchmark of the ATHAD_COND model-iteration hot path on B200.

One step = one model iteration of cAtmosphereModel::run_3D_loop restricted to the hot path,
at the reference cadence (cAtmosphereModel.cpp:1156-1509): the RK4 step every iteration, one
pressure-Poisson sweep every 4th, saturation adjustment, moist convection and the column
densities every 2nd, and the time-level copy (storeIntermediateData3D) that closes it,
written by the last RK4 stage (athad_step_scalars.store_n_level: nothing runs in between).
Metric: grid-point RK4 steps per second = im*jm*km * steps / time.

Workload: the 41 x 181 x 361 grid, 1000 iterations, run twice from the reference's
deterministic initial state (cAtmosphereModel::RunTimeSlice: the integrated moist adiabat
over the symmetric parabolic sea-surface temperature, built on the device by
athad_initial_state): the plain FP64 form and the mixed-precision form
(athad_params.precision = MIXED: FP32 RK4 stencil arithmetic and stage storage, FP64 time
level and column physics).  The headline value is the mixed form; both forms' rates, their
RK4 rooflines, the mixed form's per-field error against the FP64 form after the same
iterations, the FP64 form's own one-ulp sensitivity over those iterations and a leg on the
reference's own 61 x 181 x 361 grid (the grid, state and cadence of the reference arm) are
in the line.  The inputs (about 40 fields of 21 MB) are far larger than the 126 MB L2, so
no flush is needed between steps.

--gpus N > 1 (under torchrun): independent replicas, one per GPU (the path has no
cross-replica exchange), weak scaling; value = all ranks' grid-point steps / max time.
--impl reference: the reference's CPU path timed on the host cores (see cpu_reference()).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GRID = (41, 181, 361)
CHECKPOINT = 20                # the reference's output cadence (cli/config_cond.xml: checkpoint)
NATIVE_GRID = (61, 181, 361)   # the reference's compiled-in grid (cAtmosphereModel.h:162)
# fields the reference's off-path modules (boundary conditions, filters, turbulence, ice
# scheme, radiation) write between hot-path calls, uploaded every step by the hybrid drop-in;
# E2E_DOWN: the fields they read back afterwards, and the fields the end-to-end leg copies to
# the host at the output cadence.
E2E_UP = ["t", "u", "v", "w", "c", "cloud", "ice", "gr", "co2", "tke", "dis", "nue",
          "S_c", "S_r", "S_i", "S_s", "S_g", "S_v", "t_eq"]
E2E_DOWN = ["t", "u", "v", "w", "c", "cloud", "ice", "gr", "co2", "tke", "dis", "p_dyn"]
# algorithmic bytes moved per grid point by one RK4 step with the time-level copy fused into
# stage 4.  FP64 form: 273 fields of 8 B (level mean 1 read; stage 1: 37 reads + 22 writes;
# stages 2-3: 48 + 22; stage 4: 48 + 14 + the 11 time-level writes).  Mixed form: level mean
# 8 B, stage 1 296 B read + 176 B written, stages 2-3 176 + 88 B, stage 4 220 + 200 B (the
# field lists of k_rk4m.cu) = 1428 B.
RK4_BYTES_PER_POINT = {0: 8 * (1 + 59 + 70 + 70 + 62 + 11), 1: 8 + 472 + 264 + 264 + 332 + 88}
# algorithmic bytes per grid point of one pressure call (PressureSolverAtm::run with one
# sweep): source 24 + 8, sweep 24, ceiling 8
PRESSURE_BYTES_PER_POINT = 64
# DRAM bytes (read + write) of one RK4 step (level mean and the four stage launches, the
# time-level copy fused) measured by ncu (one capture of each form's stage launches): per form, grid
RK4_TRAFFIC = {("fp64", (41, 181, 361)): 6.680e9, ("mixed", (41, 181, 361)): 3.880e9}
# fields compared between the two forms after the timed iterations: the 11 prognostics and
# the diagnosed pressure and densities
ERR_FIELDS = ["t", "u", "v", "w", "c", "cloud", "ice", "gr", "co2", "tke", "dis",
              "p_dyn", "p_stat", "r_humid"]


def iteration(g, it: int, dt: float):
    """One model iteration at the reference cadence."""
    if it % 4 == 0:
        g.PressureSolverAtm_run(total_iter_count=it)
    if it % 2 == 0:
        g.SaturationAdjustment_run()
        g.MoistConvection_run(it)
        g.densities()
    g.solveRungeKutta_Atmosphere_Turb(dt, 1.0, min(1.0, it / 300.0), store_n_level=True)


class ClockSampler:
    """SM clocks and clock-event reasons during the timed region.  NVML is polled every 5 ms
    from a thread, so that a region of a few tens of milliseconds has samples; nvidia-smi's
    200 ms loop is the fallback where NVML cannot be loaded.  Only reads the GPU's state."""
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
               ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.nv = None
        self.lines = []
        self.samples = []
        self.max_mhz = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.nv = (pynvml, h)
            self.stop = threading.Event()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return self
        except Exception:
            self.nv = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _poll(self):
        nv, h = self.nv
        while not self.stop.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                self.samples.append((sm, r))
            except Exception:
                pass
            self.stop.wait(0.005)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.nv:
            self.stop.set()
            self.t.join(timeout=2)
            try:
                self.nv[0].nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], self.max_mhz, set()
        for v, r in self.samples:
            sm.append(v)
            for n, bit in self.REASONS:
                if r & bit:
                    reasons.add(n)
        names = [n for n, _ in self.REASONS]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.samples else "nvidia-smi"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def max_over_ranks(x: float, device=None) -> float:
    """The largest of a per-rank time over all ranks of the process group (the value
    itself without one).  NCCL ranks pass their CUDA device; gloo ranks pass None."""
    import torch
    import torch.distributed as tdist
    if not (tdist.is_available() and tdist.is_initialized()) or tdist.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(points: int, steps: int, world: int, ms: float) -> float:
    """Grid-point steps per second of all replicas together: every rank advances its own
    copy of the grid by `steps` iterations; the job takes the slowest rank's time."""
    return points * steps * world / (ms * 1e-3)


def cpu_baseline(seconds_budget: float = 20.0):
    """The oracle (single-threaded C restatement of the reference path) on a bounded
    sample: whole model iterations of the same grid, from the same initial state (the
    oracle's own restatement of it, not timed), until the budget is used."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from athad_cond_b200._abi import config_init, config_params
    from oracle_binding import OracleState
    im, jm, km = GRID
    o = OracleState.initial(im, jm, km, config_params(), config_init(), compat=0)
    t0 = time.perf_counter()
    it = 0
    while True:
        it += 1
        if it % 4 == 0:
            o.pressure_sweep(1, it)
        if it % 2 == 0:
            o.saturation_adjust()
            o.moist_convection(it)
            o.densities()
        o.rk4(dt=4e-5, buoyancy_ramp=min(1.0, it / 300.0))
        o.store_n_level()
        el = time.perf_counter() - t0
        if el >= seconds_budget or it >= 8:
            break
    val = im * jm * km * it / el
    return {"value": val, "unit": "grid-point RK4 steps/s", "cores": 1, "kind": "port",
            "sample": f"{it} model iterations of {im}x{jm}x{km} through the C oracle "
                      f"(-O2, 1 thread), {el:.1f} s"}


def time_reference(max_iter: int = 4, budget_s: float | None = None):
    """The reference's own CPU implementation of the path, timed on this host's cores.

    The reference is built from its sources into oracle/_ref/stock with its own Makefile
    flags (-ffast-math, no -O level) and driven through its own functions: its initial
    state (not timed), then whole model iterations at its cadence (pressure sweep every
    4th, saturation adjustment + moist convection + densities every 2nd, RK4 and the
    time-level copy every iteration), with all host threads.  It supports only its
    compiled-in 61 x 181 x 361 grid, so the sample runs there; the metric is per grid point.
    A bounded sample of iterations (at least two, so one moist iteration is included) keeps
    the run within a few minutes.  Returns (value, threads, sample, kind, grid), or None
    without the built reference."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import ref_binding
    if not ref_binding.available("stock"):
        return None
    threads = len(os.sched_getaffinity(0))
    cwd = os.getcwd()
    os.chdir(os.environ.get("TMPDIR", "/tmp"))
    # the reference prints its progress with printf; keep stdout for the JSON line
    sys.stdout.flush()
    saved_fd = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        R = ref_binding.Reference("stock", threads=threads)
        t0 = time.perf_counter()
        R.init_state()
        t_init = time.perf_counter() - t0
        im, jm, km = R.shape
        it, el = 0, 0.0
        budget = float(os.environ.get("ATHAD_REF_BUDGET_S", "90")) if budget_s is None else budget_s
        t0 = time.perf_counter()
        while True:
            it += 1
            R.set_scalars(4e-5, 1.0, min(1.0, it / 300.0), it, it)
            if it % 4 == 0:
                R.lib.ref_pressure(R.h)
            if it % 2 == 0:
                R.lib.ref_satadj(R.h)
                R.lib.ref_moist(R.h, it)
                R.lib.ref_densities(R.h, 0)
            R.lib.ref_rk4(R.h)
            R.lib.ref_store(R.h)
            el = time.perf_counter() - t0
            if it >= 2 and (el >= budget or it >= max_iter):
                break
        R.close()
    finally:
        os.dup2(saved_fd, 1)
        os.close(saved_fd)
        os.close(devnull)
        os.chdir(cwd)
    sample = (f"{it} model iterations of the reference's own {im}x{jm}x{km} grid through its own "
              f"functions, built with its Makefile flags (-ffast-math, no -O), OMP_NUM_THREADS={threads}, "
              f"{el:.1f} s (initial state {t_init:.1f} s, not timed)")
    return im * jm * km * it / el, threads, sample, "reference", [im, jm, km]


def reference_arm(args):
    """The reference arm: the reference's own CPU path (time_reference); without the built
    reference it times the oracle instead."""
    metric = "grid-point RK4 steps/s (model iteration of the hot path, reference cadence)"
    r = time_reference()
    if r is None:
        b = cpu_baseline(seconds_budget=20.0)
        val, cores, sample, kind, grid = b["value"], 1, b["sample"], "port", list(GRID)
    else:
        val, cores, sample, kind, grid = r
    line = {"impl": "reference", "metric": metric, "value": val, "unit": "grid-point steps/s",
            "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "dtype": "f64", "data": "the reference initial state",
            "config": {"workload": f"plain FP64 model iteration, {grid[0]}x{grid[1]}x{grid[2]} grid", "grid": grid},
            "cpu_baseline": {"value": val, "unit": "grid-point steps/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": val, "unit": "grid-point steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


def run_form(args, rank, world, device, precision, grid=None, steps=None, perturb_t=False, e2e=True):
    """One form (FP64 or mixed) of the model iteration from the reference's initial state
    (built on the device by athad_initial_state): warm-up, the device-timed region of
    `steps` iterations, then the end-to-end leg through the C ABI with host buffers.
    perturb_t: t raised by one ulp everywhere after the initial state (the FP64 form's own
    sensitivity to rounding).  Returns the timings and the final fields of ERR_FIELDS."""
    import numpy as np
    import torch
    from athad_cond_b200 import GpuAtmosphere
    from athad_cond_b200._abi import StepScalars, config_params

    im, jm, km = grid or GRID
    steps = args.steps if steps is None else steps
    pts = im * jm * km
    p = config_params()
    p.precision = int(precision)
    g = GpuAtmosphere(im, jm, km, p)
    stream = torch.cuda.Stream(device=device)
    g.initial_state()
    if perturb_t:
        t = g.download("t")
        g.upload("t", np.nextafter(t, np.inf))
    g.set_stream(stream.cuda_stream)
    dt = 4e-5
    dist = world > 1
    if dist:
        import torch.distributed as tdist

    it = 0
    for _ in range(args.warmup):
        it += 1
        iteration(g, it, dt)
    g.synchronize()
    # ---- device-timed region ----
    if dist:
        tdist.barrier()
    torch.cuda.synchronize(device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    rk_ev, ps_ev, col_ev = [], [], []
    with ClockSampler(device.index if device.index is not None else 0) as clk:
        ev0.record(stream)
        for _ in range(steps):
            it += 1
            if it % 4 == 0:
                pa = torch.cuda.Event(enable_timing=True)
                pb = torch.cuda.Event(enable_timing=True)
                pa.record(stream)
                g.PressureSolverAtm_run(total_iter_count=it)
                pb.record(stream)
                ps_ev.append((pa, pb))
            if it % 2 == 0:
                ce = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
                ce[0].record(stream)
                g.SaturationAdjustment_run()
                ce[1].record(stream)
                g.MoistConvection_run(it)
                ce[2].record(stream)
                g.densities()
                ce[3].record(stream)
                col_ev.append(ce)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            g.solveRungeKutta_Atmosphere_Turb(dt, 1.0, min(1.0, it / 300.0), store_n_level=True)
            b.record(stream)
            rk_ev.append((a, b))
        ev1.record(stream)
        stream.synchronize()
    torch.cuda.synchronize(device)
    ms = ev0.elapsed_time(ev1)
    rk_ms = [a.elapsed_time(b) for a, b in rk_ev]
    ps_ms = [a.elapsed_time(b) for a, b in ps_ev]
    # per call of the column passes (every 2nd iteration): saturation adjustment, moist
    # convection, densities
    col_ms = [[ce[q].elapsed_time(ce[q + 1]) for q in range(3)] for ce in col_ev]
    if dist:
        tdist.barrier()
    ms = max_over_ranks(ms, device)
    final = {n: g.download(n) for n in ERR_FIELDS}
    fields_per_point = RK4_BYTES_PER_POINT[int(precision)]
    rk_avg = sum(rk_ms) / len(rk_ms)
    res = {"value": whole_job_value(pts, steps, world, ms), "ms_per_step": ms / steps,
           "rk4_ms": rk_avg, "achieved": fields_per_point * pts / (rk_avg * 1e-3) / 1e9,
           "rk4_bytes_per_point": fields_per_point, "clocks": clk.summary(), "final": final,
           "pressure_ms": (sum(ps_ms) / len(ps_ms)) if ps_ms else None,
           "column_ms": ({n: sum(c[q] for c in col_ms) / len(col_ms)
                          for q, n in enumerate(("saturation_adjust", "moist_convection", "densities"))}
                         if col_ms else None),
           "e2e_value": None, "h2d": 0, "d2h": 0, "finite": True}
    if args.no_e2e or not e2e:
        g.close()
        return res

    # ---- end to end through the C ABI, the state resident (the drop-in's resident mode) ----
    # Every step: the hot-path calls with their scalars from the host, then a device-to-host
    # read of the step's result, the level-mean temperature profile the RK4 step forms, into
    # one of two pinned buffers (athad_download_profile_async); the host reads each step's
    # profile one step later, once the copy is done, so it enqueues the next step while the
    # device works.  Every CHECKPOINT steps (the reference's output cadence) the output
    # fields are copied to pinned host memory on a side stream (athad_checkpoint_begin).  All
    # copies finish before the clock stops.
    lib = g.lib
    from athad_cond_b200._abi import FIELD, PROFILE
    D = ctypes.POINTER(ctypes.c_double)
    host_down = [torch.empty((im, jm, km), dtype=torch.float64).pin_memory() for _ in E2E_DOWN]
    ids = (ctypes.c_int32 * len(E2E_DOWN))(*[FIELD[n] for n in E2E_DOWN])
    hosts = (D * len(E2E_DOWN))(*[ctypes.cast(h.data_ptr(), D) for h in host_down])
    profs = [torch.empty(im, dtype=torch.float64).pin_memory() for _ in range(2)]
    prof_ps = [ctypes.cast(p.data_ptr(), D) for p in profs]
    prof_ev = [None, None]
    prof_ok = [True]

    def read_profile(b):
        prof_ev[b].synchronize()
        prof_ok[0] = prof_ok[0] and bool(np.isfinite(profs[b].numpy()).all())
        prof_ev[b] = None
    g._check(lib.athad_checkpoint_begin(g._h, ids, len(E2E_DOWN), hosts))   # allocates the snapshot
    g._check(lib.athad_checkpoint_wait(g._h))
    # ten output periods (200 steps, under half a second): the copy of the last checkpoint,
    # which no later step overlaps, is inside the timed region once, as in a run of any length
    e2e_steps = 10 * CHECKPOINT
    g.synchronize()
    if dist:
        tdist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for q in range(e2e_steps):
        it += 1
        iteration(g, it, dt)
        b = q % 2
        if prof_ev[b] is not None:
            read_profile(b)                      # step q-2's profile
        g._check(lib.athad_download_profile_async(g._h, PROFILE["t_ref_level"], prof_ps[b], im))
        prof_ev[b] = torch.cuda.Event()
        prof_ev[b].record(stream)
        if (q + 1) % CHECKPOINT == 0:
            g._check(lib.athad_checkpoint_begin(g._h, ids, len(E2E_DOWN), hosts))
    for b in (e2e_steps % 2, (e2e_steps + 1) % 2):   # the last two steps' profiles, in order
        if prof_ev[b] is not None:
            read_profile(b)
    g._check(lib.athad_checkpoint_wait(g._h))
    e1.record(stream)
    stream.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), device)
    res["finite"] = all(np.isfinite(h.numpy()).all() for h in host_down[:1] + host_down[-1:]) and \
        prof_ok[0]
    res.update({"e2e_value": whole_job_value(pts, e2e_steps, world, e2e_ms), "e2e_steps": e2e_steps,
                "h2d": ctypes.sizeof(StepScalars),
                "d2h": 8 * im + 8 * pts * len(E2E_DOWN) // CHECKPOINT})

    # ---- for comparison: the hybrid drop-in, the reference's other modules on the host ----
    # (the fields they write uploaded and the fields they read downloaded around every
    # hot-path iteration: what the adapter's per-call entry points cost over PCIe)
    host_up = {n: torch.from_numpy(g.download(n)).pin_memory() for n in E2E_UP}
    hyb_down = {n: torch.empty((im, jm, km), dtype=torch.float64).pin_memory() for n in E2E_DOWN}
    hyb_steps = 8
    g.synchronize()
    e0.record(stream)
    for _ in range(hyb_steps):
        it += 1
        for n in E2E_UP:
            h = host_up[n]
            lib.athad_upload(g._h, FIELD[n], ctypes.cast(h.data_ptr(), D), h.numel())
        iteration(g, it, dt)
        for n in E2E_DOWN:
            h = hyb_down[n]
            lib.athad_download(g._h, FIELD[n], ctypes.cast(h.data_ptr(), D), h.numel())
    e1.record(stream)
    stream.synchronize()
    hyb_ms = max_over_ranks(e0.elapsed_time(e1), device)
    g.close()
    res["e2e_hybrid"] = {"value": whole_job_value(pts, hyb_steps, world, hyb_ms),
                         "h2d_bytes_per_step": 8 * pts * len(E2E_UP), "d2h_bytes_per_step": 8 * pts * len(E2E_DOWN)}
    return res


def field_errors(a: dict, b: dict, beyond: float = 1e-5) -> dict:
    """Per field: max |a - b| / max |b| (b the FP64 form) and the fraction of cells where
    |a - b| / max |b| exceeds `beyond`."""
    import numpy as np
    out, frac = {}, {}
    for n in ERR_FIELDS:
        den = float(np.max(np.abs(b[n])))
        d = np.abs(a[n] - b[n])
        out[n] = float(np.max(d)) / den if den > 0 else float(np.max(np.abs(a[n])))
        frac[n] = float(np.count_nonzero(d > beyond * den)) / d.size if den > 0 else 0.0
    return out, frac


def _iteration_fp64(g, it: int, dt: float = 4e-5):
    iteration(g, it, dt)


def run_ensemble(args, device) -> dict:
    """Batched ensemble of seeded members with uneven grids and condition points
    (athad_cond_b200.ensemble.draw_ensemble): the mixed-precision batch, autotuned, one
    CUDA graph per iteration, against the same members advanced one after another in the
    plain FP64 form.  Every member starts from the reference's initial state for its grid and
    condition point, built on the device (athad_initial_state)."""
    import numpy as np
    import torch
    from athad_cond_b200 import GpuAtmosphere, GpuBatch
    from athad_cond_b200._abi import Precision
    from athad_cond_b200.ensemble import draw_ensemble, condition_params, init_config
    specs = draw_ensemble(args.members)
    pts = sum(s.grid[0] * s.grid[1] * s.grid[2] for s in specs)
    stream = torch.cuda.Stream(device=device)

    def build(prec):
        gs = []
        with torch.cuda.stream(stream):
            for s in specs:
                g = GpuAtmosphere(*s.grid, condition_params(s.cond, prec))
                g.set_stream(stream.cuda_stream)
                g.initial_state(init_config(s.cond))
                gs.append(g)
        stream.synchronize()
        return gs

    out = {"members": len(specs), "points": pts}
    gs = build(Precision.MIXED)
    b = GpuBatch(gs)
    b.set_stream(stream.cuda_stream)
    best, times = b.autotune(reps=3)
    for _ in range(args.warmup):
        b.iteration(graph=True)
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(device.index or 0) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            b.iteration(graph=True)
        e1.record(stream)
        stream.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    finite = all(bool(np.isfinite(g.download("t")).all()) for g in gs[:4])
    b.close()
    for g in gs:
        g.close()
    torch.cuda.empty_cache()
    out.update({"batched_mixed": {"ms_per_iteration": ms, "value": pts / (ms * 1e-3), "shape": best,
                                  "autotune_ms": times, "finite": finite}, "clocks": clk.summary()})
    gs = build(Precision.FP64)
    k64 = max(4, min(args.steps, 20))
    for it in range(1, 4):
        for g in gs:
            _iteration_fp64(g, it)
    stream.synchronize()
    e0.record(stream)
    for it in range(4, 4 + k64):
        for g in gs:
            _iteration_fp64(g, it)
    e1.record(stream)
    stream.synchronize()
    ms64 = e0.elapsed_time(e1) / k64
    for g in gs:
        g.close()
    torch.cuda.empty_cache()
    out["sequential_fp64"] = {"ms_per_iteration": ms64, "value": pts / (ms64 * 1e-3), "iterations": k64}
    out["batched_mixed_over_fp64"] = out["batched_mixed"]["value"] / out["sequential_fp64"]["value"]
    return out


def run_serving(args, device) -> dict:
    """Serving loop (athad_cond_b200.serving): Poisson arrivals, continuous batching,
    admission by HBM footprint; then a seeded sample of the served requests run again, each
    alone in the plain FP64 form for its full number of iterations from the same initial
    state (the 'each request alone in the FP64 form' baseline, measured)."""
    import numpy as np
    import torch
    from athad_cond_b200 import GpuAtmosphere
    from athad_cond_b200.ensemble import condition_params, init_config
    from athad_cond_b200.serving import Server, poisson_requests
    from athad_cond_b200._abi import Precision
    reqs = poisson_requests(rate=args.rate, duration=args.duration, steps=(args.min_steps, args.max_steps))
    srv = Server(max_slots=args.slots, graph_after=args.graph_after, rebuild_every=args.rebuild_every)
    rep = srv.run(reqs)
    done = [r for r in reqs if r.finished >= 0]
    rng = np.random.default_rng(20261203)
    sample = [done[q] for q in sorted(rng.choice(len(done), size=min(args.solo_sample, len(done)), replace=False))]
    stream = torch.cuda.Stream(device=device)
    solo = []
    for r in sample:
        g = GpuAtmosphere(*r.grid, condition_params(r.cond, Precision.FP64))
        g.initial_state(init_config(r.cond))
        g.set_stream(stream.cuda_stream)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for it in range(1, r.steps + 1):
            _iteration_fp64(g, it)
        e1.record(stream)
        stream.synchronize()
        solo.append({"grid": list(r.grid), "steps": r.steps, "seconds": e0.elapsed_time(e1) * 1e-3})
        g.close()
    work = sum(x["grid"][0] * x["grid"][1] * x["grid"][2] * x["steps"] for x in solo)
    secs = sum(x["seconds"] for x in solo)
    rep["fp64_alone"] = {"sample": len(solo), "gp_steps_per_s": work / secs if secs > 0 else None,
                         "runs": solo,
                         "measure": "a seeded sample of the served requests, each run alone in the plain FP64 "
                                    "form for its full iterations from the same initial state, device time"}
    if rep.get("gp_steps_per_s") and rep["fp64_alone"]["gp_steps_per_s"]:
        rep["served_over_fp64_alone"] = rep["gp_steps_per_s"] / rep["fp64_alone"]["gp_steps_per_s"]
    rep["offered"] = {"rate_per_s": args.rate, "duration_s": args.duration,
                      "steps": [args.min_steps, args.max_steps], "requests": len(reqs)}
    rep["batch_rebuilds"] = srv.rebuilds
    rep["batched_iterations"] = srv.iterations
    return rep


def run_poisson(args, device) -> dict:
    """Pressure-Poisson stress solve: a 61 x 361 x 721 grid, the source the divergence of
    a seeded mirror-symmetric Gaussian velocity perturbation of 0.5 m/s (u, w symmetric,
    v antisymmetric; torch's Philox generator, seed 20261203) on the nominal state (the
    reference's initial state for this grid), solved
    to a 1e-10 relative residual (athad_pressure_solve)."""
    import torch
    from athad_cond_b200 import GpuAtmosphere
    from athad_cond_b200._abi import config_params
    im, jm, km = args.poisson_grid
    stream = torch.cuda.Stream(device=device)
    g = GpuAtmosphere(im, jm, km, config_params())
    g.set_stream(stream.cuda_stream)
    gen = torch.Generator(device=device)
    gen.manual_seed(20261203)
    jh = (jm + 1) // 2
    g.initial_state()   # the nominal state: the reference's deterministic initial state
    with torch.cuda.stream(stream):
        amp = 0.5 / 8.0                                   # 0.5 m/s in units of u_0
        for n, anti in (("aux_u", False), ("aux_v", True), ("aux_w", False)):
            half = amp * torch.randn((im, jh, km), generator=gen, dtype=torch.float64, device=device)
            full = torch.empty((im, jm, km), dtype=torch.float64, device=device)
            full[:, :jh] = half
            full[:, jh:] = (-1.0 if anti else 1.0) * torch.flip(half[:, :jm - jh], dims=[1])
            if anti:
                full[:, jm // 2] = 0.0
            g.upload_tensor(n, full.contiguous())
        g.upload_tensor("p_dyn", torch.zeros((im, jm, km), dtype=torch.float64, device=device))
    stream.synchronize()
    reps = []
    with ClockSampler(device.index or 0) as clk:
        for _ in range(max(1, args.steps)):
            g.upload_tensor("p_dyn", torch.zeros((im, jm, km), dtype=torch.float64, device=device))
            g.synchronize()
            reps.append(g.pressure_solve(1e-10, 500))
    # the median solve (by time) is the reported one; the best and worst are kept beside it
    ordered = sorted(reps, key=lambda r: r["seconds"])
    med = ordered[len(ordered) // 2]
    pts = im * jm * km
    g.close()
    return {"grid": [im, jm, km], "points": pts, "iterations": med["iterations"],
            "converged": med["converged"], "rel_residual": med["rel_residual"],
            "seconds": med["seconds"], "best_seconds": ordered[0]["seconds"],
            "worst_seconds": ordered[-1]["seconds"], "all_seconds": [r["seconds"] for r in reps],
            "levels": med["levels"], "history": med["history"], "clocks": clk.summary()}


def run_loop(args, device) -> dict:
    """The whole model iteration on the device (athad_cond_b200.loop.ModelLoop): every module
    of the reference's run_3D_loop at its cadence, through the C ABI, on one mixed-precision
    (or FP64) context; the readbacks the reference prints (residuum, budgets, skin
    temperature) inside the timed region."""
    import torch
    from athad_cond_b200 import GpuAtmosphere
    from athad_cond_b200._abi import Precision, config_params
    from athad_cond_b200.loop import ModelLoop
    import numpy as np
    im, jm, km = tuple(int(x) for x in args.grid.lower().split("x")) if args.grid else GRID
    p = config_params()
    p.precision = int(Precision.MIXED if args.precision != "fp64" else Precision.FP64)
    g = GpuAtmosphere(im, jm, km, p)
    stream = torch.cuda.Stream(device=device)
    g.initial_state()
    g.set_stream(stream.cuda_stream)
    loop = ModelLoop(g)
    for _ in range(args.warmup):
        loop.iteration()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    last = None
    for _ in range(args.steps):
        last = loop.iteration()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    finite = all(bool(np.isfinite(g.download(n)).all()) for n in ("t", "u", "v", "w", "c", "p_dyn"))
    g.close()
    return {"grid": [im, jm, km], "ms_per_iteration": ms, "value": im * jm * km / (ms * 1e-3),
            "finite": finite, "residuum": last["residuum"]["residuum"], "t_skin": last["t_skin"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", default=None, help="IMxJMxKM (default: the 41x181x361 workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-envelope", action="store_true",
                    help="skip the FP64 one-ulp sensitivity run of the error report")
    ap.add_argument("--no-native-reference", action="store_true",
                    help="skip timing the reference itself beside the native-grid leg")
    ap.add_argument("--native-steps", type=int, default=100,
                    help="iterations of the leg on the reference's own 61x181x361 grid (0: skip)")
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "fp64"],
                    help="forms to run; the headline value is the mixed form when it runs")
    ap.add_argument("--workload", default="iteration", choices=["iteration", "ensemble", "serving", "poisson", "loop"],
                    help="iteration: the 41x181x361 model iteration (default); ensemble: the "
                         "batched ensemble; serving: the serving loop")
    ap.add_argument("--members", type=int, default=64, help="ensemble members")
    ap.add_argument("--rate", type=float, default=2.0, help="serving: arrivals per second")
    ap.add_argument("--duration", type=float, default=30.0, help="serving: seconds of arrivals")
    ap.add_argument("--min-steps", type=int, default=200, help="serving: fewest iterations of a run")
    ap.add_argument("--max-steps", type=int, default=2000, help="serving: most iterations of a run")
    ap.add_argument("--slots", type=int, default=64, help="serving: most resident runs")
    ap.add_argument("--graph-after", type=int, default=0,
                    help="serving: iterations a batch runs before it captures CUDA graphs")
    ap.add_argument("--rebuild-every", type=int, default=1,
                    help="serving: fewest iterations between two rebuilds of the batch")
    ap.add_argument("--solo-sample", type=int, default=8,
                    help="serving: requests re-run alone in the FP64 form for the baseline")
    ap.add_argument("--poisson-grid", default="61x361x721", help="poisson: IMxJMxKM")
    args = ap.parse_args()
    global GRID
    if args.grid:
        GRID = tuple(int(x) for x in args.grid.lower().split("x"))
    if args.warmup < 3:
        args.warmup = 3
    args.poisson_grid = tuple(int(x) for x in args.poisson_grid.lower().split("x"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    im, jm, km = GRID

    if args.impl == "reference":
        if rank != 0:
            return
        line = reference_arm(args)
        print(json.dumps(line))
        return

    import torch
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if args.workload != "iteration":
        if world > 1 and rank != 0:
            return
        fn = {"ensemble": run_ensemble, "serving": run_serving, "poisson": run_poisson,
              "loop": run_loop}[args.workload]
        r = fn(args, device)
        if args.workload == "poisson":
            line = {"metric": "pressure-Poisson solve to 1e-10 relative residual: seconds",
                    "value": r["seconds"], "unit": "s", "n_gpus": 1, "higher_is_better": False,
                    "dtype": "f64+f32", "data": "seeded perturbation on the reference initial state",
                    "config": {"workload": "61x361x721 stress solve, mirror-symmetric Gaussian "
                                           "velocity perturbation 0.5 m/s", "grid": r["grid"]},
                    "detail": r}
        elif args.workload == "loop":
            line = {"metric": "grid-point steps/s of the whole model iteration on the device",
                    "value": r["value"], "unit": "grid-point steps/s", "n_gpus": 1,
                    "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_iteration"],
                    "higher_is_better": True, "dtype": "f32+f64" if args.precision != "fp64" else "f64",
                    "data": "the reference's deterministic initial state, built on the device",
                    "config": {"workload": "run_3D_loop with every module on the device, "
                                           f"{r['grid'][0]}x{r['grid'][1]}x{r['grid'][2]} grid",
                               "grid": r["grid"]}, "detail": r}
        elif args.workload == "ensemble":
            line = {"metric": "ensemble grid-point steps/s (batched mixed-precision model iterations)",
                    "value": r["batched_mixed"]["value"], "unit": "grid-point steps/s", "n_gpus": 1,
                    "steps": args.steps, "warmup": args.warmup,
                    "ms_per_step": r["batched_mixed"]["ms_per_iteration"], "higher_is_better": True,
                    "dtype": "f32+f64", "data": "the reference initial state of each member, built on the device",
                    "config": {"workload": f"{r['members']} members, uneven grids, seeded condition points",
                               "points": r["points"]}, "detail": r}
        else:
            line = {"metric": "serving: grid-point steps/s and latency per simulated day",
                    "value": r.get("gp_steps_per_s"), "unit": "grid-point steps/s", "n_gpus": 1,
                    "higher_is_better": True, "dtype": "f32+f64", "data": "seeded arrivals, the reference initial state of each request",
                    "config": {"workload": "Poisson arrivals, continuous batching", **r.get("offered", {})},
                    "detail": r}
        print(json.dumps(line))
        return
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=device)
    from athad_cond_b200._abi import Precision
    forms = {"fp64": Precision.FP64, "mixed": Precision.MIXED}
    wanted = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    runs = {f: run_form(args, rank, world, device, forms[f]) for f in wanted}
    envelope = None
    if "fp64" in runs and "mixed" in runs and not args.no_envelope:
        # the FP64 form against itself with t one ulp higher: how far rounding alone moves
        # each field over the same iterations
        pert = run_form(args, rank, world, device, Precision.FP64, perturb_t=True, e2e=False)
        envelope = field_errors(pert["final"], runs["fp64"]["final"])
    native = None
    if args.native_steps > 0:
        # the reference's own grid, initial state and cadence (what the reference arm runs)
        native = {}
        for f in wanted:
            rr = run_form(args, rank, world, device, forms[f], grid=NATIVE_GRID, steps=args.native_steps)
            native[f] = {"value": rr["value"], "ms_per_step": rr["ms_per_step"], "rk4_ms": rr["rk4_ms"],
                         "e2e": rr["e2e_value"], "finite": rr["finite"]}
        native["grid"] = list(NATIVE_GRID)
        native["steps"] = args.native_steps
        if rank == 0 and world == 1 and not args.no_native_reference:
            # the reference itself on the same grid, state and cadence (four iterations, one
            # full cadence cycle, on all host cores): the like-for-like ratio of this leg
            r = time_reference(max_iter=4, budget_s=1.0e9)
            if r is not None:
                native["reference"] = {"value": r[0], "cores": r[1], "sample": r[2]}
                native["vs_reference_native"] = {
                    f"{f}_{k}": native[f][k] / r[0] for f in wanted for k in ("value", "e2e")
                    if native[f].get(k)}
    base = cpu_baseline() if (rank == 0 and world == 1 and not args.no_cpu_baseline) else None
    if world > 1:
        import torch.distributed as tdist
        tdist.barrier()
        tdist.destroy_process_group()
    if rank != 0:
        return
    head_name = "mixed" if "mixed" in runs else "fp64"
    r = runs[head_name]
    peak, peak_kind = measured_peaks()
    # kernel launches per step of our own kernels, averaged over the cadence cycle:
    # RK4 = level mean (row sums + combine) + 4 stages; pressure = source (with the aux
    # boundary) + 2 colours + boundaries + ceiling; saturation adjustment 1; moist convection
    # 1; densities 4 (columns, row sums, per-level mean density, its log-derivative)
    launches = args.steps * 6 + (args.steps // 4) * 5 + (args.steps // 2) * 6
    summary = {}
    for f, rr in runs.items():
        summary[f] = {"value": rr["value"], "ms_per_step": rr["ms_per_step"], "rk4_ms": rr["rk4_ms"],
                      "rk4_gbs": rr["achieved"], "rk4_roofline_frac": rr["achieved"] / peak,
                      "rk4_bytes_per_point": rr["rk4_bytes_per_point"], "e2e": rr["e2e_value"],
                      "e2e_hybrid": rr.get("e2e_hybrid"), "finite": rr["finite"]}
        if rr.get("pressure_ms"):
            # one pressure call: the source from aux_u/v/w (24 B read, 8 B written per point),
            # one red-black sweep (p and the source read, p written: 24 B) and the ceiling
            # pass (8 B read)
            pgbs = PRESSURE_BYTES_PER_POINT * im * jm * km / (rr["pressure_ms"] * 1e-3) / 1e9
            summary[f]["pressure_ms"] = rr["pressure_ms"]
            summary[f]["pressure_gbs"] = pgbs
            summary[f]["pressure_roofline_frac"] = pgbs / peak
        if rr.get("column_ms"):
            summary[f]["column_ms_per_call"] = rr["column_ms"]
    errors = None
    if "fp64" in runs and "mixed" in runs:
        err, frac = field_errors(runs["mixed"]["final"], runs["fp64"]["final"])
        errors = {"after_iterations": args.warmup + args.steps, "fields": err,
                  "fraction_of_cells_beyond_1e-5": frac, "measure": "max|mixed-fp64| / max|fp64|"}
        if envelope is not None:
            errors["fp64_one_ulp_envelope"] = {
                "fields": envelope[0], "fraction_of_cells_beyond_1e-5": envelope[1],
                "measure": "max|fp64(t + 1 ulp) - fp64| / max|fp64| after the same iterations"}
            errors["within_max_1e-5_envelope"] = {
                n: bool(err[n] <= max(1e-5, envelope[0][n])) for n in ERR_FIELDS}
        summary["mixed_over_fp64"] = runs["mixed"]["value"] / runs["fp64"]["value"]
    form_text = {"mixed": "mixed-precision (FP32 RK4 stencil arithmetic and stage storage, FP64 time "
                          "level, final combination and column physics)",
                 "fp64": "plain FP64"}[head_name]
    line = {
        "metric": "grid-point RK4 steps/s (model iteration of the hot path, reference cadence)",
        "value": r["value"], "unit": "grid-point steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if head_name == "mixed" else "f64",
        "data": "the reference's deterministic initial state (integrated moist adiabat, symmetric "
                "parabolic sea-surface temperature, prescribed circulation cells), built on the device",
        "config": {"workload": f"{form_text} model iteration, {im}x{jm}x{km} grid "
                               "(RK4 every step, pressure sweep every 4th, saturation adjustment, "
                               "moist convection and densities every 2nd)",
                   "grid": [im, jm, km], "points": im * jm * km,
                   "l2": "inputs larger than L2 (about 40 fields x 21 MB per step), no flush",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": r["e2e_value"], "unit": "grid-point steps/s",
                "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"]},
        "roofline": {"bound": "hbm", "achieved": r["achieved"], "peak": peak, "unit": "GB/s",
                     "frac": r["achieved"] / peak, "traffic": RK4_TRAFFIC.get((head_name, GRID)),
                     "kernel": f"{head_name} rk4 step (level mean + 4 stage launches, the "
                               "time-level copy fused into stage 4), "
                               f"{r['rk4_bytes_per_point']} algorithmic B per grid point",
                     "peak_source": peak_kind},
        "forms": summary,
        "error_vs_fp64": errors,
        "native_grid": native,
        "cpu_baseline": base,
        "gpu_launches": launches,
        "clocks": r["clocks"],
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
