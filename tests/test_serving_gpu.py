"""The serving loop (athad_cond_b200.serving): continuous batching of runs on one GPU.

Requests with different grids, condition points and lengths arrive while others are on the
GPU; the server admits them by slot and HBM footprint and advances every resident run by
one iteration per step in one batch.  Checked: every result is bit-for-bit the result of
the same request served alone (the stated tolerance is exact equality: a run executes the
same per-cell code on its own fields whatever else is in the batch); admission never
exceeds the slot count or the HBM budget; latency and throughput are reported.
"""
import numpy as np
import pytest

from athad_cond_b200 import _abi
from athad_cond_b200.ensemble import draw_condition
from athad_cond_b200.serving import Request, Server

pytestmark = pytest.mark.gpu

SMALL = [(11, 21, 41), (13, 31, 61), (9, 25, 45)]
KEEP = ("t", "u", "c", "cloud", "p_stat")


def requests():
    rng = np.random.default_rng(5)
    out = []
    for q in range(6):
        out.append(Request(q, 0.02 * q, SMALL[q % 3], draw_condition(rng), 6 + 3 * q, 900 + q))
    return out


class TickClock:
    """Loop time that advances 0.01 s per batched iteration: admission order is then
    independent of how fast the machine is."""

    def __init__(self):
        self.server = None

    def __call__(self):
        return 0.01 * self.server.iterations


def serve(reqs, **kw):
    clk = TickClock()
    s = Server(keep_fields=KEEP, **kw)
    clk.server = s
    rep = s.run(reqs, clock=clk)
    return s, rep


@pytest.mark.parametrize("graph", [False, True])
def test_each_result_equals_the_request_served_alone(graph):
    mix = requests()
    s, rep = serve(mix, use_graph=graph, shape=0)
    assert rep["requests"] == len(mix)
    assert s.rebuilds > 1                       # membership changed while runs were resident
    overlap = sum(1 for a in mix for b in mix
                  if a.rid < b.rid and b.admitted < a.finished and a.admitted < b.finished)
    assert overlap > 0                          # runs shared the GPU
    for r in mix:
        alone = [Request(r.rid, 0.0, r.grid, r.cond, r.steps, r.seed)]
        serve(alone, use_graph=graph, shape=0)
        for n in KEEP:
            assert np.isfinite(r.result[n]).all(), (r.rid, n)
            assert np.array_equal(r.result[n], alone[0].result[n]), (r.rid, n)


def test_admission_respects_the_hbm_budget_and_slots():
    reqs = requests()
    probe = Server(keep_fields=KEEP)
    fps = [probe.footprint(r) for r in reqs]
    budget = sorted(fps)[-1] + sorted(fps)[-2]     # room for two runs at most
    clk = TickClock()
    s = Server(hbm_budget_bytes=budget, max_slots=3, keep_fields=KEEP, shape=0)
    clk.server = s
    peak = {"n": 0, "bytes": 0}
    orig = s._admit

    def admit(req, now):
        ok = orig(req, now)
        peak["n"] = max(peak["n"], len(s.runs))
        peak["bytes"] = max(peak["bytes"], s.used)
        return ok

    s._admit = admit
    rep = s.run(reqs, clock=clk)
    assert rep["requests"] == len(reqs)
    assert peak["n"] <= 2 and peak["bytes"] <= budget
    assert rep["latency_per_sim_day_s"]["p99"] >= rep["latency_per_sim_day_s"]["p50"] > 0
    assert s.used == 0


def test_footprint_matches_the_context_footprint():
    import ctypes
    lib = _abi.load_library()
    r = requests()[0]
    from athad_cond_b200.ensemble import condition_params
    p = condition_params(r.cond)
    g = _abi.Grid(*r.grid)
    assert Server(keep_fields=KEEP).footprint(r) == lib.athad_footprint_bytes_params(ctypes.byref(g), ctypes.byref(p))
