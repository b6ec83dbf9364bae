"""Host logic of the ensemble and serving workloads (no GPU): seeded draws, condition points
against the reference's own numbers, the arrival process and the latency report."""
import math

import numpy as np
import pytest

from athad_cond_b200.ensemble import (boiling_point, condition_params, draw_condition, draw_ensemble,
                                      resolve, saturation_pressure)
from athad_cond_b200.serving import GRIDS, Request, dt_phys_seconds, poisson_requests, report


def test_boiling_points_match_the_reference_dew_point():
    # SaturationH2O::dewPoint at 40, 60 and 100 bar (test/cond_column_selftest.cpp:73 gives 548.7)
    assert boiling_point(40000.0) == pytest.approx(523.5, abs=0.05)
    assert boiling_point(60000.0) == pytest.approx(548.7, abs=0.05)
    assert boiling_point(100000.0) == pytest.approx(584.2, abs=0.06)
    assert saturation_pressure(513.15) / 1000.0 == pytest.approx(33.470, rel=5e-3)


def test_resolve_matches_the_nominal_column():
    s = resolve(0.5578, 0.4109, 0.0313)      # cond_column_selftest.cpp:112-116
    assert s["M_mean"] * 1000 == pytest.approx(29.01, rel=1e-2)
    assert s["R_mix"] == pytest.approx(286.6, rel=1e-2)
    assert s["q_H2O"] == pytest.approx(0.3464, rel=2e-2)
    d = resolve(0.010, 0.920, 0.070)         # :135-139
    assert d["R_mix"] == pytest.approx(195.0, rel=1e-3)
    assert d["q_H2O"] == pytest.approx(0.00423, rel=2e-2)


def test_condition_points_are_consistent_and_below_boiling():
    rng = np.random.default_rng(3)
    for _ in range(50):
        c = draw_condition(rng)
        assert 40.0 <= c.p_surf_bar <= 100.0 and 503.0 <= c.T_sea <= 523.0
        assert c.T_sea <= boiling_point(c.p_surf_bar * 1000.0) - 0.5
        assert sum(c.x_dry) == pytest.approx(1.0) and sum(c.x_surf) == pytest.approx(1.0)
        assert 0.004 / 1.2 <= c.x_dry[0] <= 0.02 / 0.94
        # the densities anchor 1e-2 r_air R_mix T_sea gives back p_surf [hPa]
        assert 1e-2 * c.r_air * c.surf["R_mix"] * c.T_sea == pytest.approx(c.p_surf_bar * 1000.0)
        p = condition_params(c)
        assert p.c_0 == pytest.approx(c.surf["q_H2O"]) and p.p_0 == pytest.approx(c.p_surf_bar * 1000)


def test_ensemble_draw_is_seeded_with_odd_uneven_grids():
    a, b = draw_ensemble(64), draw_ensemble(64)
    assert [m.grid for m in a] == [m.grid for m in b]
    assert len({m.grid for m in a}) > 32
    for m in a:
        im, jm, km = m.grid
        assert 21 <= im <= 41 and 61 <= jm <= 181 and 121 <= km <= 361
        assert jm % 2 == 1 and km % 2 == 1


def test_arrivals_form_a_poisson_process():
    reqs = poisson_requests(rate=2.0, duration=600.0)
    assert reqs == poisson_requests(rate=2.0, duration=600.0) or \
        [r.arrival for r in reqs] == [r.arrival for r in poisson_requests(rate=2.0, duration=600.0)]
    assert 1080 <= len(reqs) <= 1320                       # 1200 expected
    gaps = np.diff([0.0] + [r.arrival for r in reqs])
    assert np.mean(gaps) == pytest.approx(0.5, rel=0.1)
    assert np.std(gaps) == pytest.approx(0.5, rel=0.15)    # exponential: std = mean
    assert {tuple(r.grid) for r in reqs} == set(GRIDS)
    assert min(r.steps for r in reqs) >= 200 and max(r.steps for r in reqs) <= 2000


def test_dt_phys_and_report():
    assert dt_phys_seconds(4e-5) == pytest.approx((math.exp(3.0) - 1.0) * 6287.5 * 4e-5 / 8.0)
    assert dt_phys_seconds(4e-5) == pytest.approx(0.60, abs=0.01)
    rng = np.random.default_rng(0)
    done = []
    for q in range(10):
        r = Request(q, float(q), (21, 91, 181), draw_condition(rng), 100 * (q + 1), q)
        r.admitted, r.finished = r.arrival, r.arrival + 1.0 + q
        done.append(r)
    rep = report(done, 30.0)
    assert rep["requests"] == 10
    lat = np.array([1.0 + q for q in range(10)])
    assert rep["latency_s"]["p50"] == pytest.approx(np.percentile(lat, 50))
    per_day = lat / (np.array([100 * (q + 1) for q in range(10)]) * dt_phys_seconds() / 86400.0)
    assert rep["latency_per_sim_day_s"]["p99"] == pytest.approx(np.percentile(per_day, 99))
    assert rep["gp_steps"] == pytest.approx(sum(21 * 91 * 181 * 100 * (q + 1) for q in range(10)))
