"""The oracle against the reference's own known answers (its self-tests), plus the
properties of the restatement that need no reference: exact mirror symmetry of the
mirror-symmetric semantics and the size of the Jacobi-vs-in-place RK4 difference."""
import json
import os

import numpy as np
import pytest

from athad_cond_b200 import make_state, mirror
from athad_cond_b200._abi import config_params, Wall
from oracle_binding import OracleState, lib

KAT = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "thermo_kat.json")))


def rel(a, b):
    return abs(a - b) / abs(b)


def test_saturation_pressure_known_answers():
    L = lib()
    for c in KAT["saturation_pressure_hPa"]:
        assert rel(L.or_saturation_pressure(c["T"]), c["want"]) <= c["rel"], c
    for T in KAT["no_saturation_at"]:
        assert L.or_saturation_pressure(T) == -1.0
    for c in KAT["sublimation_pressure_hPa"]:
        assert rel(L.or_sublimation_pressure(c["T"]), c["want"]) <= c["rel"], c
    for c in KAT["latent_heat"]:
        assert rel(L.or_latent_heat(c["T"]), c["want"]) <= c["rel"], c
    assert L.or_latent_heat(647.096) == 0.0
    for c in KAT["saturation_mass_fraction"]:
        assert rel(L.or_saturation_mass_fraction(c["E"], c["p"], c["M_other"]), c["want"]) <= c["rel"]
    assert L.or_saturation_mass_fraction(2000.0, 1000.0, 0.034) == 1.0
    assert L.or_saturation_mass_fraction(-1.0, 1000.0, 0.034) == 1.0
    d = KAT["dew_point_boiling_60bar"]
    assert rel(L.or_dew_point(d["e"]), d["want"]) <= d["rel"]
    # monotone over the model's range (saturation_selftest.cpp:67-75)
    prev = -1.0
    for T in np.arange(150.0, 647.096, 0.5):
        p = L.or_saturation_pressure(T) if T >= 273.16 else L.or_sublimation_pressure(T)
        assert p > prev and np.isfinite(p)
        prev = p


def _resolve(x):
    import ctypes
    out = (ctypes.c_double * 7)()
    xs = (ctypes.c_double * 8)(*(list(x) + [0.0] * (8 - len(x))))
    lib().or_resolve(xs, out)
    return list(out)


def test_mixture_and_lapse_known_answers():
    L = lib()
    s = KAT["surface_mixture"]
    M_mean, R_mix, q_H2O, q_CO2, q_bg, M_bg, R_bg = _resolve(s["x"])
    assert rel(M_mean * 1000, s["M_mean_g"]) <= s["rel"][0]
    assert rel(R_mix, s["R_mix"]) <= s["rel"][1]
    assert rel(q_H2O, s["q_H2O"]) <= s["rel"][2]
    cp = L.or_cp_of(q_H2O, q_CO2, s["cp_T"], M_bg)
    assert rel(cp, s["cp"]) <= s["cp_rel"]
    M_nw = L.or_M_nonwater(q_H2O, q_CO2, M_bg)
    assert rel(M_nw * 1000, s["M_nonwater_g"]) <= s["M_nonwater_rel"]
    d = KAT["dry_mixture"]
    M_mean, R_mix_d, q_H2O_d, *_ = _resolve(d["x"])
    assert rel(M_mean * 1000, d["M_mean_g"]) <= d["rel"][0]
    assert rel(R_mix_d, d["R_mix"]) <= d["rel"][1]
    assert rel(q_H2O_d, d["q_H2O"]) <= d["rel"][2]
    lp = KAT["lapse"]
    g = lp["g"]
    assert rel(g / cp * 1000, lp["dry_K_per_km"]) <= lp["dry_rel"]
    gm = L.or_moist_lapse(513.15, 60000.0, M_nw, cp, R_mix, g)
    assert rel(gm * 1000, lp["moist_K_per_km"]) <= lp["moist_rel"]
    ge = L.or_moist_lapse(lp["earth_T"], lp["earth_p"], lp["earth_M"], lp["earth_cp"], lp["earth_R"], g)
    assert rel(ge * 1000, lp["earth_K_per_km"]) <= lp["earth_rel"]
    assert rel(L.or_moist_lapse(700.0, 60000.0, M_nw, cp, R_mix, g), g / cp) <= KAT["dry_limit_rel"]
    assert rel(L.or_moist_lapse(200.0, 60000.0, M_nw, cp, R_mix, g), g / cp) <= KAT["cold_limit_rel"]


def test_config_composition_matches_resolve():
    p = config_params()
    M_mean, R_mix, *_, M_bg, R_bg = _resolve([0.5578, 0.4109, 0.0313])
    assert p.R_mix == R_mix and p.M_bg == M_bg and p.R_bg == R_bg


@pytest.mark.parametrize("grid", [(11, 21, 41), (9, 19, 33)])
def test_symmetric_semantics_are_exactly_mirror_symmetric(grid):
    # jm odd: rows j and jm-1-j have the same red-black colour, so the pressure sweep maps
    # onto itself under the mirror (every grid of the reference and its configurations has
    # an odd jm, i.e. an equator row)
    p = config_params()
    st = make_state(*grid, seed=2, symmetric=True)
    o = OracleState(st, p)
    for it in range(1, 5):
        if it % 2 == 0:
            o.saturation_adjust()
            o.densities()
        o.rk4(buoyancy_ramp=0.5)
        o.pressure_sweep(1, it)
        o.store_n_level()
    for n in ["t", "u", "v", "w", "c", "cloud", "ice", "tke", "dis", "p_dyn", "aux_v", "p_stat"]:
        a = o.f[n]
        assert np.array_equal(a, mirror(a, n in ("v", "aux_v"))), n


def test_reference_semantics_break_symmetry_only_through_wall_distance_and_order():
    """The reference's own RK4 (in place, north-pole wall distance) is not mirror
    symmetric; the difference to the symmetric restatement stays at the size of the
    sweep-order effect."""
    p = config_params()
    p.wall_mode = Wall.REFERENCE
    st = make_state(11, 21, 41, seed=4, symmetric=True)
    a = OracleState(st, p)
    a.rk4(compat=1)
    b = OracleState(st, p)
    b.rk4(compat=0)
    for n in ["t", "u", "v", "w", "tke"]:
        scale = np.max(np.abs(b.f[n]))
        d = np.max(np.abs(a.f[n] - b.f[n])) / scale
        step = np.max(np.abs(b.f[n] - st[n])) / scale
        assert d <= 1e-3 * max(step, 1e-12), (n, d, step)
