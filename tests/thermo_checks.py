"""Known-answer and oracle checks of the device thermodynamics (csrc/thermo.cuh), shared by
the GPU test (the functions evaluated by a kernel through athad_thermo_eval) and the CPU test
(the same source compiled for the host).  `ev(fn, *cols)` evaluates function `fn` for the
tuples given column-wise and returns an array.

The known answers are those the reference's own self-tests assert (tests/golden/
thermo_kat.json: test/saturation_selftest.cpp, test/cond_column_selftest.cpp), each with its
assertion's tolerance.
"""
import json
import os

import numpy as np

from oracle_binding import lib as oracle_lib

KAT = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "thermo_kat.json")))
SAT_P, SUBL_P, LATENT, Q_SAT, DEW, CP_OF, M_NW, LAPSE, R_OF, Q_SAT_AT, DQ_DT = range(1, 12)


def rel(a, b):
    return abs(a - b) / abs(b)


def check_saturation_known_answers(dev):
    for c in KAT["saturation_pressure_hPa"]:
        assert rel(dev(SAT_P, c["T"])[0], c["want"]) <= c["rel"], c
    assert (dev(SAT_P, KAT["no_saturation_at"]) == -1.0).all()
    for c in KAT["sublimation_pressure_hPa"]:
        assert rel(dev(SUBL_P, c["T"])[0], c["want"]) <= c["rel"], c
    for c in KAT["latent_heat"]:
        assert rel(dev(LATENT, c["T"])[0], c["want"]) <= c["rel"], c
    assert dev(LATENT, 647.096)[0] == 0.0
    for c in KAT["saturation_mass_fraction"]:
        assert rel(dev(Q_SAT, c["E"], c["p"], c["M_other"])[0], c["want"]) <= c["rel"]
    assert dev(Q_SAT, [2000.0, -1.0], 1000.0, 0.034).tolist() == [1.0, 1.0]
    d = KAT["dew_point_boiling_60bar"]
    assert rel(dev(DEW, d["e"])[0], d["want"]) <= d["rel"]
    T = np.arange(150.0, 647.096, 0.5)
    p = np.where(T >= 273.16, dev(SAT_P, T), dev(SUBL_P, T))
    assert np.isfinite(p).all() and (np.diff(p) > 0).all()      # monotone (saturation_selftest.cpp:67-75)


def check_mixture_and_lapse_known_answers(dev):
    from athad_cond_b200._abi import composition
    s = KAT["surface_mixture"]
    comp = composition(list(s["x"]) + [0.0] * 5)
    cp = dev(CP_OF, comp["q_H2O"], comp["q_CO2"], s["cp_T"], comp["M_bg"])[0]
    assert rel(cp, s["cp"]) <= s["cp_rel"]
    M_nw = dev(M_NW, comp["q_H2O"], comp["q_CO2"], comp["M_bg"])[0]
    assert rel(M_nw * 1000, s["M_nonwater_g"]) <= s["M_nonwater_rel"]
    lp = KAT["lapse"]
    g = lp["g"]
    gm = dev(LAPSE, 513.15, 60000.0, M_nw, cp, comp["R_mix"], g)[0]
    assert rel(gm * 1000, lp["moist_K_per_km"]) <= lp["moist_rel"]
    ge = dev(LAPSE, lp["earth_T"], lp["earth_p"], lp["earth_M"], lp["earth_cp"], lp["earth_R"], g)[0]
    assert rel(ge * 1000, lp["earth_K_per_km"]) <= lp["earth_rel"]
    assert rel(dev(LAPSE, 700.0, 60000.0, M_nw, cp, comp["R_mix"], g)[0], g / cp) <= KAT["dry_limit_rel"]
    assert rel(dev(LAPSE, 200.0, 60000.0, M_nw, cp, comp["R_mix"], g)[0], g / cp) <= KAT["cold_limit_rel"]


def check_against_the_oracle_over_the_model_range(dev, tol):
    O = oracle_lib()
    rng = np.random.default_rng(20261203)
    T = np.concatenate([np.linspace(150.0, 700.0, 2001), rng.uniform(180.0, 650.0, 2000)])
    p = rng.uniform(1e-3, 1e5, T.size)                  # hPa, the column's range
    c = rng.uniform(0.0, 0.6, T.size)
    co2 = (1.0 - c) * rng.uniform(0.5, 0.99, T.size)
    M = rng.uniform(0.02, 0.045, T.size)

    def cmp(fn, ofn, *cols):
        got = dev(fn, *cols)
        want = np.array([ofn(*args) for args in zip(*[np.broadcast_to(np.asarray(x, float), T.shape) for x in cols])])
        den = np.maximum(np.abs(want), 1e-300)
        bad = np.abs(got - want) > tol * den
        assert not bad.any(), (fn, int(bad.sum()), float(np.max(np.abs(got - want) / den)))

    cmp(SAT_P, O.or_saturation_pressure, T)
    cmp(SUBL_P, O.or_sublimation_pressure, np.minimum(T, 273.16))
    cmp(LATENT, O.or_latent_heat, T)
    cmp(CP_OF, O.or_cp_of, c, co2, np.clip(T, 200.0, 2000.0), 0.028014)
    cmp(M_NW, O.or_M_nonwater, c, co2, 0.028014)
    cmp(R_OF, O.or_R_of, c, co2, 296.8)
    E = np.abs(dev(SAT_P, np.clip(T, 280.0, 640.0)))
    cmp(Q_SAT, O.or_saturation_mass_fraction, E, p, M)
