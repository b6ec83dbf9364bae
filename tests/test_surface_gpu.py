"""The surface-flux modules of the moist iteration on the device against the oracle, which
is pinned bit for bit against the reference (test_pin_reference.py).

athad_water_vapour_evaporation (ThermoAtm::waterVapourEvaporation, ThermoAtm.h:115-398):
c, Evaporation, the Dalton / Meyer / Rohwer rates and c_fix within 1e-12 of each field's
largest magnitude (CUDA's exp, log and sqrt in the saturation curves against glibc's pow and
exp), a supercritical surface column left alone.  athad_latent_sensible_heat
(ThermoAtm::latentSensibleHeat, ThermoAtm.h:36-112): Q_Sensible and Q_Latent bit for bit (no
transcendental but the correctly rounded sqrt).  A mirror-symmetric state stays
mirror-symmetric, bit for bit.  athad_co2_column / athad_water_budget (co2Column,
waterBudget): co2_total bit for bit, the mass-weighted means and first-call references within
1e-12 (FP64 sums in another fixed order), the drifts after the state changes.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state, mirror
from athad_cond_b200._abi import config_params
from oracle_binding import OracleState

pytestmark = pytest.mark.gpu

EVAP2D = ("Evaporation", "Evaporation_Dalton", "Evaporation_Meyer", "Evaporation_Rohwer", "c_fix")


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("grid", [(11, 21, 41), (41, 181, 361)])
def test_water_vapour_evaporation_matches_oracle(grid):
    im, jm, km = grid
    st = make_state(*grid, seed=131)
    t = st["t"].copy()
    t[0, 3, 7] = 700.0 / 273.15              # supercritical surface: no evaporation, c kept
    st["t"] = t
    st["c_fix"] = np.full((jm, km), 0.25)
    o = OracleState(st, config_params())
    o.water_vapour_evaporation()
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.upload_2d("c_fix", st["c_fix"])
        g.water_vapour_evaporation()
        c = g.download("c")
        assert relerr(c, o.f["c"]) <= 1e-12
        assert np.array_equal(c[4:], o.f["c"][4:])            # only levels 0-3 change
        assert np.array_equal(c[:4, 3, 7], st["c"][:4, 3, 7])
        for n in EVAP2D:
            a, b = g.download_2d(n), o.f2[n]
            assert relerr(a, b) <= 1e-12, (n, relerr(a, b))
        assert g.download_2d("Evaporation")[3, 7] == 0.0 and g.download_2d("c_fix")[3, 7] == 0.25


@pytest.mark.parametrize("grid", [(11, 21, 41), (41, 181, 361)])
def test_latent_sensible_heat_matches_oracle(grid):
    st = make_state(*grid, seed=137)
    o = OracleState(st, config_params())
    o.latent_sensible_heat(compat=0)
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.fill("Q_Sensible", 0.0)
        g.fill("Q_Latent", 0.0)
        g.latent_sensible_heat()
        for n in ("Q_Sensible", "Q_Latent"):
            assert np.array_equal(g.download(n), o.f[n]), n


def test_surface_fluxes_mirror_symmetric():
    grid = (21, 91, 181)
    st = make_state(*grid, seed=139, symmetric=True)
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.water_vapour_evaporation()
        g.latent_sensible_heat()
        for n in ("c", "Q_Sensible"):
            a = g.download(n)
            assert np.array_equal(a, mirror(a, False)), n
        for n in EVAP2D:
            a = g.download_2d(n)
            assert np.array_equal(a, a[::-1, :]), n


@pytest.mark.parametrize("grid", [(11, 21, 41), (41, 181, 361)])
def test_mass_budgets_match_oracle(grid):
    st = make_state(*grid, seed=149)
    o = OracleState(st, config_params())
    want = o.budgets()
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        co2 = g.co2_column()
        h2o = g.water_budget()
        assert np.array_equal(g.download_2d("co2_total"), o.f2["co2_total"])
        for got, key in ((co2["q_mean"], "q_co2_ref"), (h2o["q_mean"], "q_h2o_ref"),
                         (h2o["q_fixed"], "q_h2o_fixed_ref")):
            assert abs(got - want[key]) <= 1e-12 * want[key], key
        assert co2["drift_pct"] == 0.0 and h2o["drift_pct"] == 0.0 and not np.any(h2o["level_drift"])
        assert abs(h2o["air_now"] - want["air_levels"].sum()) <= 1e-12 * want["air_levels"].sum()
        # more water: the budget drifts by the change, the references stay
        g.upload("c", 1.01 * st["c"])
        h2o2 = g.water_budget()
        assert h2o2["q_ref"] == h2o["q_mean"] and h2o2["drift_pct"] > 0.0
        assert h2o2["air_drift_pct"] == 0.0 and np.all(h2o2["level_drift"] >= 0.0)
