"""Parity over many iterations, from the reference's deterministic initial state.

  * the plain FP64 hot path (RK4 every iteration, pressure sweep every 4th, saturation
    adjustment, moist convection and densities every 2nd, the time-level copy) for 100
    iterations on configuration 1's 21 x 91 x 181 grid against the oracle: every prognostic
    field and the diagnosed pressure and densities within 1e-9 of the field's largest
    magnitude, and the device state exactly mirror symmetric;
  * the same for 4 iterations on configuration 2's 41 x 181 x 361 grid;
  * the whole model iteration (athad_cond_b200.loop.ModelLoop: boundary conditions,
    filters, turbulence, ice scheme, radiation, surface fluxes, caps, diagnostics, the force
    fields, the right-hand side's outputs and the skin temperature around the hot path) for
    10 iterations against the oracle driving the same module sequence.
The oracle runs the same initial state (or_init_state, the device semantics); it is pinned
against the reference in tests/test_pin_initial_state.py and tests/test_pin_reference.py.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, config_init
from athad_cond_b200._abi import config_params
from athad_cond_b200.loop import (CONVECTION_FIELDS, ICE_FLUXES, MOIST_FIELDS_AFTER_SATADJ,
                                  TURBULENCE_FIELDS, ModelLoop)
from oracle_binding import OracleState, update_skin_temperature

pytestmark = pytest.mark.gpu

FIELDS = ["t", "u", "v", "w", "c", "cloud", "ice", "gr", "co2", "tke", "dis", "p_dyn", "p_stat", "r_humid"]
ANTISYMMETRIC = {"v", "vn", "aux_v", "MC_v", "v_u", "v_d"}
TOL = 1e-9
DT = 4e-5


def errors(g, o, names):
    out = {}
    for n in names:
        a, b = g.download(n), o.f[n]
        den = float(np.max(np.abs(b)))
        out[n] = float(np.max(np.abs(a - b))) / den if den > 0 else float(np.max(np.abs(a)))
    return out


def hot_path_iteration_device(g, it):
    if it % 4 == 0:
        g.PressureSolverAtm_run(total_iter_count=it)
    if it % 2 == 0:
        g.SaturationAdjustment_run()
        g.MoistConvection_run(it)
        g.densities()
    g.solveRungeKutta_Atmosphere_Turb(DT, 1.0, min(1.0, it / 300.0), store_n_level=True)


def hot_path_iteration_oracle(o, it):
    if it % 4 == 0:
        o.pressure_sweep(1, it)
    if it % 2 == 0:
        o.saturation_adjust()
        o.moist_convection(it)
        o.densities()
    o.rk4(dt=DT, buoyancy_ramp=min(1.0, it / 300.0))
    o.store_n_level()


@pytest.mark.parametrize("grid,iterations", [((21, 91, 181), 100), ((41, 181, 361), 4)])
def test_fp64_hot_path_from_the_initial_state(grid, iterations):
    p = config_params()
    cfg = config_init()
    o = OracleState.initial(*grid, p, cfg)
    with GpuAtmosphere(*grid, p) as g:
        g.initial_state(cfg)
        for it in range(1, iterations + 1):
            hot_path_iteration_device(g, it)
            hot_path_iteration_oracle(o, it)
        err = errors(g, o, FIELDS)
        for n in FIELDS + ["vn", "aux_v", "MC_v"]:
            a = g.download(n)
            m = -a[:, ::-1, :] if n in ANTISYMMETRIC else a[:, ::-1, :]
            assert np.array_equal(a, m), n
    bad = {n: e for n, e in err.items() if not e <= TOL}
    assert not bad, (bad, err)


def oracle_loop_iteration(o, it, total, tropopause, omega_rad=0.05, t_skin_relax=0.25, checkpoint=20):
    """cAtmosphereModel::run_3D_loop's module sequence on the oracle, in ModelLoop's order."""
    if it % 4 == 0:
        o.pressure_sweep(1, total)
    if it % 2 == 0:
        o.saturation_adjust()
        for n in MOIST_FIELDS_AFTER_SATADJ:
            o.damp_wiggles(n)
        o.ice_scheme()
        for n in ICE_FLUXES:
            o.damp_wiggles(n)
        o.moist_convection(it)
        for n in CONVECTION_FIELDS:
            o.damp_wiggles(n)
        o.moist_caps()
        o.vapour_ceiling()
        o.densities()
        o.forces()
        o.stand_atm_dew_point(tropopause)
        o.water_vapour_evaporation()
        o.latent_sensible_heat()
        o.turbulence_run()
        for n in TURBULENCE_FIELDS:
            o.damp_wiggles(n)
    o.boundary_conditions()
    budget = 2 if it % checkpoint == 0 else 0
    o.rk4(dt=DT, buoyancy_ramp=min(1.0, total / 300.0), write_diagnostics=1 | budget)
    o.post_rk4_filters()
    o.store_n_level()
    o.radiative_heating(omega_rad)
    o.params.t_skin = update_skin_temperature(o.params, o.f2["albedo"], o.params.t_skin, t_skin_relax)


def test_model_loop_matches_oracle_for_ten_iterations():
    grid = (21, 91, 181)
    im, jm, _ = grid
    p = config_params()
    cfg = config_init()
    o = OracleState.initial(*grid, p, cfg)
    # ModelLoop's default tropopause: the configured heights lie above the 120 km lid, so
    # every row's level is im - 1 (the equator row's neighbour rule changes nothing)
    trop = np.full(jm, im - 1)
    with GpuAtmosphere(*grid, p) as g:
        g.initial_state(cfg)
        loop = ModelLoop(g)
        skins = []
        for it in range(1, 11):
            rep = loop.iteration()
            oracle_loop_iteration(o, it, it, trop)
            skins.append((rep["t_skin"], o.params.t_skin))
        names = FIELDS + ["nue", "P_rain", "P_snow", "Precipitation", "TempDewPoint", "HumidityRel",
                          "Q_Latent", "Q_Sensible", "radiation", "S_v", "S_c", "MC_t", "MC_q",
                          "CoriolisForce", "BuoyancyForce", "PressureGradientForce", "prod"]
        err = errors(g, o, names)
    bad = {n: e for n, e in err.items() if not e <= TOL}
    assert not bad, (bad, err)
    for a, b in skins:
        assert abs(a - b) <= 1e-12 * abs(b)
