"""Pin of the oracle against the reference itself.

The reference is built from its own sources (oracle/ref/Makefile -> oracle/_ref/pin, an
IEEE build) and driven through its own functions on its own initial state at its only
grid, 61 x 181 x 361 (cAtmosphereModel.h:162).  The oracle, in its reference-compatible
semantics, must reproduce every hot-path function bit for bit:

  * RHS_Atmosphere_Turb at sampled cells;
  * solveRungeKutta_Atmosphere_Turb, the in-place sweep run with T OpenMP threads;
  * PressureSolverAtm::run; SaturationAdjustment::run; ThermoAtm::densities (both modes);
  * the per-iteration boundary conditions (bcRadius, apply_wall_bc, bcTheta, bcPhi);
  * the filters after the RK4 step and the moist iteration's damp_wiggles;
  * TurbulenceAtm::run (its in-place sweep on one thread) for the three closures;
  * TwoCatIceScheme::run, and the schemes of the other CategoryIceScheme values (ZeroCat,
    OneCat, ThreeCat); MultiLayerRadiation::run and radiation mode 2's heating;
  * the diagnostics standAtm_DewPoint_HumidRel and findResiduumAtm;
  * the surface fluxes waterVapourEvaporation and latentSensibleHeat;
  * the mass budgets co2Column and waterBudget (their sums on one thread);
  * updateSkinTemperature with planetaryShortWave.

Skipped where the reference was not built (a machine without the reference sources).
"""
import concurrent.futures
import ctypes
import os

import numpy as np
import pytest

import ref_binding
from athad_cond_b200._abi import FIELD_NAMES, config_params, Wall
from oracle_binding import OracleState, update_skin_temperature

pytestmark = pytest.mark.skipif(not ref_binding.available("pin"),
                                reason="reference not built (oracle/_ref/pin)")

THREADS = max(1, min(8, os.cpu_count() or 1))
DT = 4e-5


@pytest.fixture(scope="module")
def ref():
    cwd = os.getcwd()
    os.chdir(os.environ.get("TMPDIR", "/tmp"))
    try:
        R = ref_binding.Reference("pin", threads=THREADS)
        R.init_state()
        snap = {n: R.get(n) for n in FIELD_NAMES}
        snap2 = {n: R.get2(n) for n in ("t_top_init", "p_stat_landscape", "vel_star")}
        yield R, snap, snap2
        R.close()
    finally:
        os.chdir(cwd)


_ORACLE_THREAD = concurrent.futures.ThreadPoolExecutor(max_workers=1)


def side_by_side(reference_call, oracle_call):
    """Run the oracle's call on a worker thread while the reference's runs on this one: both
    are C calls that release the interpreter and work on their own copies of the state."""
    done = _ORACLE_THREAD.submit(oracle_call)
    reference_call()
    done.result()


def fresh(ref):
    R, snap, snap2 = ref
    for n, a in snap.items():
        R.set(n, a)
    for n, a in snap2.items():
        R.set2(n, a)
    p = config_params()
    p.wall_mode = Wall.REFERENCE
    st = dict(snap)
    st.update(snap2)
    return R, OracleState(st, p)


def assert_identical(R, o, names):
    for n in names:
        a, b = R.get(n), o.f[n]
        assert np.array_equal(a, b), (n, float(np.max(np.abs(a - b))), int(np.count_nonzero(a != b)))


def test_derived_constants(ref):
    R, _, _ = ref
    c = R.constants()
    p = config_params()
    assert c["re_turb"] == p.re_turb
    assert c["M_bg"] == p.M_bg and c["R_bg"] == p.R_bg and c["R_mix"] == p.R_mix
    assert c["dt_visc"] == DT


def test_rhs_cells_bit_exact(ref):
    R, o = fresh(ref)
    R.lib.ref_level_mean(R.h)
    o.prof["t_ref_level"][:] = R.getp("t_ref_level")
    R.set_scalars(DT, 1.0, 0.3, 90, 90)
    im, jm, km = R.shape
    rng = np.random.default_rng(2026)
    cells = [(1 + rng.integers(im - 2), 1 + rng.integers(jm - 2), 1 + rng.integers(km - 2)) for _ in range(400)]
    cells += [(1, 1, 1), (im - 2, jm - 2, km - 2), (1, jm // 2, km // 2), (im // 2, 1, 1)]
    for (i, j, k) in cells:
        a = R.rhs_cell(i, j, k)
        b = o.rhs_cell(i, j, k, dt=DT, buoyancy_ramp=0.3, compat=1)
        assert np.array_equal(a, b), ((i, j, k), a - b)


def test_rk4_step_bit_exact(ref):
    R, o = fresh(ref)
    R.set_scalars(DT, 1.0, 0.3, 90, 90)
    side_by_side(lambda: R.lib.ref_rk4(R.h), lambda: o.rk4(dt=DT, buoyancy_ramp=0.3, compat=THREADS))
    assert_identical(R, o, ["t", "u", "v", "w", "c", "cloud", "ice", "gr", "co2", "tke", "dis",
                            "aux_u", "aux_v", "aux_w"])
    assert np.array_equal(R.getp("t_ref_level"), o.prof["t_ref_level"])


DIAGNOSTICS = ["prod", "tke_source", "dis_source", "CoriolisForce", "BuoyancyForce",
               "PressureGradientForce", "Q_Latent", "Q_Sensible",
               "vbud_pgf", "vbud_cor", "vbud_advv", "vbud_advh", "vbud_diff", "vbud_other",
               "wbud_pgf", "wbud_cor", "wbud_advv", "wbud_advh", "wbud_diff", "wbud_other"]


def test_rk4_step_diagnostic_outputs_bit_exact(ref):
    """The right-hand side's diagnostic outputs of the last stage (RHS_Atm_Turb.cpp:447-491,
    1031-1057), with the momentum-budget capture of a checkpoint iteration."""
    R, o = fresh(ref)
    R.set_scalars(DT, 1.0, 0.3, 90, 90)
    R.lib.ref_set_budget_capture.argtypes = [ctypes.c_void_p, ctypes.c_int]
    R.lib.ref_set_budget_capture(R.h, 1)
    side_by_side(lambda: R.lib.ref_rk4(R.h),
                 lambda: o.rk4(dt=DT, buoyancy_ramp=0.3, compat=THREADS, write_diagnostics=3))
    R.lib.ref_set_budget_capture(R.h, 0)
    interior = (slice(1, -1), slice(1, -1), slice(1, -1))
    for n in DIAGNOSTICS:
        a, b = R.get(n)[interior], o.f[n][interior]
        assert np.array_equal(a, b), (n, float(np.max(np.abs(a - b))))
    assert float(np.max(np.abs(o.f["CoriolisForce"]))) > 0.0 and float(np.max(np.abs(o.f["Q_Sensible"]))) > 0.0


def test_pressure_sweep_bit_exact(ref):
    R, o = fresh(ref)
    rng = np.random.default_rng(5)
    for n in ("aux_u", "aux_v", "aux_w"):
        a = 1e-2 * rng.standard_normal(R.shape)
        R.set(n, a)
        o.f[n][:] = a
    for it in (4, 400):
        R.set_scalars(DT, 1.0, 1.0, it, it)
        R.lib.ref_pressure(R.h)
        o.pressure_sweep(1, it, compat=1)
    assert_identical(R, o, ["p_dyn", "aux_u", "aux_v", "aux_w"])


def test_saturation_adjustment_bit_exact(ref):
    R, o = fresh(ref)
    R.lib.ref_satadj(R.h)
    o.saturation_adjust(compat=1)
    assert_identical(R, o, ["t", "c", "cloud", "ice", "gr", "S_c_c", "P_rain", "P_snow", "S_v", "S_c"])


@pytest.mark.parametrize("set_water", [0, 1])
def test_densities_bit_exact(ref, set_water):
    R, o = fresh(ref)
    R.lib.ref_densities(R.h, set_water)
    o.densities(set_water_profile=bool(set_water), compat=1)
    assert_identical(R, o, ["t", "p_stat", "r_humid", "r_dry", "c"])
    for n in ("t_top_init", "p_stat_landscape"):
        assert np.array_equal(R.get2(n), o.f2[n]), n
    for n in ("rho_base", "dlnrho_dr"):
        assert np.array_equal(R.getp(n), o.prof[n]), n


MC_FIELDS = ["s", "s_u", "s_d", "M_u", "M_d", "q_v_u", "q_c_u", "q_v_d", "u_u", "v_u", "w_u",
             "u_d", "v_d", "w_d", "E_u", "D_u", "E_d", "D_d", "c_u", "e_l", "e_d", "e_p", "g_p",
             "P_conv", "CloudBase", "LevelFreeSinking", "Deep_beg", "Deep_end",
             "MC_t", "MC_q", "MC_v", "MC_w"]


def test_moist_convection_bit_exact_two_calls(ref):
    """Two consecutive calls: the second reads the first's leftovers (E_u, D_u, w_u, ...
    are not reset between calls, MoistConvection.h:339-376)."""
    R, o = fresh(ref)
    for n in ("Evaporation", "Q_sensible_2D"):
        o.f2[n][:] = R.get2(n)
    for it in (2, 4):
        side_by_side(lambda: R.lib.ref_moist(R.h, it), lambda: o.moist_convection(it, compat=1))
        assert_identical(R, o, MC_FIELDS)


def test_boundary_conditions_bit_exact(ref):
    """bcRadius + apply_wall_bc + bcTheta + bcPhi on a state whose every field was moved off
    its boundary-consistent values (so every boundary formula writes something new)."""
    R, o = fresh(ref)
    im, jm, km = R.shape
    pattern = 1.0 + 1e-3 * np.sin(np.arange(im * jm * km, dtype=np.float64) * 0.37).reshape(im, jm, km)
    for n in FIELD_NAMES:
        a = R.get(n) * pattern
        R.set(n, a)
        o.f[n][...] = a
    R.bc()
    o.boundary_conditions()
    assert_identical(R, o, FIELD_NAMES)


def test_post_rk4_filters_bit_exact(ref):
    """The post-RK4 filter sequence of the reference (its orographic, steep-massif and
    coastal filters included, which flat terrain leaves without effect) against the
    oracle's polar zonal and radial Shapiro filters."""
    R, o = fresh(ref)
    im, jm, km = R.shape
    rng = np.random.default_rng(31)
    for n in ("u", "v", "w"):
        a = R.get(n) + 1e-3 * rng.standard_normal((im, jm, km))
        R.set(n, a)
        o.f[n][...] = a
    R.post_rk4_filters()
    o.post_rk4_filters()
    assert_identical(R, o, FIELD_NAMES)


def test_damp_wiggles_bit_exact(ref):
    R, o = fresh(ref)
    for n in ("t", "ice", "c", "cloud"):
        R.damp_wiggles(n)
        o.damp_wiggles(n, compat=1)
    assert_identical(R, o, ["t", "ice", "c", "cloud"])


@pytest.mark.parametrize("model", ["k_epsilon", "k_omega", "k_omega_SST"])
def test_turbulence_run_bit_exact(ref, model):
    """TurbulenceAtm::run on one thread (its serial in-place sweep) against the oracle's
    compat mode, on the initial state with tke pulled below its background floor in a band
    of cells, so the floors bind at neighbours visited before and after."""
    from athad_cond_b200._abi import Turb
    R, o = fresh(ref)
    im, jm, km = R.shape
    R.set_turb_model(model)
    o.params.turb_model = {"k_epsilon": Turb.K_EPSILON, "k_omega": Turb.K_OMEGA,
                           "k_omega_SST": Turb.K_OMEGA_SST}[model]
    rng = np.random.default_rng(47)
    tke = R.get("tke")
    tke[:, jm // 3: jm // 3 + 20, :] *= rng.uniform(0.0, 1.0, (im, 20, km))
    tke[2:6, :, 100:110] = -1e-4
    R.set("tke", tke)
    o.f["tke"][...] = tke
    for n in ("u", "v", "w"):
        a = R.get(n) * (1.0 + 0.1 * rng.standard_normal((im, jm, km)))
        R.set(n, a)
        o.f[n][...] = a
    try:
        R.turbulence_run(threads=1)
    finally:
        R.set_turb_model("k_omega_SST")
    o.turbulence_run(compat=1)
    assert_identical(R, o, ["tke", "dis", "nue", "prod", "tke_source", "dis_source"])
    assert np.array_equal(R.get2("vel_star"), o.f2["vel_star"])


ICE_FIELDS = ["t", "c", "cloud", "ice", "gr", "P_rain", "P_snow", "P_graupel", "Precipitation",
              "P_rainn", "P_snown", "S_v", "S_c", "S_i", "S_r", "S_s", "S_g", "S_c_c"]


def test_two_cat_ice_scheme_bit_exact(ref):
    """TwoCatIceScheme::run (the configuration's CategoryIceScheme 2) on the reference's state
    after a saturation adjustment, with falling rain and snow seeded from above."""
    R, o = fresh(ref)
    im, jm, km = R.shape
    R.lib.ref_satadj(R.h)
    o.saturation_adjust(compat=1)
    rng = np.random.default_rng(53)
    for n in ("P_rainn", "P_snown"):
        a = 2e-4 * rng.random((im, jm, km))
        R.set(n, a)
        o.f[n][...] = a
    R.two_cat_ice()
    o.two_cat_ice_scheme()
    assert_identical(R, o, ICE_FIELDS)


def seed_precipitation_state(R, o, seed, cold_band):
    """The reference's state after a saturation adjustment, with falling rain, snow and
    graupel seeded from above, cloud ice and graupel present, and cloud water in every cell
    of the k = 1 plane (OneCat's serial loop reads its carried autoconversion rate before any
    assignment otherwise).  cold_band: levels 40-52 redrawn between 230 and 285 K with cloud
    water and vapour around saturation, so that the sub-freezing branches act."""
    im, jm, km = R.shape
    R.lib.ref_satadj(R.h)
    o.saturation_adjust(compat=1)
    rng = np.random.default_rng(seed)
    new = {}
    for n in ("P_rainn", "P_snown", "P_graupel"):
        new[n] = 2e-4 * rng.random((im, jm, km))
    for n in ("ice", "gr"):
        a = o.f[n].copy()
        a[30:55] += np.where(rng.random((25, jm, km)) < 0.5, 0.0, 1e-5 * rng.random((25, jm, km)))
        new[n] = a
    cloud = o.f["cloud"].copy()
    if cold_band:
        t = o.f["t"].copy()
        t[40:53] = (230.0 + 55.0 * rng.random((13, jm, km))) / 273.15
        new["t"] = t
        cloud[40:53] = np.where(rng.random((13, jm, km)) < 0.3, 0.0, 2e-3 * rng.random((13, jm, km)))
        c = o.f["c"].copy()
        c[40:53] *= 0.5 + rng.random((13, jm, km))
        new["c"] = c
    cloud[:, :, 1] = np.maximum(cloud[:, :, 1], 1e-5)
    new["cloud"] = cloud
    for n, a in new.items():
        R.set(n, a)
        o.f[n][...] = a


@pytest.mark.parametrize("category", [0, 1, 3])
@pytest.mark.parametrize("cold_band", [False, True])
def test_other_ice_schemes_bit_exact(ref, category, cold_band):
    """ZeroCat, OneCat and ThreeCatIceScheme::run on the reference's state with falling
    precipitation seeded (and a sub-freezing band redrawn)."""
    R, o = fresh(ref)
    seed_precipitation_state(R, o, 60 + category, cold_band)
    side_by_side(lambda: R.ice_scheme(category), lambda: o.ice_scheme(category))
    assert_identical(R, o, ICE_FIELDS)


def test_multilayer_radiation_bit_exact(ref):
    """MultiLayerRadiation::run on the reference's state (cloud and ice seeded so the cloud
    optical depth and the short-wave albedo bump act), then radiation mode 2's heating."""
    R, o = fresh(ref)
    im, jm, km = R.shape
    rng = np.random.default_rng(67)
    for n in ("cloud", "ice"):
        a = 2e-4 * rng.random((im, jm, km))
        R.set(n, a)
        o.f[n][...] = a
    R.mlr()
    o.multilayer_radiation()
    assert_identical(R, o, ["t", "radiation", "epsilon"])
    for n in ("epsilon_2D", "albedo"):
        assert np.array_equal(R.get2(n), o.f2[n]), n
    R, o = fresh(ref)
    R.radiative_heating(0.05)
    o.radiative_heating(0.05)
    assert_identical(R, o, ["t", "radiation", "epsilon"])


def test_precipitation_sum_bit_exact(ref):
    """UtilsAtm::precipitationSum against the oracle's moist caps (the caps themselves are
    inline code of run_3D_loop; on this state's values within the caps they change nothing
    but Precipitation)."""
    R, o = fresh(ref)
    im, jm, km = R.shape
    rng = np.random.default_rng(71)
    for n in ("P_rain", "P_snow", "P_graupel", "P_conv"):
        a = 1e-4 * rng.random((im, jm, km))
        R.set(n, a)
        o.f[n][...] = a
    for n in ("S_v", "S_c", "S_i", "S_r", "S_s", "S_g", "S_c_c"):
        z = np.zeros((im, jm, km))
        R.set(n, z)
        o.f[n][...] = z
    R.precipitation_sum()
    o.moist_caps()
    assert np.array_equal(R.get("Precipitation"), o.f["Precipitation"])


def equator_rule(layers):
    """ThermoAtm.h:414-419: the equator row (row 90 of the reference's 181) takes its
    northern neighbour's tropopause level."""
    jm = len(layers)
    return [int(layers[j - 1] if j == (jm - 1) // 2 else layers[j]) for j in range(jm)]


def test_stand_atm_dew_point_bit_exact(ref):
    """ThermoAtm::standAtm_DewPoint_HumidRel on the reference's state, with a supercritical
    patch (no saturation state: the -1 sentinel) and a dry patch (zero vapour)."""
    R, o = fresh(ref)
    t = R.get("t")
    t[5:8, 20:24, 100:110] = 700.0 / 273.15
    c = R.get("c")
    c[10:12, 60:64, 200:210] = 0.0
    for n, a in (("t", t), ("c", c)):
        R.set(n, a)
        o.f[n][...] = a
    layers = equator_rule(R.tropopause_layers())
    side_by_side(R.stand_atm, lambda: o.stand_atm_dew_point(layers))
    assert_identical(R, o, ["TempStand", "TempDewPoint", "HumidityRel"])
    hr = o.f["HumidityRel"]
    assert np.all(hr[5:8, 20:24, 100:110] == -1.0) and np.all(hr[10:12, 60:64, 200:210] == 0.0)


def test_find_residuum_bit_exact(ref):
    """UtilsAtm::findResiduumAtm on the reference's state and with a non-finite velocity
    planted in the band: the residuum and its cell exactly, the finite and non-finite counts,
    the grid average to the 8 digits the reference prints."""
    for plant in (False, True):
        R, o = fresh(ref)
        if plant:
            u = R.get("u")
            u[15, 40, 100] = np.nan
            R.set("u", u)
            o.f["u"][...] = u
        r, q = R.find_residuum(threads=1), o.find_residuum()
        assert r["residuum"] == q["residuum"] and r["at"] == q["at"]
        assert r["n_cells"] == q["n_cells"] and r["n_nonfinite"] == q["n_nonfinite"]
        assert abs(r["avg_abs_8"] - q["avg_abs"]) <= 1e-7 * q["avg_abs"]
        if plant:
            assert q["n_nonfinite"] == 2 and q["first_nonfinite"] == (14, 40, 100)


def test_surface_fluxes_bit_exact(ref):
    """ThermoAtm::waterVapourEvaporation (with one supercritical surface column, where the
    reference leaves c and c_fix alone and reports no evaporation) and ::latentSensibleHeat
    on the reference's state."""
    R, o = fresh(ref)
    t = R.get("t")
    t[0, 5, 10] = 700.0 / 273.15
    R.set("t", t)
    o.f["t"][...] = t
    cf = R.get2("c_fix")
    o.f2["c_fix"][...] = cf
    R.evaporation()
    o.water_vapour_evaporation()
    assert_identical(R, o, ["c"])
    for n in ("Evaporation", "Evaporation_Dalton", "Evaporation_Meyer", "Evaporation_Rohwer", "c_fix"):
        assert np.array_equal(R.get2(n), o.f2[n]), n
    assert o.f2["Evaporation"][5, 10] == 0.0 and o.f2["c_fix"][5, 10] == cf[5, 10]
    R.latent_sensible()
    o.latent_sensible_heat(compat=1)
    for n in ("Q_Sensible", "Q_Latent"):
        a, b = R.get(n), o.f[n]
        assert np.array_equal(a[1:-1, 1:-1, 1:-1], b[1:-1, 1:-1, 1:-1]) and np.array_equal(a[0], b[0]), n


def test_mass_budgets_bit_exact(ref):
    """ThermoAtm::co2Column and ::waterBudget as first calls, the reference on one thread: the
    references they set (mass-weighted means, level air masses, level water) and co2_total."""
    R, o = fresh(ref)
    r, q = R.budgets(threads=1), o.budgets()
    for key in ("q_co2_ref", "q_h2o_ref", "q_h2o_fixed_ref"):
        assert r[key] == q[key], key
    for key in ("air_levels", "h2o_levels"):
        assert np.array_equal(r[key], q[key]), key
    assert np.array_equal(R.get2("co2_total"), o.f2["co2_total"])


def test_skin_temperature_bit_exact(ref):
    """cAtmosphereModel::updateSkinTemperature after MultiLayerRadiation::run (which sets the
    albedo and the insolation profile), twice in a row."""
    R, o = fresh(ref)
    R.mlr()
    albedo = R.get2("albedo")
    p = config_params()
    t = R.skin(0.0)
    for _ in range(2):
        want = update_skin_temperature(p, albedo, t, 0.25)
        t = R.skin(0.25)
        assert t == want
