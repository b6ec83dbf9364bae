"""Parity of the CUDA path (through the C ABI) with the CPU oracle on identical seeded
states, and exact north-south mirror symmetry of the CUDA results.

Tolerances (relative to the field's max magnitude, FP64):
  * Poisson sweep, project_initial_velocity, level mean: bit-identical (no
    transcendentals; both sides round every operation as written).
  * RK4 step: 1e-12 (the SST blending function calls tanh/pow, whose last bit differs
    between CUDA and glibc).
  * saturation adjustment, densities: 1e-11 (IAPWS exp/pow chains inside a Newton
    iteration / a column ODE).
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state, mirror
from athad_cond_b200._abi import FIELD_NAMES, Precision, config_params, Wall, Turb
from oracle_binding import OracleState

pytestmark = pytest.mark.gpu

GRIDS = [(11, 21, 41), (21, 91, 181)]
PROG = ["t", "u", "v", "w", "c", "cloud", "ice", "gr", "co2", "tke", "dis"]
ANTI = {"v", "vn", "aux_v", "MC_v"}


def relerr(a, b):
    scale = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(a - b)) / scale)


def gpu_with(state, params):
    im, jm, km = state["t"].shape
    g = GpuAtmosphere(im, jm, km, params)
    g.upload_state(state)
    return g


@pytest.mark.parametrize("grid", GRIDS)
@pytest.mark.parametrize("wall", [Wall.MIRROR, Wall.REFERENCE])
def test_rk4_step_matches_oracle(grid, wall):
    p = config_params()
    p.wall_mode = wall
    st = make_state(*grid, seed=7)
    o = OracleState(st, p)
    o.rk4(dt=4e-5, diffusion_ramp=1.0, buoyancy_ramp=0.5, write_diagnostics=True)
    with gpu_with(st, p) as g:
        g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, 0.5, write_diagnostics=True)
        for n in PROG + ["aux_u", "aux_v", "aux_w", "prod", "tke_source", "dis_source"]:
            e = relerr(g.download(n), o.f[n])
            assert e <= 1e-12, (n, e)
        tr = g.download_profile("t_ref_level")
        assert np.array_equal(tr, o.prof["t_ref_level"])


DIAGNOSTICS = ["prod", "tke_source", "dis_source", "CoriolisForce", "BuoyancyForce",
               "PressureGradientForce", "Q_Latent", "Q_Sensible",
               "vbud_pgf", "vbud_cor", "vbud_advv", "vbud_advh", "vbud_diff", "vbud_other",
               "wbud_pgf", "wbud_cor", "wbud_advv", "wbud_advh", "wbud_diff", "wbud_other"]


@pytest.mark.parametrize("precision", [Precision.FP64, Precision.MIXED])
def test_rk4_step_diagnostic_outputs(precision):
    """The right-hand side's diagnostic outputs (acting forces, heat diagnostics, momentum
    budget terms) on a diagnostic step: within 1e-12 of the oracle in FP64 (the same IEEE
    operations; CUDA's saturation curve only decides the latent-heat branch), exactly mirror
    symmetric (v-terms antisymmetric).  The mixed form forms them in FP64 from its FP32 stage
    state, whose rounding the first and second differences amplify: checked for symmetry
    and finiteness, and the smooth ones (buoyancy, Coriolis) within 1e-5."""
    grid = (11, 21, 41)
    p = config_params()
    p.precision = int(precision)
    st = make_state(*grid, seed=17, symmetric=True)
    o = OracleState(st, p)
    o.rk4(dt=4e-5, diffusion_ramp=1.0, buoyancy_ramp=0.5, write_diagnostics=3)
    with gpu_with(st, p) as g:
        g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, 0.5, write_diagnostics=3)
        for n in DIAGNOSTICS:
            a = g.download(n)
            assert np.isfinite(a).all(), n
            e = relerr(a, o.f[n])
            if precision == Precision.FP64:
                assert e <= 1e-12, (n, e)
            elif n in ("BuoyancyForce", "CoriolisForce"):
                assert e <= 1e-5, (n, e)
            anti = n.startswith("vbud") or n == "v"
            assert np.array_equal(a, mirror(a, anti)), n
            assert float(np.max(np.abs(a))) > 0.0, n


@pytest.mark.parametrize("turb", [Turb.K_EPSILON, Turb.K_OMEGA])
def test_rk4_other_closures(turb):
    p = config_params()
    p.turb_model = turb
    st = make_state(11, 21, 41, seed=3)
    o = OracleState(st, p)
    o.rk4()
    with gpu_with(st, p) as g:
        g.solveRungeKutta_Atmosphere_Turb(4e-5)
        for n in PROG:
            assert relerr(g.download(n), o.f[n]) <= 1e-12, n


def test_rk4_switches():
    p = config_params()
    p.coriolis_nontrad = 1
    p.metric_curvature = 1
    p.tracer_diff_flux = 1
    p.metric_r0 = 0.0
    st = make_state(11, 21, 41, seed=5)
    st["dlnrho_dr"] = np.linspace(-1.0, -3.0, 11)
    o = OracleState(st, p)
    o.rk4()
    with gpu_with(st, p) as g:
        g.solveRungeKutta_Atmosphere_Turb(4e-5)
        for n in PROG:
            assert relerr(g.download(n), o.f[n]) <= 1e-12, n


@pytest.mark.parametrize("grid", GRIDS)
def test_rk4_mirror_symmetry_exact(grid):
    p = config_params()
    st = make_state(*grid, seed=11, symmetric=True)
    with gpu_with(st, p) as g:
        for it in range(3):
            g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, 0.2)
            g.storeIntermediateData3D()
        for n in PROG + ["aux_u", "aux_v", "aux_w"]:
            a = g.download(n)
            assert np.array_equal(a, mirror(a, n in ANTI)), n


@pytest.mark.parametrize("grid", GRIDS)
def test_pressure_sweep_bit_exact(grid):
    p = config_params()
    st = make_state(*grid, seed=13)
    rng = np.random.default_rng(1)
    for n in ("aux_u", "aux_v", "aux_w"):
        st[n] = 1e-3 * rng.standard_normal(st["t"].shape)
    st["aux_v"][:, 3, 5] = 1e6       # one clamped source
    o = OracleState(st, p)
    cells, clamped = o.pressure_sweep(n_sweeps=3, total_iter_count=400)
    with gpu_with(st, p) as g:
        g.PressureSolverAtm_run(total_iter_count=400, n_sweeps=3)
        for n in ("p_dyn", "aux_u", "aux_v", "aux_w"):
            assert np.array_equal(g.download(n), o.f[n]), n
        r = g.report()
        assert r["poisson_src_cells"] == cells and r["poisson_src_clamped"] == clamped


def test_pressure_sweep_anelastic_and_divergence():
    p = config_params()
    p.anelastic = 1
    p.metric_divergence = 1
    p.poisson_metric_fix = 0
    st = make_state(11, 21, 41, seed=17)
    st["dlnrho_dr"] = np.linspace(-1.0, -3.0, 11)
    rng = np.random.default_rng(2)
    for n in ("aux_u", "aux_v", "aux_w"):
        st[n] = 1e-3 * rng.standard_normal(st["t"].shape)
    o = OracleState(st, p)
    o.pressure_sweep(n_sweeps=2, total_iter_count=4)
    with gpu_with(st, p) as g:
        g.PressureSolverAtm_run(total_iter_count=4, n_sweeps=2)
        assert np.array_equal(g.download("p_dyn"), o.f["p_dyn"])


def test_project_initial_velocity_bit_exact():
    p = config_params()
    st = make_state(11, 21, 41, seed=19)
    o = OracleState(st, p)
    o.project_initial_velocity(n_sweeps=20)
    with gpu_with(st, p) as g:
        g.project_initial_velocity(n_sweeps=20)
        for n in ("u", "v", "w", "p_dyn", "aux_u"):
            assert np.array_equal(g.download(n), o.f[n]), n


@pytest.mark.parametrize("grid", GRIDS)
def test_saturation_adjust_matches_oracle(grid):
    p = config_params()
    st = make_state(*grid, seed=23)
    im = grid[0]
    # drive part of the column supersaturated / subsaturated with condensate, and make some
    # cells supercritical or superheated so every branch of clampAndFade runs
    st["c"] = st["c"] * 1.5
    st["cloud"][im // 2:, :, ::3] += 2e-3
    st["t"][1, :, ::5] = 700.0 / 273.15
    st["P_rain"][:, :, ::7] = 1e-5
    st["co2"][2, :, ::11] = 0.99
    o = OracleState(st, p)
    hits = o.saturation_adjust()
    with gpu_with(st, p) as g:
        g.SaturationAdjustment_run()
        for n in ("t", "c", "cloud", "ice", "gr", "S_c_c", "P_rain", "S_v"):
            assert relerr(g.download(n), o.f[n]) <= 1e-11, n
        assert g.report()["satadj_ceiling_hits"] == hits


@pytest.mark.parametrize("grid", GRIDS)
@pytest.mark.parametrize("set_water", [False, True])
def test_densities_matches_oracle(grid, set_water):
    p = config_params()
    st = make_state(*grid, seed=29)
    o = OracleState(st, p)
    o.densities(set_water_profile=set_water)
    with gpu_with(st, p) as g:
        g.densities(set_water_profile=set_water)
        for n in ("t", "p_stat", "r_humid", "r_dry", "c"):
            assert relerr(g.download(n), o.f[n]) <= 1e-11, n
        for n in ("t_top_init", "p_stat_landscape"):
            assert relerr(g.download_2d(n), o.f2[n]) <= 1e-11, n
        for n in ("rho_base", "dlnrho_dr"):
            assert relerr(g.download_profile(n), o.prof[n]) <= 1e-11, n


def test_cadence_loop_matches_oracle():
    """Ten model iterations at the reference cadence: RK4 every iteration, one pressure
    sweep every 4th, saturation adjustment + moist convection + densities every 2nd
    (run_3D_loop, cAtmosphereModel.cpp:1156-1509)."""
    p = config_params()
    grid = (11, 21, 41)
    st = make_state(*grid, seed=31)
    o = OracleState(st, p)
    with gpu_with(st, p) as g:
        for it in range(1, 11):
            br = min(1.0, it / 300.0)
            if it % 4 == 0:
                o.pressure_sweep(1, it)
                g.PressureSolverAtm_run(it)
            if it % 2 == 0:
                o.saturation_adjust()
                g.SaturationAdjustment_run()
                o.moist_convection(it)
                g.MoistConvection_run(it)
                o.densities()
                g.densities()
            o.rk4(dt=4e-5, buoyancy_ramp=br)
            g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, br)
            o.store_n_level()
            g.storeIntermediateData3D()
        for n in PROG + ["p_dyn", "p_stat", "r_humid"]:
            assert relerr(g.download(n), o.f[n]) <= 1e-10, n


@pytest.mark.parametrize("precision", [0, 1])
def test_fused_time_level_copy_equals_separate_copy(precision):
    """athad_step_scalars.store_n_level: the time-level copy written by the last RK4 stage
    (and the precipitation fluxes copied after it) is bit-identical to the RK4 step followed
    by storeIntermediateData3D, boundary cells included, and the following step starts
    from it."""
    p = config_params()
    p.precision = precision
    st = make_state(11, 21, 41, seed=29)
    rng = np.random.default_rng(29)
    st["P_rain"] = 1e-5 * rng.random(st["t"].shape)
    st["P_snow"] = 1e-5 * rng.random(st["t"].shape)
    with gpu_with(st, p) as a, gpu_with(st, p) as b:
        for it in range(3):
            a.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, 0.5)
            a.storeIntermediateData3D()
            b.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, 0.5, store_n_level=True)
        for n in PROG + [x + "n" for x in PROG] + ["P_rainn", "P_snown"]:
            assert np.array_equal(a.download(n), b.download(n)), n


@pytest.mark.parametrize("grid", GRIDS + [(4, 5, 5), (6, 7, 9)])
def test_pressure_boundaries_and_ceiling_bit_exact(grid):
    """The boundary passes (radial, pole, seam) and the |p| ceiling in the reference's order,
    with p far beyond the ceiling next to the seam, the poles and the lid, and non-finite
    values beside them: the seam average is formed from unclamped values and clamped after,
    a non-finite neighbour turns an extrapolation into NaN and the ceiling into 0.  The
    smallest grid the context accepts (4 x 5 x 5) included: there every interior cell is one
    the boundary passes read."""
    p = config_params()
    st = make_state(*grid, seed=17)
    im, jm, km = grid
    rng = np.random.default_rng(3)
    for n in ("aux_u", "aux_v", "aux_w"):
        st[n] = 1e-3 * rng.standard_normal(st["t"].shape)
    pd = 40.0 * rng.standard_normal(st["t"].shape)
    pd[2, 3, 2] = np.inf
    pd[im - 3, jm - 3, km - 3] = np.nan
    pd[2, 2, km // 2] = -np.inf
    st["p_dyn"] = pd
    for it in (4, 400):          # ceiling 10, then 3
        o = OracleState(st, p)
        o.pressure_sweep(n_sweeps=1, total_iter_count=it)
        with gpu_with(st, p) as g:
            g.PressureSolverAtm_run(total_iter_count=it, n_sweeps=1)
            a = g.download("p_dyn")
        assert np.array_equal(a, o.f["p_dyn"], equal_nan=True), it
        assert np.max(np.abs(a)) <= (10.0 if it <= 300 else 3.0)


def test_pressure_ceiling_skipped_only_when_nothing_reaches_it():
    """The ceiling pass ends early when no colour formed a value beyond the ceiling (every
    boundary value is then a copy or average of such values).  Interior values well inside
    the ceiling, and before the call values far beyond it and non-finite on the grid's edges
    (cells that no interior cell reads, so the sweep itself stays inside the ceiling): the
    boundary passes replace them, and the result is the oracle's bit for bit."""
    grid = (11, 21, 41)
    p = config_params()
    st = make_state(*grid, seed=23)
    im, jm, km = grid
    rng = np.random.default_rng(4)
    for n in ("aux_u", "aux_v", "aux_w"):
        st[n] = 1e-4 * rng.standard_normal(st["t"].shape)
    pd = 0.5 * rng.standard_normal(st["t"].shape)
    pd[0, 0, :] = 1e6
    pd[im - 1, jm - 1, :] = -1e6
    pd[:, 0, km - 1] = np.inf
    pd[0, :, 0] = np.nan
    st["p_dyn"] = pd
    o = OracleState(st, p)
    o.pressure_sweep(n_sweeps=1, total_iter_count=400)
    with gpu_with(st, p) as g:
        g.PressureSolverAtm_run(total_iter_count=400, n_sweeps=1)
        a = g.download("p_dyn")
    assert np.array_equal(a, o.f["p_dyn"], equal_nan=True)
    assert np.isfinite(a).all() and np.max(np.abs(a)) <= 3.0


@pytest.mark.parametrize("precision", [Precision.FP64, Precision.MIXED])
def test_report_counts_nonfinite_temperature_and_times_the_step(precision):
    """athad_get_report: the level mean of each RK4 step counts the non-finite cells of its
    input t; last_kernel_ms is the step's device time."""
    grid = (11, 21, 41)
    p = config_params()
    p.precision = int(precision)
    st = make_state(*grid, seed=11)
    with GpuAtmosphere(*grid, p) as g:
        g.upload_state(st)
        assert g.report()["last_kernel_ms"] == 0.0
        g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, 0.5)
        r = g.report()
        assert r["nonfinite_inputs"] == 0 and r["last_kernel_ms"] > 0.0
        t = st["t"].copy()
        t[3, 5, 7] = np.nan
        t[4, 10, 0] = np.inf
        t[9, 20, 40] = -np.inf
        g.upload("t", t)
        g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, 0.5)
        assert g.report()["nonfinite_inputs"] == 3
