"""The mixed-precision RK4 step (athad_params.precision = MIXED) on the device.

Its reference is the FP64 oracle (the plain GPU form equals the oracle to 1e-12 per step,
test_parity_gpu.py).  Stated tolerances, max |mixed - oracle| / max |oracle| per field:
  * one RK4 step: 1e-8 (the FP32 right-hand side perturbs only the dt-sized increment);
  * 100 RK4 steps on 21 x 91 x 181: 1e-6;
  * 1000 RK4 steps on 41 x 181 x 361 against the FP64 GPU form: 1e-5 for every
    prognostic field (the accuracy bar the mixed form is held to for the dynamics);
  * 300 whole model iterations from the reference's initial state on 41 x 181 x 361
    against the FP64 form: 1e-5 for every prognostic field, p_stat and r_humid.
The column physics (pressure, saturation adjustment, moist convection, densities) is FP64
in both forms and identical between them from the same state.
Mirror symmetry is exact (bit for bit) for the mixed form too, as for the FP64 form.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state, mirror
from athad_cond_b200._abi import Precision, config_params
from oracle_binding import OracleState

pytestmark = pytest.mark.gpu

PROG = ["t", "u", "v", "w", "c", "cloud", "ice", "gr", "co2", "tke", "dis"]
ANTI = {"v", "vn", "aux_v", "MC_v"}


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def mixed(state, params=None):
    p = params if params is not None else config_params()
    p.precision = int(Precision.MIXED)
    im, jm, km = state["t"].shape
    g = GpuAtmosphere(im, jm, km, p)
    g.upload_state(state)
    return g


@pytest.mark.parametrize("grid", [(11, 21, 41), (21, 91, 181)])
def test_mixed_one_step_against_oracle(grid):
    st = make_state(*grid, seed=7)
    o = OracleState(st, config_params())
    o.rk4(dt=4e-5, buoyancy_ramp=0.5)
    with mixed(st) as g:
        g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, 0.5)
        for n in PROG:
            assert relerr(g.download(n), o.f[n]) <= 1e-8, n
        for n in ("aux_u", "aux_v", "aux_w"):
            assert relerr(g.download(n), o.f[n]) <= 1e-4, n


def test_mixed_hundred_steps_against_oracle():
    grid = (21, 91, 181)
    st = make_state(*grid, seed=9)
    o = OracleState(st, config_params())
    with mixed(st) as g:
        for it in range(1, 101):
            o.rk4(dt=4e-5, buoyancy_ramp=min(1.0, it / 300.0))
            o.store_n_level()
            g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, min(1.0, it / 300.0))
            g.storeIntermediateData3D()
        for n in PROG:
            assert relerr(g.download(n), o.f[n]) <= 1e-6, n


def test_mixed_thousand_steps_against_fp64_form():
    grid = (41, 181, 361)
    st = make_state(*grid, seed=20261203)
    p64 = config_params()
    g64 = GpuAtmosphere(*grid, p64)
    g64.upload_state(st)
    with mixed(st) as gm:
        for it in range(1, 1001):
            for g in (g64, gm):
                g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, min(1.0, it / 300.0))
                g.storeIntermediateData3D()
        for n in PROG:
            a, b = gm.download(n), g64.download(n)
            assert np.isfinite(a).all(), n
            assert relerr(a, b) <= 1e-5, n
    g64.close()


@pytest.mark.parametrize("grid", [(11, 21, 41), (21, 91, 181)])
def test_mixed_mirror_symmetry_exact(grid):
    st = make_state(*grid, seed=11, symmetric=True)
    with mixed(st) as g:
        for it in range(3):
            g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, 0.2)
            g.storeIntermediateData3D()
        for n in PROG + ["aux_u", "aux_v", "aux_w"]:
            a = g.download(n)
            assert np.array_equal(a, mirror(a, n in ANTI)), n


def test_mixed_form_keeps_pressure_moist_convection_and_densities_fp64():
    """The pressure sweep, saturation adjustment, moist convection and densities are FP64
    in both forms: from the same state they give identical results."""
    grid = (11, 21, 41)
    st = make_state(*grid, seed=5)
    st["Evaporation"] = np.full(grid[1:], 20.0)
    g64 = GpuAtmosphere(*grid, config_params())
    g64.upload_state(st)
    with mixed(st) as gm:
        for g in (g64, gm):
            g.PressureSolverAtm_run(total_iter_count=4)
            g.SaturationAdjustment_run()
            g.MoistConvection_run(2)
            g.densities()
        for n in ("p_dyn", "MC_t", "MC_q", "p_stat", "r_humid", "t", "c", "cloud", "ice", "S_c_c"):
            assert np.array_equal(gm.download(n), g64.download(n)), n
    g64.close()


def test_mixed_model_iterations_within_1e5_of_fp64():
    """300 model iterations at the reference cadence (pressure sweep every 4th iteration,
    saturation adjustment, moist convection and densities every 2nd, the RK4 step every
    one) from the reference's initial state on 41 x 181 x 361, mixed against FP64: every
    prognostic field and the diagnosed pressure and humidity within 1e-5 of the field's
    largest magnitude, in every cell (measured: 1e-9 and below)."""
    grid = (41, 181, 361)

    def ctx(prec):
        p = config_params()
        p.precision = int(prec)
        g = GpuAtmosphere(*grid, p)
        g.initial_state()
        return g

    g64, gm = ctx(Precision.FP64), ctx(Precision.MIXED)
    try:
        for it in range(1, 301):
            for g in (g64, gm):
                if it % 4 == 0:
                    g.PressureSolverAtm_run(total_iter_count=it)
                if it % 2 == 0:
                    g.SaturationAdjustment_run()
                    g.MoistConvection_run(it)
                    g.densities()
                g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, min(1.0, it / 300.0), store_n_level=True)
        for n in PROG + ["p_dyn", "p_stat", "r_humid"]:
            a, b = gm.download(n), g64.download(n)
            assert np.isfinite(a).all(), n
            assert relerr(a, b) <= 1e-5, (n, relerr(a, b))
    finally:
        g64.close()
        gm.close()


