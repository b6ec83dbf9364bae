"""The device path on the reference's own initial state at its native grid (61 x 181 x 361).

The reference (built into oracle/_ref) builds its initial state; the device path and the
oracle (mirror-symmetric semantics) then run every hot-path function on it and must agree
within the parity tolerances.  The difference between the device path and the reference
itself is reported: it is the in-place vs Jacobi RK4 sweep and the mirror-symmetric
rounding, not an error.
"""
import os

import numpy as np
import pytest

import ref_binding
from athad_cond_b200 import GpuAtmosphere
from athad_cond_b200._abi import FIELD_NAMES, config_params
from oracle_binding import OracleState

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_binding.available("pin"), reason="reference not built")]

PROG = ["t", "u", "v", "w", "c", "cloud", "ice", "gr", "co2", "tke", "dis"]


@pytest.fixture(scope="module")
def ref_state():
    cwd = os.getcwd()
    os.chdir(os.environ.get("TMPDIR", "/tmp"))
    try:
        R = ref_binding.Reference("pin", threads=max(1, min(8, os.cpu_count() or 1)))
        R.init_state()
        st = {n: R.get(n) for n in FIELD_NAMES}
        for n in ("t_top_init", "p_stat_landscape", "Evaporation", "Q_sensible_2D"):
            st[n] = R.get2(n)
        yield R, st
        R.close()
    finally:
        os.chdir(cwd)


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_iteration_on_reference_state(ref_state):
    R, st = ref_state
    p = config_params()
    o = OracleState(st, p)
    with GpuAtmosphere(*R.shape, params=p) as g:
        g.upload_state(st)
        # one moist iteration of run_3D_loop's hot path
        o.saturation_adjust(); g.SaturationAdjustment_run()
        o.moist_convection(2); g.MoistConvection_run(2)
        o.densities(); g.densities()
        o.rk4(dt=4e-5, buoyancy_ramp=2 / 300.0); g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, 2 / 300.0)
        o.pressure_sweep(1, 4); g.PressureSolverAtm_run(4)
        for n in PROG + ["p_dyn", "p_stat", "r_humid", "MC_t", "MC_q", "MC_v", "MC_w", "aux_u"]:
            e = relerr(g.download(n), o.f[n])
            assert e <= 1e-10, (n, e)


def test_rk4_difference_to_reference_is_the_sweep_order(ref_state):
    """Device (Jacobi, mirror-symmetric) vs the reference (in-place): the relative difference
    after one RK4 step stays far below the step's own change."""
    R, st = ref_state
    for n in FIELD_NAMES:
        R.set(n, st[n])
    R.set_scalars(4e-5, 1.0, 0.3, 90, 90)
    R.lib.ref_rk4(R.h)
    p = config_params()
    with GpuAtmosphere(*R.shape, params=p) as g:
        g.upload_state(st)
        g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, 0.3)
        for n in ["t", "u", "v", "w", "tke", "dis"]:
            a, b = g.download(n), R.get(n)
            diff = np.max(np.abs(a - b))
            step = np.max(np.abs(b - st[n]))
            assert diff <= 1e-2 * step, (n, diff, step)
