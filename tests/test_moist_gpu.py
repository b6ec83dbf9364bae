"""Moist convection on the device against the oracle, and its mirror symmetry.

Tolerance: 1e-10 relative to the field's largest magnitude.  The kernel is compiled with
fused multiply-add and calls CUDA's exp/pow/sqrt/cbrt, so single operations differ from the
host in the last bit; the column recurrences carry that forward without amplifying it.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state, mirror
from athad_cond_b200._abi import config_params
from oracle_binding import OracleState

pytestmark = pytest.mark.gpu

MC_FIELDS = ["s", "s_u", "s_d", "M_u", "M_d", "q_v_u", "q_c_u", "q_v_d", "u_u", "v_u", "w_u",
             "u_d", "v_d", "w_d", "E_u", "D_u", "E_d", "D_d", "c_u", "e_l", "e_d", "e_p", "g_p",
             "P_conv", "CloudBase", "LevelFreeSinking", "Deep_beg", "Deep_end",
             "MC_t", "MC_q", "MC_v", "MC_w"]
ANTI = {"v_u", "v_d", "MC_v"}


def convective_state(grid, seed, symmetric=False):
    """A synthetic state moist enough near the surface to trigger the scheme."""
    st = make_state(*grid, seed=seed, symmetric=symmetric)
    im = grid[0]
    st["c"][: im // 3] *= 1.6
    st["Evaporation"] = np.full(grid[1:], 20.0)
    st["Q_sensible_2D"] = np.zeros(grid[1:])
    return st


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("grid", [(11, 21, 41), (21, 91, 181)])
def test_moist_convection_matches_oracle(grid):
    p = config_params()
    st = convective_state(grid, seed=37)
    o = OracleState(st, p)
    with GpuAtmosphere(*grid, params=p) as g:
        g.upload_state(st)
        for it in (2, 4):
            o.moist_convection(it)
            g.MoistConvection_run(it)
            for n in MC_FIELDS:
                e = relerr(g.download(n), o.f[n])
                assert e <= 1e-10, (it, n, e)
        assert np.max(np.abs(o.f["M_u"])) > 0.0   # the scheme did fire


def test_moist_convection_mirror_symmetric():
    p = config_params()
    grid = (21, 91, 181)
    st = convective_state(grid, seed=41, symmetric=True)
    with GpuAtmosphere(*grid, params=p) as g:
        g.upload_state(st)
        g.MoistConvection_run(2)
        g.MoistConvection_run(4)
        for n in MC_FIELDS:
            a = g.download(n)
            assert np.array_equal(a, mirror(a, n in ANTI)), n
