"""athad_two_cat_ice_scheme (TwoCatIceScheme::run) on the device against the oracle, which is
pinned bit for bit against the reference (test_pin_reference.py).

Tolerance: 1e-10 of each field's largest magnitude.  The scheme forms a dozen fractional
powers in every cell and the saturation curves (the device from exp/log/cbrt/sqrt, the
oracle from glibc's pow/exp); the differences
stay at rounding level because no threshold of the scheme sits on a rounding edge in these
states.  A mirror-symmetric state stays mirror-symmetric, bit for bit.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state, mirror
from athad_cond_b200._abi import config_params
from oracle_binding import OracleState

pytestmark = pytest.mark.gpu

OUT = ["t", "c", "cloud", "ice", "gr", "P_rain", "P_snow", "Precipitation", "P_rainn", "P_snown",
       "S_v", "S_c", "S_i", "S_r", "S_s", "S_c_c"]


def state(grid, seed, symmetric=False):
    """The synthetic state after the saturation adjustment (condensate, S_c_c), with falling
    rain and snow of the previous iteration and a cold upper band where ice processes run."""
    st = make_state(*grid, seed=seed, symmetric=symmetric)
    im, jm, km = grid
    rng = np.random.default_rng(seed)
    jh = (jm + 1) // 2
    shape = (im, jh if symmetric else jm, km)

    def field(scale):
        a = scale * rng.random(shape)
        if symmetric:
            a = np.concatenate([a, a[:, :jm - jh][:, ::-1]], axis=1)
        return a
    st["P_rainn"] = field(2e-4)
    st["P_snown"] = field(2e-4)
    st["S_c_c"] = field(1e-6) - 5e-7
    st["ice"] = field(1e-4)
    st["cloud"] = st["cloud"] + field(1e-3)
    return st


@pytest.mark.parametrize("grid", [(11, 21, 41), (21, 91, 181), (41, 181, 361)])
def test_two_cat_ice_scheme_matches_oracle(grid):
    st = state(grid, 71)
    o = OracleState(st, config_params())
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.two_cat_ice_scheme()
        o.two_cat_ice_scheme()
        for n in OUT:
            a, b = g.download(n), o.f[n]
            e = float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
            assert e <= 1e-10, (n, e)
    # the scheme did something: fluxes and sources in most cells
    assert np.count_nonzero(o.f["S_r"]) > o.f["S_r"].size // 4


def test_two_cat_ice_scheme_keeps_mirror_symmetry():
    grid = (21, 91, 181)
    st = state(grid, 73, symmetric=True)
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.two_cat_ice_scheme()
        for n in OUT:
            a = g.download(n)
            assert np.array_equal(a, mirror(a, False)), n
