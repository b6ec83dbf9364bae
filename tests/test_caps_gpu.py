"""athad_moist_caps (precipitationSum and the source / condensate caps) and
athad_vapour_ceiling on the device against the oracle: fields bit-identical (comparisons,
copies and one product per cell); the ceiling's sums within 1e-12 (a fixed-order
reduction against the oracle's serial sum)."""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state, mirror
from athad_cond_b200._abi import config_params
from oracle_binding import OracleState

pytestmark = pytest.mark.gpu

FIELDS = ["c", "cloud", "ice", "Precipitation", "S_v", "S_c", "S_i", "S_r", "S_s", "S_g", "S_c_c"]


def state(grid, seed, symmetric=False):
    """The synthetic state with out-of-range sources, condensate and vapour planted: NaN/Inf,
    values beyond the caps, cloud + ice above cloud_cap, c above 1 - co2 and below 0."""
    st = make_state(*grid, seed=seed, symmetric=symmetric)
    im, jm, km = grid
    rng = np.random.default_rng(seed)
    jh = (jm + 1) // 2

    def field(scale, offset=0.0):
        a = offset + scale * rng.standard_normal((im, jh if symmetric else jm, km))
        if symmetric:
            a = np.concatenate([a, a[:, :jm - jh][:, ::-1]], axis=1)
        return a
    for n in ("P_rain", "P_snow", "P_graupel", "P_conv"):
        st[n] = np.abs(field(1e-4))
    for n in ("S_v", "S_c", "S_i", "S_r", "S_s", "S_g", "S_c_c"):
        a = field(2e-3)
        a[:, :, 3] = np.nan
        a[:, :, 5] = np.inf
        st[n] = a
    st["cloud"] = np.abs(field(0.05))
    st["ice"] = field(0.03)
    st["c"] = st["c"] + field(0.3)
    st["c"][:, :, 7] = np.nan
    return st


@pytest.mark.parametrize("grid", [(11, 21, 41), (41, 181, 361)])
def test_caps_and_ceiling_match_oracle(grid):
    st = state(grid, 91)
    o = OracleState(st, config_params())
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        rg = g.vapour_ceiling()      # first, so that it finds vapour above its ceiling
        g.moist_caps()
        ro = o.vapour_ceiling()
        o.moist_caps()
        for n in FIELDS:
            a = g.download(n)
            assert np.array_equal(a, o.f[n]), n
        assert rg["n_ceiling"] == ro["n_ceiling"] > 0
        for key in ("q_clipped", "w_air"):
            assert abs(rg[key] - ro[key]) <= 1e-12 * abs(ro[key]), key


def test_caps_keep_mirror_symmetry():
    grid = (21, 91, 181)
    st = state(grid, 93, symmetric=True)
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.vapour_ceiling()
        g.moist_caps()
        for n in FIELDS:
            a = g.download(n)
            assert np.array_equal(a, mirror(a, False)), n
