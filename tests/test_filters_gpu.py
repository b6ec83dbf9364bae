"""The smoothing filters on the device against the oracle (pinned bit for bit against the
reference in test_pin_reference.py): athad_post_rk4_filters (polar zonal filter of u, v, w;
radial Shapiro filters) and athad_damp_wiggles.  Tolerance: bit-identical (1-2-1 and
4th-order sums in the oracle's order, no fused multiply-add; damp_wiggles' meridional pass
adds the two neighbours first, the oracle's mirror-exact form).  Both filters keep a
mirror-symmetric state mirror-symmetric.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state, mirror
from athad_cond_b200._abi import config_params
from oracle_binding import OracleState

pytestmark = pytest.mark.gpu

GRIDS = [(11, 21, 41), (21, 91, 181), (41, 181, 361)]


def rough(grid, seed, symmetric=False):
    """The synthetic state plus grid-scale noise on the filtered fields."""
    st = make_state(*grid, seed=seed, symmetric=symmetric)
    if not symmetric:
        rng = np.random.default_rng(seed)
        for n in ("u", "v", "w", "t", "c", "cloud", "ice"):
            st[n] = st[n] + 1e-3 * np.abs(st[n]).max() * rng.standard_normal(grid)
    return st


@pytest.mark.parametrize("grid", GRIDS)
def test_post_rk4_filters_bit_exact(grid):
    st = rough(grid, 41)
    o = OracleState(st, config_params())
    o.post_rk4_filters()
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.post_rk4_filters()
        for n in ("u", "v", "w", "t"):
            a = g.download(n)
            assert np.array_equal(a, o.f[n]), (n, float(np.max(np.abs(a - o.f[n]))))


@pytest.mark.parametrize("grid", GRIDS[:2])
def test_damp_wiggles_bit_exact(grid):
    st = rough(grid, 43)
    o = OracleState(st, config_params())
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        for n in ("t", "ice", "c", "cloud"):
            o.damp_wiggles(n)
            g.damp_wiggles(n)
        for n in ("t", "ice", "c", "cloud", "u"):
            a = g.download(n)
            assert np.array_equal(a, o.f[n]), (n, float(np.max(np.abs(a - o.f[n]))))


def test_filters_keep_mirror_symmetry():
    grid = (21, 91, 181)
    st = rough(grid, 47, symmetric=True)
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.post_rk4_filters()
        g.damp_wiggles("t")
        for n, anti in (("u", False), ("v", True), ("w", False), ("t", False)):
            a = g.download(n)
            assert np.array_equal(a, mirror(a, anti)), n
