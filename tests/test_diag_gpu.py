"""Diagnostics and checkpoints on the device.

athad_min_max (searchMinMax_3D, MinMax_Atm.cpp:51-109): the extreme finite values and the
first cell in (i, j, k) order holding each, identical to the oracle's serial scan, with
non-finite values, ties and an all-non-finite field planted.  athad_checkpoint_begin /
athad_checkpoint_wait: the host copy is the state at the call even when later calls change
the fields before the copy finishes.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state
from athad_cond_b200._abi import config_params
from oracle_binding import OracleState

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("grid", [(11, 21, 41), (41, 181, 361)])
def test_min_max_matches_serial_scan(grid):
    st = make_state(*grid, seed=101)
    im, jm, km = grid
    u = st["u"].copy()
    u[3, 5, 7] = np.nan
    u[1, 2, 3] = np.inf
    top = np.nanmax(np.where(np.isfinite(u), u, -np.inf)) + 1.0
    u[4, 9, 11] = top          # tie: two cells hold the maximum, the first one wins
    u[6, 2, 1] = top
    st["u"] = u
    st["v"] = np.full(grid, np.nan)          # no finite value: 0 at (0, 0, 0)
    st["w"] = np.round(st["w"], 1)           # many ties
    o = OracleState(st, config_params())
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        for n in ("u", "v", "w", "t", "c"):
            a, b = g.min_max(n), o.min_max(n)
            assert a == b, (n, a, b)
    assert o.min_max("u")["at_max"] == (4, 9, 11)
    assert o.min_max("v") == {"max": 0.0, "min": 0.0, "at_max": (0, 0, 0), "at_min": (0, 0, 0)}


def test_checkpoint_is_the_state_at_the_call():
    grid = (21, 91, 181)
    st = make_state(*grid, seed=103)
    names = ["t", "u", "v", "w", "c", "p_dyn"]
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, 0.5, store_n_level=True)
        want = {n: g.download(n) for n in names}
        host = g.checkpoint_begin(names)
        for _ in range(3):                   # change every checkpointed field meanwhile
            g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, 0.5, store_n_level=True)
            g.PressureSolverAtm_run(total_iter_count=8)
        g.checkpoint_wait()
        for n in names:
            assert np.array_equal(host[n], want[n]), n
        assert not np.array_equal(g.download("t"), want["t"])
        # a second, larger checkpoint reuses the side stream and grows the snapshot
        host2 = g.checkpoint_begin(names + ["tke", "dis"])
        g.checkpoint_wait()
        for n in names + ["tke", "dis"]:
            assert np.array_equal(host2[n], g.download(n)), n
