"""Diagnostics and checkpoints on the device.

athad_min_max (searchMinMax_3D, MinMax_Atm.cpp:51-109): the extreme finite values and the
first cell in (i, j, k) order holding each, identical to the oracle's serial scan, with
non-finite values, ties and an all-non-finite field planted.  athad_checkpoint_begin /
athad_checkpoint_wait: the host copy is the state at the call even when later calls change
the fields before the copy finishes.  athad_find_residuum (findResiduumAtm, UtilsAtm.h:70-220):
the residuum, its cell (smallest (i, j, k) on equal values) and the counts identical to the
oracle's, the average within 1e-12.  athad_stand_atm_dew_point (standAtm_DewPoint_HumidRel,
ThermoAtm.h:400-516): TempStand bit for bit; the dew point (a 60-step bisection of the IAPWS
curve) and the relative humidity within 1e-12 of the field's largest magnitude (CUDA's exp,
log and sqrt against glibc's pow and exp), mirror-symmetric bit for bit.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state, mirror
from athad_cond_b200._abi import config_params
from athad_cond_b200.context import AthadError
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


@pytest.mark.parametrize("grid", [(11, 21, 41), (21, 91, 181), (41, 181, 361)])
def test_find_residuum_matches_oracle(grid):
    st = make_state(*grid, seed=107)
    im, jm, km = grid
    if im >= 21:
        u = st["u"].copy()
        u[12, jm // 3, km // 2] = np.nan     # two non-finite residuals, i = 11 and 13
        st["u"] = u
    o = OracleState(st, config_params())
    want = o.find_residuum()
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        got = g.find_residuum()
        again = g.find_residuum()
    for key in ("residuum", "at", "n_cells", "n_nonfinite", "first_nonfinite"):
        assert got[key] == want[key], (key, got[key], want[key])
    assert abs(got["avg_abs"] - want["avg_abs"]) <= 1e-12 * max(want["avg_abs"], 1e-300)
    assert got["residuum_prev"] == 1e-5 and again["residuum_prev"] == got["residuum"]
    if im < 12:
        assert got["n_cells"] == 0 and got["residuum"] == 0.0 and got["at"] == (0, 0, 0)
    else:
        assert got["n_nonfinite"] == 2 and got["first_nonfinite"] == (11, jm // 3, km // 2)


def test_find_residuum_ties_take_the_smallest_cell():
    grid = (21, 91, 181)
    st = make_state(*grid, seed=109)
    u = np.zeros(grid)
    u[16, 30, 120] = 1.0                     # equal residuals at (15, 30, 120) and (15, 50, 60)
    u[16, 50, 60] = 1.0
    st.update(u=u, v=np.zeros(grid), w=np.zeros(grid))
    o = OracleState(st, config_params())
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        got = g.find_residuum()
    assert got["at"] == o.find_residuum()["at"] == (15, 30, 120)


def tropopause(im, jm):
    """A mirror-symmetric tropopause level per row, high at the equator, low at the poles."""
    the = np.linspace(0.0, np.pi, jm)
    lev = np.round((im - 1) * (0.25 + 0.5 * np.sin(the)))
    return (lev + lev[::-1]) / 2 // 1


def equator_rule(layers):
    jm = len(layers)
    return [int(layers[j - 1] if j == (jm - 1) // 2 else layers[j]) for j in range(jm)]


@pytest.mark.parametrize("grid", [(11, 21, 41), (41, 181, 361)])
def test_stand_atm_dew_point_matches_oracle(grid):
    im, jm, km = grid
    st = make_state(*grid, seed=113)
    t, c = st["t"].copy(), st["c"].copy()
    t[1:3, 2:4, 5:9] = 700.0 / 273.15        # supercritical: no saturation state
    c[4, 3:6, 10:14] = 0.0                   # no vapour
    st.update(t=t, c=c)
    layers = tropopause(im, jm)
    o = OracleState(st, config_params())
    o.stand_atm_dew_point(equator_rule(layers))
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        with pytest.raises(AthadError):
            g.stand_atm_dew_point()          # the tropopause levels are not set yet
        bad = layers.copy()
        bad[3] = im
        with pytest.raises(AthadError):
            g.set_tropopause_layers(bad)
        g.set_tropopause_layers(layers)
        g.stand_atm_dew_point()
        assert np.array_equal(g.download("TempStand"), o.f["TempStand"])
        for n in ("TempDewPoint", "HumidityRel"):
            a, b = g.download(n), o.f[n]
            e = float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
            assert e <= 1e-12, (n, e)
        hr = g.download("HumidityRel")
        assert np.all(hr[1:3, 2:4, 5:9] == -1.0) and np.all(hr[4, 3:6, 10:14] == 0.0)


def test_stand_atm_dew_point_mirror_symmetric():
    grid = (21, 91, 181)
    im, jm, km = grid
    st = make_state(*grid, seed=127, symmetric=True)
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.set_tropopause_layers(tropopause(im, jm))
        g.stand_atm_dew_point()
        for n in ("TempStand", "TempDewPoint", "HumidityRel"):
            a = g.download(n)
            assert np.array_equal(a, mirror(a, False)), n


def test_download_profile_async_equals_the_waiting_download():
    """athad_download_profile_async into page-locked memory: after the stream has passed the
    copy the host array holds what athad_download_profile returns; a kernel enqueued after
    the call does not change it."""
    import ctypes
    import torch
    from athad_cond_b200._abi import PROFILE
    grid = (11, 21, 41)
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(make_state(*grid, seed=5))
        g.computeLevelMeanTemperature()
        want = g.download_profile("t_ref_level")
        host = torch.full((grid[0],), -1.0, dtype=torch.float64).pin_memory()
        ptr = ctypes.cast(host.data_ptr(), ctypes.POINTER(ctypes.c_double))
        g._check(g.lib.athad_download_profile_async(g._h, PROFILE["t_ref_level"], ptr, grid[0]))
        g.fill("t", 1.0)
        g.computeLevelMeanTemperature()
        g.synchronize()
        assert np.array_equal(host.numpy(), want)
        assert not np.array_equal(g.download_profile("t_ref_level"), want)
        with pytest.raises(AthadError):
            g._check(g.lib.athad_download_profile_async(g._h, PROFILE["t_ref_level"], ptr, grid[0] + 1))
