"""athad_multilayer_radiation (MultiLayerRadiation::run) and athad_radiative_heating
(radiation mode 2) on the device against the oracle, which is pinned bit for bit against
the reference (test_pin_reference.py).

Tolerance: 1e-12 of each field's largest magnitude (the sweeps call pow and exp, whose last
bit differs between CUDA and glibc).  A mirror-symmetric state stays mirror-symmetric.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state, mirror
from athad_cond_b200._abi import config_params
from oracle_binding import OracleState, update_skin_temperature

pytestmark = pytest.mark.gpu


def state(grid, seed, symmetric=False):
    st = make_state(*grid, seed=seed, symmetric=symmetric)
    im, jm, km = grid
    rng = np.random.default_rng(seed)
    jh = (jm + 1) // 2
    for n in ("cloud", "ice"):
        a = 2e-4 * rng.random((im, jh if symmetric else jm, km))
        if symmetric:
            a = np.concatenate([a, a[:, :jm - jh][:, ::-1]], axis=1)
        st[n] = a
    return st


def close(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("grid", [(11, 21, 41), (41, 181, 361)])
@pytest.mark.parametrize("heating", [False, True])
def test_radiation_matches_oracle(grid, heating):
    st = state(grid, 81)
    o = OracleState(st, config_params())
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        if heating:
            g.radiative_heating(0.05)
            o.radiative_heating(0.05)
        else:
            g.multilayer_radiation()
            o.multilayer_radiation()
        for n in ("t", "radiation", "epsilon"):
            assert close(g.download(n), o.f[n]) <= 1e-12, n
        for n in ("epsilon_2D", "albedo"):
            assert close(g.download_2d(n), o.f2[n]) <= 1e-12, n
    # the sweeps moved the air layers and the clouds raised the albedo
    assert np.any(o.f["t"] != st["t"])
    assert np.all(o.f2["albedo"] > config_params().albedo_surface)


def test_radiation_keeps_mirror_symmetry():
    grid = (21, 91, 181)
    st = state(grid, 83, symmetric=True)
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.radiative_heating(0.05)
        for n in ("t", "radiation", "epsilon"):
            a = g.download(n)
            assert np.array_equal(a, mirror(a, False)), n
        for n in ("epsilon_2D", "albedo"):
            a = g.download_2d(n)
            assert np.array_equal(a, a[::-1, :]), n


def test_skin_temperature_matches_oracle():
    """athad_update_skin_temperature (cAtmosphereModel::updateSkinTemperature): the new t_skin
    identical to the oracle's, twice in a row from the albedo on the device; t_skin_relax = 0
    leaves it."""
    grid = (11, 21, 41)
    rng = np.random.default_rng(151)
    albedo = 0.05 + 0.5 * rng.random(grid[1:])
    p = config_params()
    with GpuAtmosphere(*grid, p) as g:
        g.upload_2d("albedo", albedo)
        t = p.t_skin
        assert g.update_skin_temperature(0.0) == t
        for _ in range(2):
            want = update_skin_temperature(p, albedo, t, 0.25)
            t = g.update_skin_temperature(0.25)
            assert t == want and t != p.t_skin
