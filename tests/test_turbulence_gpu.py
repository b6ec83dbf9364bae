"""athad_turbulence_run (TurbulenceAtm::run: compute_vel_star, compute_sources with the
k-epsilon, k-omega or k-omega SST closure, clamp_nue) on the device against the oracle in
its order-free form; the oracle's reference form is pinned bit for bit against the
reference (test_pin_reference.py).

Tolerances: vel_star, tke, dis and prod bit-identical (square roots, divisions and the
floors round the same on both sides); nue, tke_source and dis_source within 1e-12 of the
field's largest magnitude (the closures call exp, pow and tanh, whose last bit differs
between CUDA and glibc).  A mirror-symmetric state stays mirror-symmetric.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state, mirror
from athad_cond_b200._abi import Turb, config_params
from oracle_binding import OracleState

pytestmark = pytest.mark.gpu

EXACT = ("tke", "dis", "prod")
CLOSE = ("nue", "tke_source", "dis_source")


def state(grid, seed, symmetric=False):
    """The synthetic state with tke pulled below its background floor in a band of rows and
    a few negative cells, so that both floors bind."""
    st = make_state(*grid, seed=seed, symmetric=symmetric)
    im, jm, km = grid
    low = np.zeros(grid, dtype=bool)
    low[:, jm // 3: jm // 3 + 3, :] = True
    neg = np.zeros(grid, dtype=bool)
    neg[2:4, :, km // 4: km // 4 + 5] = True
    if symmetric:
        low |= low[:, ::-1, :]
    tke = np.where(low, 0.01 * st["tke"], st["tke"])
    st["tke"] = np.where(neg, -1e-4, tke)
    return st


@pytest.mark.parametrize("grid", [(11, 21, 41), (21, 91, 181)])
@pytest.mark.parametrize("turb", [Turb.K_EPSILON, Turb.K_OMEGA, Turb.K_OMEGA_SST])
def test_turbulence_run_matches_oracle(grid, turb):
    p = config_params()
    p.turb_model = int(turb)
    st = state(grid, 61)
    o = OracleState(st, p)
    o.turbulence_run(compat=0)
    with GpuAtmosphere(*grid, p) as g:
        g.upload_state(st)
        g.turbulence_run()
        assert np.array_equal(g.download_2d("vel_star"), o.f2["vel_star"])
        for n in EXACT:
            a = g.download(n)
            assert np.array_equal(a, o.f[n]), (n, float(np.max(np.abs(a - o.f[n]))))
        for n in CLOSE:
            a, b = g.download(n), o.f[n]
            e = float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
            assert e <= 1e-12, (n, e)
        # the floors bound somewhere
        assert np.any(o.f["tke"] != st["tke"])


def test_turbulence_run_keeps_mirror_symmetry():
    grid = (21, 91, 181)
    st = state(grid, 67, symmetric=True)
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.turbulence_run()
        for n in EXACT + CLOSE:
            a = g.download(n)
            assert np.array_equal(a, mirror(a, False)), n
        vs = g.download_2d("vel_star")
        assert np.array_equal(vs, vs[::-1, :])
