"""athad_boundary_conditions (bcRadius, apply_wall_bc, bcTheta, bcPhi) on the device against
the oracle, which is pinned bit for bit against the reference (test_pin_reference.py).

Tolerance: bit-identical.  Every formula is a copy, an average or a short sum in the
reference's order, and the kernels round each operation separately.  Also: the boundary
conditions keep a mirror-symmetric state mirror-symmetric.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state, mirror
from athad_cond_b200._abi import FIELD_NAMES, Turb, config_params
from oracle_binding import OracleState

pytestmark = pytest.mark.gpu

ANTI = {"v", "vn", "aux_v", "MC_v", "v_u", "v_d"}


def state(grid, seed, symmetric=False):
    st = make_state(*grid, seed=seed, symmetric=symmetric)
    rng = np.random.default_rng(seed)
    im, jm, km = grid
    jh = (jm + 1) // 2
    # moist-convection fields the boundary conditions extrapolate, which the synthetic
    # state leaves at zero
    for n in ("s", "s_u", "q_v_u", "q_c_u", "u_u", "w_u", "M_u", "c_u", "e_d", "P_conv", "r_dry"):
        a = rng.standard_normal((im, jh if symmetric else jm, km)) * 1e-3
        if symmetric:
            a = np.concatenate([a, a[:, :jm - jh][:, ::-1]], axis=1)
        st[n] = a
    vs = 0.05 + 0.3 * rng.random((jh if symmetric else jm, km))
    tt = st["t"][-1].copy()
    if symmetric:
        vs = np.concatenate([vs, vs[:jm - jh][::-1]], axis=0)
    st["vel_star"] = vs
    st["t_top_init"] = tt
    return st


@pytest.mark.parametrize("grid", [(11, 21, 41), (21, 91, 181)])
@pytest.mark.parametrize("turb", [Turb.K_EPSILON, Turb.K_OMEGA, Turb.K_OMEGA_SST])
def test_boundary_conditions_match_oracle_bit_exact(grid, turb):
    p = config_params()
    p.turb_model = int(turb)
    st = state(grid, 17)
    o = OracleState(st, p)
    o.boundary_conditions()
    with GpuAtmosphere(*grid, p) as g:
        g.upload_state(st)
        g.boundary_conditions()
        for n in FIELD_NAMES:
            a = g.download(n)
            assert np.array_equal(a, o.f[n]), (n, float(np.max(np.abs(a - o.f[n]))))


def test_boundary_conditions_keep_mirror_symmetry():
    grid = (11, 21, 41)
    st = state(grid, 23, symmetric=True)
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.boundary_conditions()
        for n in FIELD_NAMES:
            a = g.download(n)
            assert np.array_equal(a, mirror(a, n in ANTI)), n
