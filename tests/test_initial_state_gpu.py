"""The reference's deterministic initial state built on the device (athad_initial_state,
cAtmosphereModel::RunTimeSlice for Ma = 0, cAtmosphereModel.cpp:468-668) against the
oracle's restatement of the same sequence (or_init_state, the device semantics), which
tests/test_pin_initial_state.py pins bit for bit against the reference at its own grid.

Every field, 2-D field and profile of the state is compared, relative to the field's
largest magnitude.  The tolerance is 1e-9: the sequence runs CUDA's exp/log/pow against
glibc's through the saturation adjustment's Newton iteration, the moist convection and
200 projection sweeps.  The state is exactly north-south mirror symmetric (v-type fields
antisymmetric) on every grid.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, config_init
from athad_cond_b200._abi import FIELD_NAMES, FIELD2D_NAMES, PROFILE_NAMES, Params, config_params
from oracle_binding import OracleState

pytestmark = pytest.mark.gpu

TOL = 1e-9
ANTISYMMETRIC = {"v", "vn", "aux_v", "MC_v", "v_u", "v_d"}
# outputs the sequence leaves as resetArrays set them or that only the omitted diagnostics
# write; compared all the same (they must be the reset values on both sides)


def rel_err(a, b):
    den = float(np.max(np.abs(b)))
    d = float(np.max(np.abs(a - b)))
    return d / den if den > 0 else d


def device_state(grid, p: Params, cfg=None):
    with GpuAtmosphere(*grid, p) as g:
        g.initial_state(cfg)
        f = {n: g.download(n) for n in FIELD_NAMES}
        f2 = {n: g.download_2d(n) for n in FIELD2D_NAMES}
        pr = {n: g.download_profile(n) for n in PROFILE_NAMES}
    return f, f2, pr


def assert_mirror(f):
    for n, a in f.items():
        m = a[:, ::-1, :]
        if n in ANTISYMMETRIC:
            m = -m
        assert np.array_equal(a, m), (n, float(np.max(np.abs(a - m))))


@pytest.mark.parametrize("grid", [(21, 91, 181), (11, 21, 41), (13, 30, 40)])
def test_initial_state_matches_oracle(grid):
    p = config_params()
    cfg = config_init()
    f, f2, pr = device_state(grid, p, cfg)
    o = OracleState.initial(*grid, p, cfg, compat=0)
    bad = {}
    for n in FIELD_NAMES:
        assert np.isfinite(f[n]).all(), n
        e = rel_err(f[n], o.f[n])
        if not e <= TOL:
            bad[n] = e
    for n in FIELD2D_NAMES:
        e = rel_err(f2[n], o.f2[n])
        if not e <= TOL:
            bad["2d:" + n] = e
    for n in PROFILE_NAMES:
        e = rel_err(pr[n], o.prof[n])
        if not e <= TOL:
            bad["profile:" + n] = e
    assert not bad, bad


def test_initial_state_mirror_symmetric_and_physical():
    """The configuration-2 grid: exact mirror symmetry of every field; the surface layer
    warmest at the equator (the prescribed parabola, 513.15 K to 503.15 K, after the wiggle
    filter); the 60 bar surface pressure."""
    grid = (41, 181, 361)
    p = config_params()
    f, f2, _ = device_state(grid, p)
    assert_mirror(f)
    assert_mirror({"2d_" + n: a[None] for n, a in f2.items()})
    for n, a in f.items():
        assert np.isfinite(a).all(), n
    t0 = f["t"][0] * p.t_0
    assert 503.15 < t0[90, 0] < 513.15 and t0[0, 0] < t0[90, 0]
    assert float(f["c"].max()) <= 1.0 and float(f["c"].min()) >= p.c_h2o_dry_top * 0.5
    assert float(f["p_stat"][0].min()) > 5.0e4     # the 60 bar surface, in hPa


def test_initial_state_native_grid_against_oracle():
    """The reference's own 61 x 181 x 361 grid."""
    grid = (61, 181, 361)
    p = config_params()
    cfg = config_init()
    f, _, _ = device_state(grid, p, cfg)
    o = OracleState.initial(*grid, p, cfg, compat=0)
    bad = {n: rel_err(f[n], o.f[n]) for n in FIELD_NAMES if not rel_err(f[n], o.f[n]) <= TOL}
    assert not bad, bad


def test_initial_state_rejects_bad_config():
    from athad_cond_b200 import AthadError
    p = config_params()
    cfg = config_init()
    cfg.tropopause_pole = -1.0
    with GpuAtmosphere(11, 21, 41, p) as g:
        with pytest.raises(AthadError):
            g.initial_state(cfg)
