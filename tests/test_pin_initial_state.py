"""Pin of the oracle's initial state against the reference itself.

The reference (built from its sources into oracle/_ref/pin, an IEEE build) runs its own
RunTimeSlice sequence (cAtmosphereModel.cpp:468-668) on one OpenMP thread; the oracle's
restatement (or_init_state, the reference's semantics) must reproduce every field, 2-D
field and profile bit for bit: after the velocities, the temperature, the water/co2/densities
fixed point and the cloud profile (cheap stages, each from a fresh model), and after the whole
sequence.  The device-semantics form (compat = 0) is checked for exact mirror symmetry.

Skipped where the reference was not built (a machine without the reference sources).
"""
import concurrent.futures
import os

import numpy as np
import pytest

import ref_binding
from athad_cond_b200._abi import FIELD_NAMES, Wall, config_init, config_params
from oracle_binding import OracleState

pytestmark = pytest.mark.skipif(not ref_binding.available("pin"),
                                reason="reference not built (oracle/_ref/pin)")

F2 = ("t_top_init", "p_stat_landscape", "vel_star", "Evaporation", "co2_total")
NATIVE_GRID = (61, 181, 361)   # the only grid the reference runs (cAtmosphereModel.h:162)


def params():
    p = config_params()
    p.wall_mode = Wall.REFERENCE
    return p


def reference_state(upto):
    cwd = os.getcwd()
    os.chdir(os.environ.get("TMPDIR", "/tmp"))
    try:
        R = ref_binding.Reference("pin", threads=1)
        R.init_state(upto)
        f = {n: R.get(n) for n in FIELD_NAMES}
        f2 = {}
        for n in F2:
            try:
                f2[n] = R.get2(n)
            except AssertionError:   # t_top_init before it is built
                pass
        prof = {n: R.getp(n) for n in ("rho_base", "dlnrho_dr")}
        prof = {n: a for n, a in prof.items() if a is not None}   # before densities builds them
        trop = R.tropopause_layers()
        shape = R.shape
        R.close()
    finally:
        os.chdir(cwd)
    return shape, f, f2, prof, trop


def assert_same(ref, o):
    _, f, f2, prof, _ = ref
    bad = [n for n in FIELD_NAMES if not np.array_equal(f[n], o.f[n])]
    bad += ["2d:" + n for n, a in f2.items() if not np.array_equal(a, o.f2[n])]
    bad += ["profile:" + n for n, a in prof.items() if not np.array_equal(a, o.prof[n])]
    assert not bad, bad


@pytest.mark.parametrize("upto", [1, 2, 3, 4])
def test_initial_state_stages_bit_exact(upto):
    ref = reference_state(upto)
    o = OracleState.initial(*ref[0], params(), config_init(), compat=1, upto=upto)
    assert_same(ref, o)


def test_initial_state_bit_exact():
    # the reference (one OpenMP thread) and the oracle build the state at the same time: both
    # are C calls that release the interpreter, and neither reads the other's memory
    with concurrent.futures.ThreadPoolExecutor(max_workers=1) as pool:
        oracle = pool.submit(OracleState.initial, *NATIVE_GRID, params(), config_init(), compat=1)
        ref = reference_state(99)
        o = oracle.result()
    assert ref[0] == NATIVE_GRID
    assert_same(ref, o)
    assert np.array_equal(o.tropopause_layers(config_init()), ref[4])


def test_device_semantics_mirror_symmetric():
    grid = (21, 91, 181)
    o = OracleState.initial(*grid, config_params(), config_init(), compat=0)
    anti = {"v", "vn", "aux_v", "MC_v", "v_u", "v_d"}
    for n in FIELD_NAMES:
        a = o.f[n]
        m = -a[:, ::-1, :] if n in anti else a[:, ::-1, :]
        assert np.array_equal(a, m), n
    t0 = o.f["t"][0] * 273.15     # the parabola after the wiggle filter and the moist adjustment
    assert 503.15 < t0[45, 7] < 513.15 and t0[0, 7] < t0[45, 7]
