"""The CUDA library's column passes (k_columns.cu), compiled for the host, against the oracle.

The per-cell body of the saturation adjustment kernel (`satadj_cell`: adjustSaturation and
clampAndFade, SaturationAdjustment.h:62-459) and the per-column body of the densities kernel
(`densities_column`: the upward integration of ThermoAtm.h:1484-1614) are __host__ __device__;
tests/host_columns.cu runs the same source on the host over every cell / column.  This
checks the kernels' logic against the oracle (oracle/or_columns.c) on a machine without a
GPU, on the reference initial state, on states that drive every branch, and with non-finite
inputs.  Both sides use the host's libm; the kernels form some quotients as products by one
reciprocal and share powers between the saturation curves, which the Newton iteration of
the adjustment carries forward: tolerance 1e-11 for the adjustment, as in the device test,
and 1e-13 for the densities (the device test, which adds CUDA's transcendentals and fused
multiply-add, uses 1e-11), relative to each field's largest magnitude.

Skipped where nvcc is not installed.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from athad_cond_b200 import make_state
from athad_cond_b200._abi import FIELD_NAMES, config_init, config_params
from oracle_binding import OracleState

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"

pytestmark = pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc not installed")

SATADJ_FIELDS = ["t", "c", "cloud", "ice", "gr", "S_c_c", "P_rain", "P_snow", "P_graupel",
                 "Precipitation", "S_v", "S_c", "S_i", "S_r", "S_s", "S_g"]
DENS_FIELDS = ["t", "c", "p_stat", "r_humid", "r_dry"]
TOL_SATADJ, TOL_DENS = 1e-11, 1e-13


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("host_columns") / "libhost_columns.so")
    cmd = [NVCC, "-O2", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "athad_cond_b200", "csrc"), "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "host_columns.cu"), "-o", out]
    subprocess.run(cmd, check=True, capture_output=True)
    lib = ctypes.CDLL(out)
    lib.host_saturation_adjust.restype = ctypes.c_longlong
    lib.host_densities_columns.restype = None
    return lib


def host_call(lib, o: OracleState, which, set_water_profile=False):
    """The host build on a copy of o's fields; returns (fields, 2-D fields, result)."""
    im, jm, km = o.shape
    p = o.params
    f = {n: np.ascontiguousarray(o.f[n], dtype=np.float64).copy() for n in FIELD_NAMES}
    F = (ctypes.c_void_p * len(FIELD_NAMES))(*[f[n].ctypes.data for n in FIELD_NAMES])
    f2 = {n: np.ascontiguousarray(o.f2[n], dtype=np.float64).copy() for n in ("t_top_init", "p_stat_landscape")}
    height, step_f = o.column_geometry()
    dp = np.array([p.t_0, p.t_00, p.t_max_phys, p.cloud_cap, p.M_bg, p.R_bg, p.R_mix, p.r_air, p.g,
                   p.t_skin, p.c_h2o_dry_top])
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    args = (im, jm, km, F, P(f2["t_top_init"]), P(f2["p_stat_landscape"]), P(height), P(step_f), P(dp))
    if which == "satadj":
        r = lib.host_saturation_adjust(*args)
    else:
        r = lib.host_densities_columns(*args, 1 if set_water_profile else 0)
    return f, f2, r


def assert_close(got: dict, want: dict, names, tag, tol):
    for n in names:
        a, b = got[n], want[n]
        assert np.array_equal(np.isfinite(a), np.isfinite(b)), (tag, n, "non-finite cells differ")
        fin = np.isfinite(b)
        den = max(float(np.max(np.abs(b[fin]), initial=0.0)), 1e-300)
        err = float(np.max(np.abs(a[fin] - b[fin]), initial=0.0)) / den
        assert err <= tol, (tag, n, err)


def satadj_state(grid, seed=23):
    """Part of each column driven supersaturated or subsaturated with condensate, some
    cells supercritical, superheated or at the vapour cap, so that every branch of the
    adjustment and of clampAndFade runs (the device test's construction)."""
    st = make_state(*grid, seed=seed)
    im = grid[0]
    st["c"] = st["c"] * 1.5
    st["cloud"][im // 2:, :, ::3] += 2e-3
    st["t"][1, :, ::5] = 700.0 / 273.15
    st["P_rain"][:, :, ::7] = 1e-5
    st["co2"][2, :, ::11] = 0.99
    return OracleState(st, config_params())


def state_off_saturation(grid, seed):
    """The reference initial state with the vapour, temperature and condensate moved off
    their values and precipitation seeded."""
    o = OracleState.initial(*grid, config_params(), config_init())
    rng = np.random.default_rng(seed)
    o.f["c"] *= rng.uniform(0.7, 1.3, grid)
    o.f["cloud"][...] = rng.uniform(0.0, 2e-3, grid) * (rng.random(grid) < 0.5)
    o.f["ice"][...] = rng.uniform(0.0, 1e-3, grid) * (rng.random(grid) < 0.3)
    o.f["t"] *= rng.uniform(0.97, 1.03, grid)
    for n in ("P_rain", "P_snow", "P_graupel", "gr"):
        o.f[n][...] = rng.uniform(0.0, 1e-4, grid) * (rng.random(grid) < 0.2)
    return o


@pytest.mark.parametrize("grid", [(11, 21, 41), (21, 91, 181)])
def test_host_saturation_adjust_matches_oracle(host_lib, grid):
    o = satadj_state(grid)
    f, _, hits = host_call(host_lib, o, "satadj")
    want = o.saturation_adjust()
    assert_close(f, o.f, SATADJ_FIELDS, "satadj", TOL_SATADJ)
    assert hits == want


def test_host_saturation_adjust_on_the_reference_initial_state(host_lib):
    o = OracleState.initial(11, 21, 41, config_params(), config_init())
    f, _, hits = host_call(host_lib, o, "satadj")
    assert hits == o.saturation_adjust()
    assert_close(f, o.f, SATADJ_FIELDS, "initial state", TOL_SATADJ)


@pytest.mark.parametrize("set_water_profile", [False, True])
@pytest.mark.parametrize("grid", [(11, 21, 41), (21, 91, 181)])
def test_host_densities_columns_match_oracle(host_lib, grid, set_water_profile):
    o = state_off_saturation(grid, seed=13)
    f, f2, _ = host_call(host_lib, o, "densities", set_water_profile)
    o.densities(set_water_profile=set_water_profile)
    assert_close(f, o.f, DENS_FIELDS, "densities", TOL_DENS)
    assert_close(f2, o.f2, ["t_top_init", "p_stat_landscape"], "densities 2-D", TOL_DENS)


def test_host_column_passes_with_non_finite_inputs(host_lib):
    grid = (11, 21, 41)
    o = satadj_state(grid, seed=17)
    rng = np.random.default_rng(17)
    for name, value in (("t", np.nan), ("c", np.inf), ("cloud", np.nan), ("p_stat", -1.0)):
        idx = tuple(rng.integers(1, s - 1, 20) for s in grid)
        o.f[name][idx] = value
    f, _, hits = host_call(host_lib, o, "satadj")
    assert hits == o.saturation_adjust()
    assert_close(f, o.f, SATADJ_FIELDS, "satadj non-finite", TOL_SATADJ)
    f, f2, _ = host_call(host_lib, o, "densities")
    o.densities()
    assert_close(f, o.f, DENS_FIELDS, "densities non-finite", TOL_DENS)
