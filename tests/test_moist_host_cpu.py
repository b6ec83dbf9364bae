"""The CUDA library's moist-convection column code, compiled for the host, against the oracle.

`mc_column` (athad_cond_b200/csrc/k_moist.cu) is __host__ __device__: the device kernel runs
it one thread per (j, k) column, and tests/host_moist.cu runs the same source on the host,
column after column.  This checks the kernel's logic (every phase of MoistConvection::run,
MoistConvection.h:106-1537, its branches, its level recurrences and the order of its loads
and stores) against the oracle's restatement (oracle/or_moist.c) on a machine without a
GPU.  Both sides use the host's libm, so the remaining differences are rounding-order ones:
tolerance 1e-12 relative to each field's largest magnitude (the device test, which adds
CUDA's exp/pow and fused multiply-add, uses 1e-10).

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

MC_FIELDS = ["s", "s_u", "s_d", "M_u", "M_d", "q_v_u", "q_c_u", "q_v_d", "u_u", "v_u", "w_u",
             "u_d", "v_d", "w_d", "E_u", "D_u", "E_d", "D_d", "c_u", "e_l", "e_d", "e_p", "g_p",
             "P_conv", "CloudBase", "LevelFreeSinking", "Deep_beg", "Deep_end",
             "MC_t", "MC_q", "MC_v", "MC_w"]
TOL = 1e-12


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("host_moist") / "libhost_moist.so")
    cmd = [NVCC, "-O2", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "athad_cond_b200", "csrc"), "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "host_moist.cu"), "-o", out]
    subprocess.run(cmd, check=True, capture_output=True)
    lib = ctypes.CDLL(out)
    lib.host_moist_convection.restype = None
    return lib


def host_run(lib, o: OracleState):
    """mc_column over every column of a copy of o's fields; returns the copy."""
    im, jm, km = o.shape
    p = o.params
    f = {n: np.ascontiguousarray(o.f[n], dtype=np.float64).copy() for n in FIELD_NAMES}
    F = (ctypes.c_void_p * len(FIELD_NAMES))(*[f[n].ctypes.data for n in FIELD_NAMES])
    ev = np.ascontiguousarray(o.f2["Evaporation"])
    qs = np.ascontiguousarray(o.f2["Q_sensible_2D"])
    height, step, cose = o.moist_geometry()
    dp = np.array([p.t_0, p.cp_l, p.s_0, p.lv, p.ls, p.g, p.u_0, p.r_Earth, p.p_0, p.co2_0, p.c_0,
                   p.M_bg, p.R_bg])
    ip = np.array([p.convection_perturbation, p.convection_mode, p.iter_prec], dtype=np.int32)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    lib.host_moist_convection(im, jm, km, F, P(ev), P(qs), P(height), P(step), P(cose), P(dp), P(ip))
    return f


def assert_close(f, o, tag):
    for n in MC_FIELDS:
        a, b = f[n], o.f[n]
        assert np.array_equal(np.isfinite(a), np.isfinite(b)), (tag, n, "non-finite cells differ")
        fin = np.isfinite(b)
        den = max(float(np.max(np.abs(b[fin]), initial=0.0)), 1e-300)
        err = float(np.max(np.abs(a[fin] - b[fin]), initial=0.0)) / den
        assert err <= TOL, (tag, n, err)


def convective_state(grid, seed):
    """A synthetic state moist enough near the surface to trigger the scheme."""
    st = make_state(*grid, seed=seed)
    st["c"][: grid[0] // 3] *= 1.6
    st["Evaporation"] = np.full(grid[1:], 20.0)
    st["Q_sensible_2D"] = np.zeros(grid[1:])
    return st


@pytest.mark.parametrize("grid", [(11, 21, 41), (21, 91, 181)])
def test_host_column_code_matches_oracle_two_calls(host_lib, grid):
    o = OracleState(convective_state(grid, seed=37), config_params())
    for it in (2, 4):   # the second call starts from the first one's fluxes and precipitation
        f = host_run(host_lib, o)
        o.moist_convection(it)
        assert_close(f, o, it)
        for n in MC_FIELDS:
            o.f[n][...] = f[n]   # continue from the host result
    for n in ("M_u", "M_d", "E_u", "E_d", "c_u", "g_p"):   # updraft and downdraft both ran
        assert np.max(np.abs(o.f[n])) > 0.0, n


def test_host_column_code_on_the_reference_initial_state(host_lib):
    """The reference's initial state convects nowhere: the deep-layer and cloud-base searches
    run through every level of every column."""
    o = OracleState.initial(11, 21, 41, config_params(), config_init())
    f = host_run(host_lib, o)
    o.moist_convection(2)
    assert_close(f, o, "initial state")


def test_host_column_code_with_non_finite_inputs(host_lib):
    grid = (11, 21, 41)
    st = convective_state(grid, seed=53)
    rng = np.random.default_rng(53)
    for name, value in (("t", np.nan), ("c", np.inf), ("M_u", np.nan), ("M_d", 7.0)):
        idx = tuple(rng.integers(0, s, 25) for s in grid)
        a = st.get(name, np.zeros(grid)).copy()
        a[idx] = value
        st[name] = a
    o = OracleState(st, config_params())
    f = host_run(host_lib, o)
    o.moist_convection(2)
    assert_close(f, o, "non-finite")
