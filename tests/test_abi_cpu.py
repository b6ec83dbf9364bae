"""The C-ABI library loads and exports every entry point include/athad_gpu.h declares.
No compute call is made: this runs on a machine without a GPU."""
import ctypes
import os
import re

import pytest

from athad_cond_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "athad_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(athad_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ["athad_create", "athad_rk4_step", "athad_pressure_sweep", "athad_saturation_adjust",
              "athad_densities", "athad_moist_convection", "athad_upload", "athad_download"]:
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_abi.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    # and the Python signatures table covers the same set
    assert set(declared_symbols()) <= set(_abi.SIGNATURES), set(declared_symbols()) - set(_abi.SIGNATURES)


def test_default_params_match_config():
    lib = _abi.load_library()
    assert lib.athad_abi_version() == 11
    assert lib.athad_params_size() == ctypes.sizeof(_abi.Params)
    a = _abi.default_params().as_dict()
    b = _abi.config_params().as_dict()
    assert a == b
    c = _abi.InitConfig()
    lib.athad_default_init_config(ctypes.byref(c))
    d = _abi.config_init()
    assert {n: getattr(c, n) for n, _ in c._fields_} == {n: getattr(d, n) for n, _ in d._fields_}


def test_footprint_and_argument_checks():
    lib = _abi.load_library()
    g = _abi.Grid(41, 181, 361)
    fp = lib.athad_footprint_bytes(ctypes.byref(g))
    assert 2e9 < fp < 8e9
    bad = _abi.Grid(2, 3, 3)
    assert lib.athad_footprint_bytes(ctypes.byref(bad)) == 0
    h = ctypes.c_void_p()
    p = _abi.config_params()
    assert lib.athad_create(ctypes.byref(bad), ctypes.byref(p), ctypes.byref(h)) == _abi.Status.ERR_INVALID
    p.struct_size = 8
    assert lib.athad_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == _abi.Status.ERR_INVALID
    p = _abi.config_params()
    p.turb_model = 0
    assert lib.athad_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == _abi.Status.ERR_UNSUPPORTED


def test_no_device_is_reported_not_faked():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _abi.load_library()
    g = _abi.Grid(11, 21, 41)
    p = _abi.config_params()
    h = ctypes.c_void_p()
    assert lib.athad_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == _abi.Status.ERR_NO_DEVICE


def test_footprint_of_mixed_context_includes_fp32_buffers():
    """athad_footprint_bytes_params: the mixed form holds 55 FP32 fields and an FP32
    geometry table on top of the FP64 context; invalid precision gives 0."""
    from athad_cond_b200._abi import Grid, Precision, config_params
    lib = _abi.load_library()
    g = Grid(21, 91, 181)
    p = config_params()
    f64 = lib.athad_footprint_bytes_params(ctypes.byref(g), ctypes.byref(p))
    assert f64 == lib.athad_footprint_bytes(ctypes.byref(g))
    p.precision = int(Precision.MIXED)
    fm = lib.athad_footprint_bytes_params(ctypes.byref(g), ctypes.byref(p))
    field32 = 21 * 91 * 192 * 4
    assert fm - f64 >= 55 * field32
    p.precision = 7
    assert lib.athad_footprint_bytes_params(ctypes.byref(g), ctypes.byref(p)) == 0
