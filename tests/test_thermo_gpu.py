"""The device thermodynamics (csrc/thermo.cuh, evaluated on the GPU by athad_thermo_eval)
against the known answers of the reference's own self-tests (tests/golden/thermo_kat.json:
test/saturation_selftest.cpp, test/cond_column_selftest.cpp, with each assertion's
tolerance), and against the oracle's restatement over the model's range (within 1e-13
relative: CUDA's exp/log/pow against glibc's).
"""
import ctypes

import numpy as np
import pytest

from athad_cond_b200 import load_library
from thermo_checks import (check_against_the_oracle_over_the_model_range, check_mixture_and_lapse_known_answers,
                           check_saturation_known_answers)

pytestmark = pytest.mark.gpu


def dev(fn, *cols):
    """Evaluate function fn on the device for the tuples given column-wise."""
    L = load_library()
    cols = [np.atleast_1d(np.asarray(c, dtype=np.float64)) for c in cols]
    n = max(len(c) for c in cols)
    x = np.ascontiguousarray(np.stack([np.broadcast_to(c, (n,)) for c in cols], axis=1))
    assert x.shape[1] == L.athad_thermo_arity(fn)
    out = np.empty(n)
    dp = ctypes.POINTER(ctypes.c_double)
    assert L.athad_thermo_eval(fn, n, x.ctypes.data_as(dp), out.ctypes.data_as(dp)) == 0
    return out


def test_saturation_known_answers_on_device():
    check_saturation_known_answers(dev)


def test_mixture_and_lapse_known_answers_on_device():
    check_mixture_and_lapse_known_answers(dev)


def test_device_thermodynamics_match_the_oracle_over_the_model_range():
    check_against_the_oracle_over_the_model_range(dev, tol=1e-13)
