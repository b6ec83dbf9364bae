"""The device thermodynamics (csrc/thermo.cuh), compiled for the host, against the known
answers of the reference's own self-tests and against the oracle's restatement.

tests/host_thermo.cu builds the evaluator that athad_thermo_eval runs on the GPU (k_thermo.cu)
for the host, so the same source is checked on a machine without a GPU.  Known answers: each
self-test assertion's tolerance (tests/golden/thermo_kat.json).  Against the oracle, over the
model's range: 1e-14 relative, both sides on the host's libm; the remaining few ulp come from
the device code's arrangement of the curves (the GPU test allows 1e-13 for CUDA's
exp/log/pow).

Skipped where nvcc is not installed.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from thermo_checks import (check_against_the_oracle_over_the_model_range, check_mixture_and_lapse_known_answers,
                           check_saturation_known_answers)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"

pytestmark = pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc not installed")


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("host_thermo") / "libhost_thermo.so")
    cmd = [NVCC, "-O2", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "athad_cond_b200", "csrc"), "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "host_thermo.cu"), "-o", out]
    subprocess.run(cmd, check=True, capture_output=True)
    lib = ctypes.CDLL(out)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.host_thermo_eval.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]

    def ev(fn, *cols):
        cols = [np.atleast_1d(np.asarray(c, dtype=np.float64)) for c in cols]
        n = max(len(c) for c in cols)
        x = np.ascontiguousarray(np.stack([np.broadcast_to(c, (n,)) for c in cols], axis=1))
        assert x.shape[1] == lib.host_thermo_arity(fn)
        out = np.empty(n)
        assert lib.host_thermo_eval(fn, n, x.ctypes.data_as(dp), out.ctypes.data_as(dp)) == 0
        return out
    return ev


def test_saturation_known_answers_host_build(host):
    check_saturation_known_answers(host)


def test_mixture_and_lapse_known_answers_host_build(host):
    check_mixture_and_lapse_known_answers(host)


def test_host_build_matches_the_oracle_over_the_model_range(host):
    check_against_the_oracle_over_the_model_range(host, tol=1e-14)
