"""The whole model iteration on the device (athad_cond_b200.loop.ModelLoop): every module
of run_3D_loop at the reference's cadence through the C ABI.  From a mirror-symmetric state
the state stays finite and exactly mirror-symmetric over eight iterations (two pressure
iterations, four moist ones); the residuum, budgets and skin temperature come back each
iteration as the reference prints them.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state, mirror
from athad_cond_b200._abi import Precision, config_params
from athad_cond_b200.loop import ModelLoop

pytestmark = pytest.mark.gpu

SYMMETRIC = ("t", "u", "w", "c", "cloud", "ice", "co2", "tke", "dis", "p_dyn", "p_stat", "r_humid",
             "nue", "P_rain", "P_snow", "TempDewPoint", "Q_Sensible")


@pytest.mark.parametrize("precision", [Precision.FP64, Precision.MIXED])
def test_model_loop_stays_finite_and_mirror_symmetric(precision):
    grid = (21, 91, 181)
    p = config_params()
    p.precision = int(precision)
    st = make_state(*grid, seed=157, symmetric=True)
    with GpuAtmosphere(*grid, p) as g:
        g.upload_state(st)
        loop = ModelLoop(g)
        reports = loop.run(8)
        for n in SYMMETRIC:
            a = g.download(n)
            assert np.isfinite(a).all(), n
            assert np.array_equal(a, mirror(a, False)), n
        v = g.download("v")
        assert np.isfinite(v).all() and np.array_equal(v, mirror(v, True))
    assert [r["iter_n"] for r in reports] == list(range(1, 9))
    assert all("h2o" in r for r in reports[1::2]) and not any("h2o" in r for r in reports[0::2])
    assert all(r["residuum"]["residuum"] > 0.0 for r in reports)
    assert reports[-1]["residuum"]["residuum_prev"] == reports[-2]["residuum"]["residuum"]
    assert reports[-1]["t_skin"] != p.t_skin
