"""The reference as it is (tier A) against the semantics the CUDA path implements (tier B) on
the reference's own grid, 61 x 181 x 361, from its own initial state.

Test infrastructure, run by hand (about 20 minutes on 8 cores; not collected by pytest):

    python tests/ab_native_grid.py --iterations 100 > ab.json

A: the reference's own functions (oracle/_ref/pin: its sources, IEEE build), on its OpenMP
   threads (default 8): the in-place RK4 sweep whose neighbours are read at whatever stage
   they have reached, so its result depends on the sweep order and the thread count
   (RungeKutta_Atm_Turb.cpp:99-266), and its asymmetric SST wall distance.
B: the oracle in the product's semantics (compat = 0: Jacobi RK4 stages, exactly mirror-
   symmetric tables and sums, the mirror-symmetric SST wall distance), which the device
   matches to 1e-9 over 100 iterations.
Both start from the reference's initial state and run the hot path at the reference cadence
(RK4 and the time-level copy every iteration, pressure sweep every 4th, saturation
adjustment, moist convection and densities every 2nd).  Printed per field after iterations
1, 10 and the last: max|A - B| / max|A|, and for scale the run's own change
max|A_n - A_0| / max|A_0|.
"""
import argparse
import concurrent.futures
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

import ref_binding  # noqa: E402
from athad_cond_b200._abi import FIELD_NAMES, config_params  # noqa: E402
from oracle_binding import OracleState  # noqa: E402

FIELDS = ["t", "u", "v", "w", "c", "cloud", "ice", "gr", "co2", "tke", "dis", "p_dyn", "p_stat", "r_humid"]
DT = 4e-5


def reference_iteration(R, it):
    R.set_scalars(DT, 1.0, min(1.0, it / 300.0), it, it)
    if it % 4 == 0:
        R.lib.ref_pressure(R.h)
    if it % 2 == 0:
        R.lib.ref_satadj(R.h)
        R.lib.ref_moist(R.h, it)
        R.lib.ref_densities(R.h, 0)
    R.lib.ref_rk4(R.h)
    R.lib.ref_store(R.h)


def oracle_iteration(o, it):
    if it % 4 == 0:
        o.pressure_sweep(1, it)
    if it % 2 == 0:
        o.saturation_adjust()
        o.moist_convection(it)
        o.densities()
    o.rk4(dt=DT, buoyancy_ramp=min(1.0, it / 300.0))
    o.store_n_level()


def rel(a, b):
    den = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b))) / den if den > 0 else float(np.max(np.abs(a)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--iterations", type=int, default=100)
    ap.add_argument("--threads", type=int, default=8, help="the reference's OpenMP threads")
    args = ap.parse_args()
    if not ref_binding.available("pin"):
        sys.exit("the reference is not built (make -C oracle/ref)")
    cwd = os.getcwd()
    os.chdir(os.environ.get("TMPDIR", "/tmp"))
    sys.stdout.flush()
    saved = os.dup(1)
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)   # the reference prints its progress
    try:
        R = ref_binding.Reference("pin", threads=args.threads)
        R.init_state()
        st = {n: R.get(n) for n in FIELD_NAMES}
        for n in ("t_top_init", "p_stat_landscape", "vel_star", "Evaporation", "Q_sensible_2D"):
            st[n] = R.get2(n)
        o = OracleState(st, config_params())
        start = {n: st[n].copy() for n in FIELDS}
        out = {"grid": list(R.shape), "reference_threads": args.threads, "after": {}}
        marks = sorted({1, 10, args.iterations})
        pool = concurrent.futures.ThreadPoolExecutor(max_workers=1)
        for it in range(1, args.iterations + 1):
            done = pool.submit(oracle_iteration, o, it)   # both release the interpreter
            reference_iteration(R, it)
            done.result()
            if it in marks:
                a = {n: R.get(n) for n in FIELDS}
                out["after"][it] = {
                    "a_vs_b": {n: rel(o.f[n], a[n]) for n in FIELDS},
                    "change_of_a": {n: rel(a[n], start[n]) for n in FIELDS},
                }
        R.close()
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.chdir(cwd)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
