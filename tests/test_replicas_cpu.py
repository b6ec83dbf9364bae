"""The multi-GPU path of bench.py on CPU: world_size-2 gloo ranks.

The hot path does not shard: `bench.py --gpus N` runs N independent replicas, one per rank,
each from the reference's deterministic initial state, and the only collectives are the
barrier around the timed region and the max-over-ranks of the measured time.  These tests run that host logic as two
gloo processes on 127.0.0.1, with the oracle standing in for the device replica:
  * every rank receives the largest of the per-rank times, and the whole-job value counts
    all ranks' grid points over that time;
  * a replica's result does not depend on the other rank (bit-identical to a run alone, and
    to the other rank's, since both start from the same deterministic state);
  * under torchrun the reference arm runs on rank 0 only: other ranks exit 0 silently.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GRID = (9, 13, 17)
ITERS = 4


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica(rank):
    """Four model iterations of the oracle at the bench cadence from the initial state;
    returns the final temperature and u fields."""
    sys.path.insert(0, ROOT)
    from athad_cond_b200._abi import config_init, config_params
    from oracle_binding import OracleState
    o = OracleState.initial(*GRID, config_params(), config_init())
    for it in range(1, ITERS + 1):
        if it % 4 == 0:
            o.pressure_sweep(1, it)
        if it % 2 == 0:
            o.saturation_adjust()
            o.moist_convection(it)
            o.densities()
        o.rk4(dt=4e-5, buoyancy_ramp=min(1.0, it / 300.0))
        o.store_n_level()
    return np.array(o.f["t"], copy=True), np.array(o.f["u"], copy=True)


def _rank_main(rank, world, port, out_dir):
    import datetime
    import torch.distributed as tdist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import bench
    tdist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                             world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        tdist.barrier()
        t, u = _replica(rank)
        tdist.barrier()
        local_ms = 10.0 + 5.0 * rank          # stand-in for the rank's device time
        ms = bench.max_over_ranks(local_ms, None)
        value = bench.whole_job_value(int(np.prod(GRID)), ITERS, world, ms)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), t=t, u=u, ms=ms, value=value)
    finally:
        tdist.destroy_process_group()


def test_two_gloo_replicas_max_time_and_independence(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    res = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    slowest = 10.0 + 5.0 * (world - 1)
    for r in res:
        assert float(r["ms"]) == slowest
        assert float(r["value"]) == pytest.approx(np.prod(GRID) * ITERS * world / (slowest * 1e-3))
    # replicas are independent: each equals the same replica run alone
    for rank in range(world):
        t, u = _replica(rank)
        assert np.array_equal(res[rank]["t"], t) and np.array_equal(res[rank]["u"], u)
    assert np.array_equal(res[0]["t"], res[1]["t"])


def test_max_over_ranks_without_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5) == 3.5


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "2", "--warmup", "3"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0
    assert p.stdout.strip() == ""


def test_bench_line_keys_are_json_serialisable():
    """The static parts of the bench line (launch count, aggregate value) for N = 1..8."""
    sys.path.insert(0, ROOT)
    import bench
    pts = int(np.prod(bench.GRID))
    for n in (1, 2, 4, 8):
        v = bench.whole_job_value(pts, 200, n, 1000.0)
        assert v == pytest.approx(pts * 200 * n)
        json.dumps({"value": v, "n_gpus": n})
