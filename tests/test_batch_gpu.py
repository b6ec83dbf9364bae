"""Batched ensembles (athad_batch_*): members of uneven grids advanced together.

The batched kernels run the per-cell code of the single-grid mixed-precision step on every
member, so each member's result must be bit-for-bit what the same iterations give on that
member alone: through a batch of one (the serving path of a request run alone), and
through the single-context entry points with the same scalars (the mixed-precision kernels
are compiled without fused multiply-add, so both kernels round every operation alike).  Covered: uneven grids, members at different iteration numbers (different
cadence phases), the CUDA-graph replay, every tile shape of the autotuner, inactive members.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, GpuBatch, make_state
from athad_cond_b200._abi import Precision, config_params

pytestmark = pytest.mark.gpu

GRIDS = [(11, 21, 41), (13, 31, 61), (9, 25, 45), (21, 45, 91)]
CHECK = ["t", "u", "v", "w", "c", "cloud", "ice", "gr", "co2", "tke", "dis",
         "tn", "un", "p_dyn", "p_stat", "r_humid", "MC_t", "aux_u"]


def member(grid, seed):
    p = config_params()
    p.precision = int(Precision.MIXED)
    st = make_state(*grid, seed=seed)
    st["Evaporation"] = np.full(grid[1:], 20.0)
    g = GpuAtmosphere(*grid, p)
    g.upload_state(st)
    return g


def alone_api(grid, seed, first_iter, n_iter):
    """The same iterations through the single-context entry points."""
    g = member(grid, seed)
    for it in range(first_iter, first_iter + n_iter):
        if it % 4 == 0:
            g.PressureSolverAtm_run(total_iter_count=it)
        if it % 2 == 0:
            g.SaturationAdjustment_run()
            g.MoistConvection_run(it)
            g.densities()
        g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, min(1.0, it / 300.0))
        g.storeIntermediateData3D()
    out = {n: g.download(n) for n in CHECK}
    g.close()
    return out


def alone_batch(grid, seed, first_iter, n_iter, graph=False):
    g = member(grid, seed)
    with GpuBatch([g], first_iter=[first_iter]) as b:
        for _ in range(n_iter):
            b.iteration(graph=graph)
        b.synchronize()
    out = {n: g.download(n) for n in CHECK}
    g.close()
    return out


@pytest.mark.parametrize("graph", [False, True])
def test_members_in_the_mix_equal_members_alone(graph):
    first = [1, 2, 3, 4]
    ms = [member(gr, 100 + q) for q, gr in enumerate(GRIDS)]
    with GpuBatch(ms, first_iter=first) as b:
        for _ in range(9):
            b.iteration(graph=graph)
        b.synchronize()
        assert [b.member_iter(q) for q in range(len(ms))] == [f + 9 for f in first]
    for q, gr in enumerate(GRIDS):
        mix = {n: ms[q].download(n) for n in CHECK}
        ref = alone_batch(gr, 100 + q, first[q], 9)
        api = alone_api(gr, 100 + q, first[q], 9)
        for n in CHECK:
            assert np.isfinite(mix[n]).all(), (q, n)
            assert np.array_equal(mix[n], ref[n]), (q, n)
            assert np.array_equal(mix[n], api[n]), (q, n)
        ms[q].close()


def test_every_tile_shape_gives_the_same_bits():
    lib_shapes = None
    results = []
    ms0 = [member(gr, 200 + q) for q, gr in enumerate(GRIDS[:3])]
    with GpuBatch(ms0) as b:
        lib_shapes = int(b.lib.athad_batch_shape_count())
    for m in ms0:
        m.close()
    for shape in range(lib_shapes):
        ms = [member(gr, 200 + q) for q, gr in enumerate(GRIDS[:3])]
        with GpuBatch(ms) as b:
            b.set_shape(shape)
            for _ in range(4):
                b.iteration()
            b.synchronize()
        results.append([{n: m.download(n) for n in CHECK} for m in ms])
        for m in ms:
            m.close()
    for r in results[1:]:
        for q in range(3):
            for n in CHECK:
                assert np.array_equal(r[q][n], results[0][q][n]), (q, n)


def test_autotune_picks_a_shape_and_leaves_the_state():
    ms = [member(gr, 300 + q) for q, gr in enumerate(GRIDS)]
    with GpuBatch(ms) as b:
        b.iteration()
        b.synchronize()
        before = [{n: m.download(n) for n in CHECK} for m in ms]
        best, times = b.autotune(reps=2)
        b.synchronize()
        assert 0 <= best < len(times) and all(t > 0 for t in times)
        assert times[best] == min(times)
        after = [{n: m.download(n) for n in CHECK} for m in ms]
    for q in range(len(ms)):
        for n in CHECK:
            assert np.array_equal(before[q][n], after[q][n]), (q, n)
        ms[q].close()


def test_inactive_member_is_left_alone():
    ms = [member(gr, 400 + q) for q, gr in enumerate(GRIDS[:2])]
    keep = {n: ms[1].download(n) for n in CHECK}
    with GpuBatch(ms) as b:
        b.set_active(1, False)
        for _ in range(3):
            b.iteration(graph=True)
        b.synchronize()
        assert b.member_iter(0) == 4 and b.member_iter(1) == 1
    for n in CHECK:
        assert np.array_equal(ms[1].download(n), keep[n]), n
    ref = alone_batch(GRIDS[0], 400, 1, 3)
    for n in CHECK:
        assert np.array_equal(ms[0].download(n), ref[n]), n
    for m in ms:
        m.close()


def test_batch_rejects_fp64_members_and_duplicates():
    from athad_cond_b200 import AthadError
    g64 = GpuAtmosphere(*GRIDS[0], config_params())
    with pytest.raises(AthadError):
        GpuBatch([g64])
    gm = member(GRIDS[0], 1)
    with pytest.raises(AthadError):
        GpuBatch([gm, gm])
    g64.close()
    gm.close()


def test_configuration4_members_in_the_mix_equal_members_alone():
    """Members drawn as the 64-member ensemble draws them (grids 21-41 x 61-181 x 121-361,
    condition points over p_surf 40-100 bar and T_sea 503-523 K), each from the reference
    initial state for its grid and condition point: six batched iterations (graph, the
    cadence of each member's own iteration counter) equal the same iterations of each member
    alone through the single-context entry points, bit for bit."""
    from athad_cond_b200.ensemble import draw_ensemble, condition_params, init_config
    specs = draw_ensemble(64)
    largest = sorted(range(len(specs)), key=lambda q: -int(np.prod(specs[q].grid)))
    picks = list(dict.fromkeys(largest[:2] + [0, 1, 2]))[:4]   # the two largest and the first
    chosen = [specs[q] for q in picks]

    def build(s):
        g = GpuAtmosphere(*s.grid, condition_params(s.cond, Precision.MIXED))
        g.initial_state(init_config(s.cond))
        return g

    first = [1, 2, 3, 4]
    ms = [build(s) for s in chosen]
    with GpuBatch(ms, first_iter=first) as b:
        for _ in range(6):
            b.iteration(graph=True)
        b.synchronize()
    for q, s in enumerate(chosen):
        mix = {n: ms[q].download(n) for n in CHECK}
        ms[q].close()
        g = build(s)
        for it in range(first[q], first[q] + 6):
            if it % 4 == 0:
                g.PressureSolverAtm_run(total_iter_count=it)
            if it % 2 == 0:
                g.SaturationAdjustment_run()
                g.MoistConvection_run(it)
                g.densities()
            g.solveRungeKutta_Atmosphere_Turb(4e-5, 1.0, min(1.0, it / 300.0))
            g.storeIntermediateData3D()
        for n in CHECK:
            a = g.download(n)
            assert np.isfinite(mix[n]).all(), (s.grid, n)
            assert np.array_equal(mix[n], a), (s.grid, n)
        g.close()
