"""The drop-in on the reference itself: the product's C++ adapter
(athad_cond_b200/host/athad_dropin.hpp), compiled against the reference's cAtmosphereModel,
replaces each hot-path call on the reference's own model object and initial state.  The
results must match what the reference's own CPU call produces on the same state:

  * saturation adjustment, densities, moist convection, pressure sweep: 1e-10 relative
    (CUDA vs glibc transcendentals, mirror-symmetric trig tables);
  * the boundary conditions and the smoothing filters: bit-identical (copies and short
    sums in the same order);
  * the RK4 step: the device integrates the four stages Jacobi-style where the reference
    updates cells in place, so the difference is bounded by a small fraction of the step's
    own change, with the reference's SST wall distance selected.
"""
import os

import numpy as np
import pytest

import ref_binding
from athad_cond_b200._abi import FIELD_NAMES

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(ref_binding.lib_path("dropin")),
                                 reason="reference + drop-in not built")]


@pytest.fixture(scope="module")
def model():
    cwd = os.getcwd()
    os.chdir(os.environ.get("TMPDIR", "/tmp"))
    try:
        R = ref_binding.Reference("dropin", threads=max(1, min(8, os.cpu_count() or 1)))
        R.init_state()
        snap = {n: R.get(n) for n in FIELD_NAMES}
        yield R, snap
        R.close()
    finally:
        os.chdir(cwd)


def reset(R, snap):
    for n, a in snap.items():
        R.set(n, a)


def relerr(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def run_both(R, snap, cpu, gpu, names):
    reset(R, snap)
    cpu()
    want = {n: R.get(n) for n in names}
    reset(R, snap)
    gpu()
    return {n: (R.get(n), want[n]) for n in names}


def test_dropin_saturation_adjustment(model):
    R, snap = model
    out = run_both(R, snap, lambda: R.lib.ref_satadj(R.h), lambda: R.dropin(2),
                   ["t", "c", "cloud", "ice", "S_c_c"])
    for n, (a, b) in out.items():
        assert relerr(a, b) <= 1e-10, n


def test_dropin_densities(model):
    R, snap = model
    out = run_both(R, snap, lambda: R.lib.ref_densities(R.h, 0), lambda: R.dropin(4),
                   ["t", "p_stat", "r_humid", "r_dry"])
    for n, (a, b) in out.items():
        assert relerr(a, b) <= 1e-10, n


def test_dropin_moist_convection(model):
    R, snap = model
    names = ["M_u", "M_d", "q_v_u", "q_c_u", "P_conv", "MC_t", "MC_q", "MC_v", "MC_w"]
    out = run_both(R, snap, lambda: R.lib.ref_moist(R.h, 2), lambda: R.dropin(3, 2), names)
    for n, (a, b) in out.items():
        assert relerr(a, b) <= 1e-10, n


def test_dropin_pressure_sweep(model):
    R, snap = model
    rng = np.random.default_rng(9)
    aux = {n: 1e-2 * rng.standard_normal(R.shape) for n in ("aux_u", "aux_v", "aux_w")}
    snap2 = dict(snap)
    snap2.update(aux)
    R.set_scalars(4e-5, 1.0, 1.0, 8, 8)
    out = run_both(R, snap2, lambda: R.lib.ref_pressure(R.h), lambda: R.dropin(1), ["p_dyn"])
    a, b = out["p_dyn"]
    assert relerr(a, b) <= 1e-10


def test_dropin_rk4(model):
    R, snap = model
    R.set_scalars(4e-5, 1.0, 0.3, 90, 90)
    names = ["t", "u", "v", "w", "c", "tke", "dis"]
    out = run_both(R, snap, lambda: R.lib.ref_rk4(R.h), lambda: R.dropin(0, 0, wall=1), names)
    for n, (a, b) in out.items():
        step = np.max(np.abs(b - snap[n]))
        assert np.max(np.abs(a - b)) <= 1e-2 * step, n


def test_dropin_boundary_conditions(model):
    """BC_Atm::bcRadius + TurbulenceAtm::apply_wall_bc + bcTheta + bcPhi through the adapter,
    on the reference's state with every field moved off its boundary values: bit-identical."""
    R, snap = model
    im, jm, km = R.shape
    pattern = 1.0 + 1e-3 * np.sin(np.arange(im * jm * km, dtype=np.float64) * 0.37).reshape(im, jm, km)
    moved = {n: a * pattern for n, a in snap.items()}
    out = run_both(R, moved, lambda: R.bc(), lambda: R.dropin(6), FIELD_NAMES)
    reset(R, snap)
    for n, (a, b) in out.items():
        assert np.array_equal(a, b), (n, float(np.max(np.abs(a - b))))


def test_dropin_filters(model):
    """The post-RK4 filters and the moist iteration's damp_wiggles through the adapter, on
    the reference's state with grid-scale noise added: the filtered velocities bit-identical
    to the reference's own AtomUtils calls; the damped fields within 1e-15 of each field's
    largest magnitude (the device adds the two meridional neighbours first, so that mirrored
    rows round alike; the reference subtracts first)."""
    R, snap = model
    im, jm, km = R.shape
    rng = np.random.default_rng(7)
    noisy = dict(snap)
    for n in ("u", "v", "w", "t", "c", "cloud", "ice"):
        noisy[n] = snap[n] + 1e-3 * np.abs(snap[n]).max() * rng.standard_normal((im, jm, km))

    def cpu():
        R.post_rk4_filters()
        for n in ("t", "ice", "c", "cloud"):
            R.damp_wiggles(n)

    def gpu():
        R.dropin(7)
        R.dropin(8)

    out = run_both(R, noisy, cpu, gpu, ["u", "v", "w", "t", "c", "cloud", "ice"])
    reset(R, snap)
    for n, (a, b) in out.items():
        if n in ("u", "v", "w"):
            assert np.array_equal(a, b), (n, float(np.max(np.abs(a - b))))
        else:
            assert relerr(a, b) <= 1e-15, (n, relerr(a, b))


def test_dropin_turbulence(model):
    """TurbulenceAtm::run through the adapter against the reference's own call on one
    thread.  The device reads every neighbour before the call; the reference's in-place
    sweep reads the floored tke/dis of the neighbours it visited first.  So: prod, nue,
    tke_source, tke, dis and vel_star within 1e-10; dis_source (whose cross-diffusion term
    reads the neighbours' tke/dis) within 1e-10 wherever no neighbour's tke was floored,
    and within 1e-2 of its largest magnitude everywhere."""
    R, snap = model
    names = ["tke", "dis", "nue", "prod", "tke_source", "dis_source"]
    out = run_both(R, snap, lambda: R.turbulence_run(threads=1), lambda: R.dropin(9), names)
    reset(R, snap)
    for n, (a, b) in out.items():
        if n != "dis_source":
            assert relerr(a, b) <= 1e-10, n
    a, b = out["dis_source"]
    floored = out["tke"][1] != snap["tke"]
    near = np.zeros_like(floored)
    near[1:] |= floored[:-1]
    near[:-1] |= floored[1:]
    near[:, 1:] |= floored[:, :-1]
    near[:, :-1] |= floored[:, 1:]
    near[:, :, 1:] |= floored[:, :, :-1]
    near[:, :, :-1] |= floored[:, :, 1:]
    scale = max(np.max(np.abs(b)), 1e-300)
    assert np.max(np.abs(a - b)[~near]) / scale <= 1e-10
    assert relerr(a, b) <= 1e-2


def test_dropin_two_cat_ice_scheme(model):
    """TwoCatIceScheme::run through the adapter against the reference's own call, on the
    reference's state after its saturation adjustment with rain and snow seeded: within
    1e-10 (CUDA vs glibc pow/exp and the saturation curves)."""
    R, snap = model
    im, jm, km = R.shape
    rng = np.random.default_rng(59)
    seeded = dict(snap)
    seeded["P_rainn"] = 2e-4 * rng.random((im, jm, km))
    seeded["P_snown"] = 2e-4 * rng.random((im, jm, km))
    names = ["t", "c", "cloud", "ice", "P_rain", "P_snow", "Precipitation", "S_v", "S_c", "S_i",
             "S_r", "S_s"]

    def prep():
        R.lib.ref_satadj(R.h)

    out = run_both(R, seeded, lambda: (prep(), R.two_cat_ice()), lambda: (prep(), R.dropin(10)), names)
    reset(R, snap)
    for n, (a, b) in out.items():
        assert relerr(a, b) <= 1e-10, (n, relerr(a, b))


@pytest.mark.parametrize("category", [0, 1, 3])
def test_dropin_other_ice_schemes(model, category):
    """The CategoryIceScheme switch through the adapter (IceSchemeRun, the model's category
    set to 0, 1 or 3) against the reference's own scheme, on the reference's state after its
    saturation adjustment with rain, snow and graupel seeded and cloud water in the k = 1
    plane (OneCat's carried rate is then assigned before it is read): within 1e-10."""
    R, snap = model
    im, jm, km = R.shape
    rng = np.random.default_rng(61 + category)
    seeded = dict(snap)
    for n in ("P_rainn", "P_snown", "P_graupel"):
        seeded[n] = 2e-4 * rng.random((im, jm, km))
    cloud = np.array(snap["cloud"], copy=True)
    cloud[:, :, 1] = np.maximum(cloud[:, :, 1], 1e-5)
    seeded["cloud"] = cloud
    names = ["t", "c", "cloud", "ice", "gr", "P_rain", "P_snow", "P_graupel", "Precipitation",
             "S_v", "S_c", "S_i", "S_r", "S_s", "S_g"]

    def prep():
        R.lib.ref_satadj(R.h)
        c = R.get("cloud")
        c[:, :, 1] = np.maximum(c[:, :, 1], 1e-5)
        R.set("cloud", c)

    out = run_both(R, seeded, lambda: (prep(), R.ice_scheme(category)),
                   lambda: (prep(), R.dropin(18, category)), names)
    reset(R, snap)
    for n, (a, b) in out.items():
        assert relerr(a, b) <= 1e-10, (n, relerr(a, b))


def test_dropin_radiation(model):
    """MultiLayerRadiation::run and radiation mode 2's heating through the adapter against the
    reference's own calls, cloud and ice seeded: within 1e-12 (CUDA vs glibc pow/exp)."""
    R, snap = model
    im, jm, km = R.shape
    rng = np.random.default_rng(61)
    seeded = dict(snap)
    seeded["cloud"] = 2e-4 * rng.random((im, jm, km))
    seeded["ice"] = 2e-4 * rng.random((im, jm, km))
    names = ["t", "radiation", "epsilon"]
    for cpu, what in ((R.mlr, 11), (lambda: R.radiative_heating(0.05), 12)):
        out = run_both(R, seeded, cpu, lambda: R.dropin(what), names)
        for n, (a, b) in out.items():
            assert relerr(a, b) <= 1e-12, (what, n, relerr(a, b))
    reset(R, snap)


def test_dropin_stand_atm_dew_point(model):
    """ThermoAtm::standAtm_DewPoint_HumidRel through the adapter against the reference's own
    call: TempStand bit for bit, the dew point and relative humidity within 1e-12 (CUDA's exp,
    log and sqrt against glibc's pow and exp in the saturation curves)."""
    R, snap = model
    names = ["TempStand", "TempDewPoint", "HumidityRel"]
    out = run_both(R, snap, R.stand_atm, lambda: R.dropin(13), names)
    reset(R, snap)
    assert np.array_equal(*out["TempStand"])
    for n in names[1:]:
        a, b = out[n]
        assert relerr(a, b) <= 1e-12, (n, relerr(a, b))


def test_dropin_find_residuum(model):
    """UtilsAtm::findResiduumAtm through the adapter: the residuum it leaves in residuum_old
    is the reference's, bit for bit."""
    R, snap = model
    reset(R, snap)
    want = R.find_residuum(threads=1)["residuum"]
    reset(R, snap)
    R.dropin(14)
    assert R.residuum_old() == want


def test_dropin_surface_fluxes(model):
    """ThermoAtm::waterVapourEvaporation and ::latentSensibleHeat through the adapter against
    the reference's own calls: c and the evaporation fields within 1e-12 (CUDA's exp, log and
    sqrt against glibc's pow and exp), Q_Sensible within 1e-12 (the reference's sin(theta)
    table is not mirror-exact; the device's is)."""
    R, snap = model
    out = run_both(R, snap, R.evaporation, lambda: R.dropin(15), ["c"])
    a, b = out["c"]
    assert relerr(a, b) <= 1e-12
    reset(R, snap)
    R.evaporation()
    want = {n: R.get2(n) for n in ("Evaporation", "Evaporation_Meyer", "c_fix")}
    reset(R, snap)
    R.dropin(15)
    for n, b in want.items():
        assert relerr(R.get2(n), b) <= 1e-12, n
    out = run_both(R, snap, R.latent_sensible, lambda: R.dropin(16), ["Q_Sensible", "Q_Latent"])
    reset(R, snap)
    for n, (a, b) in out.items():
        assert relerr(a, b) <= 1e-12, (n, relerr(a, b))


def test_dropin_mass_budgets(model):
    """ThermoAtm::co2Column and ::waterBudget through the adapter: co2_total bit for bit and the
    first-call references within 1e-12 of the reference's (sums in another fixed order)."""
    R, snap = model
    reset(R, snap)
    want = R.budgets(threads=1)
    co2_total = R.get2("co2_total")
    reset(R, snap)
    R.dropin(17)
    got = R.budget_refs()
    assert np.array_equal(R.get2("co2_total"), co2_total)
    for g, key in zip(got, ("q_co2_ref", "q_h2o_ref", "q_h2o_fixed_ref")):
        assert abs(g - want[key]) <= 1e-12 * want[key], key


F2D = ["t_top_init", "p_stat_landscape", "Evaporation", "Q_sensible_2D", "vel_star", "epsilon_2D",
       "albedo", "Evaporation_Dalton", "Evaporation_Meyer", "Evaporation_Rohwer", "c_fix", "co2_total"]


def test_dropin_resident_loop_equals_the_device_loop(model):
    """The device-resident drop-in (athad_dropin::ResidentLoop: the model's state uploaded
    once, every module of run_3D_loop's body on the device, the state synced back at the end)
    run for 20 iterations on the reference's own model is bit for bit the Python ModelLoop
    from the same state: the same entry points in the same order, checkpoint iteration 20
    (the momentum-budget capture) included.  The residuum and the skin temperature each
    iteration reports agree too."""
    from athad_cond_b200 import GpuAtmosphere
    from athad_cond_b200.loop import ModelLoop
    R, snap = model
    reset(R, snap)
    two = {n: R.get2(n) for n in F2D}
    prof = {n: R.getp(n) for n in ("t_ref_level", "rho_base", "dlnrho_dr")}
    sc = R.loop_scalars()          # what the resident loop takes from the model
    n_iter = 20
    with GpuAtmosphere(*R.shape, R.dropin_params()) as g:
        g.upload_state(dict(snap))
        for n, a in two.items():
            g.upload_2d(n, a)
        for n, a in prof.items():
            if a is not None:
                g.upload_profile(n, a)
        loop = ModelLoop(g, dt=sc["dt"], buoyancy_ramp_iters=sc["buoyancy_ramp_iters"],
                         t_skin_relax=sc["t_skin_relax"], tropopause_layers=R.tropopause_layers(),
                         checkpoint=sc["checkpoint"])
        loop.total_iter_count = sc["total_iter_count"]
        reps = loop.run(n_iter)
        want = {n: g.download(n) for n in FIELD_NAMES}
    res, skin = R.resident(n_iter)
    got = {n: R.get(n) for n in FIELD_NAMES}
    reset(R, snap)
    bad = [n for n in FIELD_NAMES if not np.array_equal(got[n], want[n])]
    assert not bad, bad
    assert res.tolist() == [r["residuum"]["residuum"] for r in reps]
    assert skin.tolist() == [r["t_skin"] for r in reps]

