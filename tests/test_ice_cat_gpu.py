"""athad_zero_cat_ice_scheme, athad_one_cat_ice_scheme and athad_three_cat_ice_scheme (the
schemes of CategoryIceScheme 0, 1 and 3) and the athad_ice_scheme switch on the device,
against the oracle, which is pinned bit for bit against the reference
(test_pin_reference.py::test_other_ice_schemes_bit_exact).

The state is the reference's deterministic initial state built on the device, after a
saturation adjustment, with falling rain, snow and graupel seeded from above, cloud ice and
graupel present and a redrawn sub-freezing band (230-285 K) with cloud water in 70 % of its
cells, so that the cold branches, OneCat's carried autoconversion rate and ThreeCat's
graupel all act.

Tolerance: 1e-10 of each field's largest magnitude, as for TwoCat: every cell forms a dozen
fractional powers and the saturation curves (CUDA's pow/exp/sin/cos against glibc's), and no
threshold of the schemes sits on a rounding edge in these states.  ZeroCat and ThreeCat keep
a mirror-symmetric state mirror-symmetric bit for bit; OneCat does not, and neither does the
reference: its autoconversion rate is carried from one column to the next in the serial
order, which has no mirror symmetry.
"""
import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, mirror
from athad_cond_b200._abi import FIELD_NAMES, Status, config_init, config_params
from athad_cond_b200.context import AthadError
from oracle_binding import OracleState

pytestmark = pytest.mark.gpu

OUT = ["t", "c", "cloud", "ice", "gr", "P_rain", "P_snow", "P_graupel", "Precipitation", "P_rainn",
       "P_snown", "S_v", "S_c", "S_i", "S_r", "S_s", "S_g", "S_c_c"]
RUN = {0: "zero_cat_ice_scheme", 1: "one_cat_ice_scheme", 2: "two_cat_ice_scheme",
       3: "three_cat_ice_scheme"}
TOL = 1e-10


def seeded_state(grid, seed, symmetric=False):
    """The device's initial state after a saturation adjustment, seeded as the module says."""
    im, jm, km = grid
    p = config_params()
    with GpuAtmosphere(*grid, p) as g:
        g.initial_state(config_init())
        g.SaturationAdjustment_run()
        st = {n: g.download(n) for n in FIELD_NAMES}
    rng = np.random.default_rng(seed)
    jh = (jm + 1) // 2

    def draw(n_i, f):
        a = f((n_i, jh if symmetric else jm, km))
        if symmetric:
            a = np.concatenate([a, a[:, :jm - jh][:, ::-1]], axis=1)
        return a

    for n in ("P_rainn", "P_snown", "P_graupel"):
        st[n] = draw(im, lambda s: 2e-4 * rng.random(s))
    lo, hi = int(0.5 * im), int(0.9 * im)
    for n in ("ice", "gr"):
        st[n][lo:hi] += draw(hi - lo, lambda s: np.where(rng.random(s) < 0.5, 0.0, 1e-5 * rng.random(s)))
    b0, b1 = int(0.65 * im), int(0.87 * im)
    st["t"][b0:b1] = draw(b1 - b0, lambda s: (230.0 + 55.0 * rng.random(s)) / 273.15)
    st["cloud"][b0:b1] = draw(b1 - b0, lambda s: np.where(rng.random(s) < 0.3, 0.0, 2e-3 * rng.random(s)))
    st["c"][b0:b1] *= draw(b1 - b0, lambda s: 0.5 + rng.random(s))
    return st


def run_both(grid, st, category, p=None):
    p = p or config_params()
    o = OracleState(st, p)
    with GpuAtmosphere(*grid, p) as g:
        g.upload_state(st)
        getattr(g, RUN[category])()
        out = {n: g.download(n) for n in OUT}
    o.ice_scheme(category)
    return out, o


def rel_errors(out, o):
    err = {}
    for n in OUT:
        a, b = out[n], o.f[n]
        den = float(np.max(np.abs(b)))
        err[n] = float(np.max(np.abs(a - b))) / den if den > 0 else float(np.max(np.abs(a)))
    return err


@pytest.mark.parametrize("category", [0, 1, 3])
@pytest.mark.parametrize("grid", [(25, 46, 91), (41, 181, 361)])
def test_ice_scheme_matches_oracle(category, grid):
    st = seeded_state(grid, 80 + category)
    out, o = run_both(grid, st, category)
    err = rel_errors(out, o)
    bad = {n: e for n, e in err.items() if not e <= TOL}
    assert not bad, (bad, err)
    # the scheme acted: rain sources in most columns, snow / graupel where the scheme has them
    assert np.count_nonzero(o.f["S_r"]) > o.f["S_r"].size // 4
    if category in (1, 3):
        assert np.count_nonzero(o.f["P_snow"]) > 0 and np.count_nonzero(o.f["S_s"]) > 0
    if category == 3:
        assert np.count_nonzero(o.f["P_graupel"]) > 0 and np.count_nonzero(o.f["S_g"]) > 0


def test_one_cat_carry_starts_at_zero_without_cloud_in_the_first_columns():
    """No cloud water in the first columns of the serial order: their cloud-free condensable
    cells use the carry's starting value (0), later columns the carried rate."""
    grid = (25, 46, 91)
    st = seeded_state(grid, 91)
    st["cloud"][:, :, :4] = 0.0
    out, o = run_both(grid, st, 1)
    err = rel_errors(out, o)
    bad = {n: e for n, e in err.items() if not e <= TOL}
    assert not bad, (bad, err)


@pytest.mark.parametrize("category", [0, 3])
def test_ice_scheme_keeps_mirror_symmetry(category):
    grid = (25, 46, 91)
    st = seeded_state(grid, 95, symmetric=True)
    for n in OUT:
        assert np.array_equal(st[n], mirror(st[n], False)), n
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        getattr(g, RUN[category])()
        for n in OUT:
            a = g.download(n)
            assert np.array_equal(a, mirror(a, False)), n


def test_ice_scheme_switch():
    """athad_ice_scheme runs the configured category's scheme (bit-identical to the direct
    call) and nothing for -1."""
    grid = (25, 46, 91)
    st = seeded_state(grid, 97)
    for category in (-1, 0, 1, 2, 3):
        p = config_params()
        p.category_ice_scheme = category
        with GpuAtmosphere(*grid, p) as g:
            g.upload_state(st)
            g.ice_scheme()
            via_switch = {n: g.download(n) for n in OUT}
        if category < 0:
            for n in OUT:
                assert np.array_equal(via_switch[n], st[n]), n
            continue
        with GpuAtmosphere(*grid, p) as g:
            g.upload_state(st)
            getattr(g, RUN[category])()
            for n in OUT:
                assert np.array_equal(via_switch[n], g.download(n)), (category, n)


@pytest.mark.parametrize("category", [0, 1, 3])
def test_ice_scheme_needs_level_23(category):
    """The schemes read the rain flux at level 23: a grid with im < 24 is refused before any
    launch, with the reason in the context's last error."""
    with GpuAtmosphere(21, 46, 91, config_params()) as g:
        with pytest.raises(AthadError) as e:
            getattr(g, RUN[category])()
        assert e.value.status == Status.ERR_UNSUPPORTED
        assert "im >= 24" in str(e.value)
