"""athad_pressure_solve: the pressure-Poisson equation of the sweep solved to a tolerance.

The check is independent of the solver: numpy restates the sweep's operator and source
(PressureSolverAtm.h:236-281 and :415-473 with the metric fix, flat terrain) from the grid
alone, applies it to the p_dyn the solver returned (its boundary cells set by the sweep's
boundary conditions) and measures ||b - A p|| / ||b|| with b the source projected onto the
operator's range.  Stated tolerance: the solve's target 1e-10, checked on the host to 1e-9
(the host's own rounding).  Also: the solution is a fixed point of the reference sweep
(one oracle sweep moves it only by the projected-out constant of the source), a
mirror-symmetric source gives a mirror-symmetric solution (1e-8 of its size), and the
report's history decreases to the target.
"""
import math

import numpy as np
import pytest

from athad_cond_b200 import GpuAtmosphere, make_state, mirror
from athad_cond_b200._abi import config_params
from oracle_binding import OracleState

pytestmark = pytest.mark.gpu


def operator(im, jm, km, p=None):
    """Per-(i, j) coefficients of the sweep, as the context builds them."""
    p = p or config_params()
    pi180 = 180.0 / math.pi
    dr = 1.0 / (im - 1)
    dthe = (180.0 / (jm - 1)) / pi180
    dphi = (360.0 / (km - 1)) / pi180
    rad = [1.0]
    for _ in range(1, im):
        rad.append(rad[-1] + dr)
    the = [0.0]
    for _ in range(1, jm):
        the.append(the[-1] + dthe)
    rad, the = np.array(rad), np.array(the)
    jj = np.minimum(np.arange(jm), jm - 1 - np.arange(jm))
    sin_f = np.maximum(0.55, np.sin(the[jj]))
    cos_t = np.where(np.arange(jm) < jm - 1 - np.arange(jm), np.cos(the[jj]),
                     np.where(np.arange(jm) > jm - 1 - np.arange(jm), -np.cos(the[jj]), 0.0))
    span = rad[-1] - rad[0]
    shell = (math.exp(p.zeta * span) - 1.0) * p.L_atm / span
    r0 = p.r_Earth * 1e3 / shell
    rm = rad[:, None]
    rmet = r0 + (rm - rad[0])
    exp_rm = 1.0 / (rm + 1.0)
    exp_2_rm = exp_rm * exp_rm
    inv_rm = 1.0 / rmet
    inv_rm2 = 1.0 / (rmet * rmet)
    s2 = sin_f[None, :] ** 2
    inv_rm2sinthe2 = inv_rm2 / s2
    inv_rmsinthe = 1.0 / (rmet * sin_f[None, :])
    num1 = np.broadcast_to(exp_2_rm / dr ** 2, (im, jm))
    num2 = np.broadcast_to(inv_rm2 / dthe ** 2, (im, jm))
    num3 = inv_rm2sinthe2 / dphi ** 2
    denom = 2 * num1 + 2 * num2 + 2 * num3
    return dict(dr=dr, dthe=dthe, dphi=dphi, exp_rm=np.broadcast_to(exp_rm, (im, jm)),
                inv_rm=np.broadcast_to(inv_rm, (im, jm)), inv_rmsinthe=inv_rmsinthe,
                num1=num1, num2=num2, num3=num3, denom=denom, cos_t=cos_t)


def source(op, u, v, w):
    """Clamped divergence source of the interior cells (aux boundary copies first)."""
    u, v, w = u.copy(), v.copy(), w.copy()
    for a in (u, v, w):
        a[0], a[-1] = a[1], a[-2]
    I, J, K = slice(1, -1), slice(1, -1), slice(1, -1)
    du = (u[2:, J, K] - u[:-2, J, K]) / (2 * op["dr"])
    dv = (v[I, 2:, K] - v[I, :-2, K]) / (2 * op["dthe"])
    dw = (w[I, J, 2:] - w[I, J, :-2]) / (2 * op["dphi"])
    src = du * op["exp_rm"][I, J, None] + dv * op["inv_rm"][I, J, None] + dw * op["inv_rmsinthe"][I, J, None]
    cap = 2.0 * op["denom"][I, J, None]
    return np.clip(src, -cap, cap)


def relative_residual(op, p, src):
    I = slice(1, -1)
    n1, n2, n3, dn = (op[k][I, I, None] for k in ("num1", "num2", "num3", "denom"))
    Ap = (dn * p[I, I, I] - n1 * (p[2:, I, I] + p[:-2, I, I]) - n2 * (p[I, 2:, I] + p[I, :-2, I])
          - n3 * (p[I, I, 2:] + p[I, I, :-2]))
    bS = -src / n1
    bS = bS - bS.mean()
    rS = bS - Ap / n1
    return float(np.linalg.norm(rS * n1) / np.linalg.norm(bS * n1))


def perturbation(grid, seed, symmetric):
    im, jm, km = grid
    rng = np.random.default_rng(seed)
    st = make_state(im, jm, km, seed=seed, symmetric=symmetric)
    jh = (jm + 1) // 2
    out = {}
    for n, anti in (("aux_u", False), ("aux_v", True), ("aux_w", False)):
        a = 0.5 / 8.0 * rng.standard_normal((im, jh if symmetric else jm, km))
        if symmetric:
            full = np.empty((im, jm, km))
            full[:, :jh] = a
            full[:, jh:] = (-1.0 if anti else 1.0) * a[:, :jm - jh][:, ::-1]
            if anti:
                full[:, jm // 2] = 0.0
            a = full
        out[n] = a
    st.update(out)
    st["p_dyn"] = np.zeros((im, jm, km))
    return st


@pytest.mark.parametrize("grid", [(11, 21, 41), (21, 91, 181)])
def test_solve_reaches_the_tolerance_on_the_reference_operator(grid):
    st = perturbation(grid, 3, symmetric=False)
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        rep = g.pressure_solve(1e-10, 200)
        p = g.download("p_dyn")
    assert rep["converged"] and rep["rel_residual"] <= 1e-10
    hist = [h for h in rep["history"][:rep["iterations"]]]
    assert hist[-1] <= 1e-10 and hist[0] > hist[-1]
    op = operator(*grid)
    src = source(op, st["aux_u"], st["aux_v"], st["aux_w"])
    assert relative_residual(op, p, src) <= 1e-9
    assert abs(p[1:-1, 1:-1, 1:-1].mean()) <= 1e-12 * max(1.0, np.abs(p).max())


def test_solution_is_a_fixed_point_of_the_reference_sweep():
    grid = (11, 21, 41)
    st = perturbation(grid, 4, symmetric=False)
    for n in ("aux_u", "aux_v", "aux_w"):
        st[n] *= 0.1                     # keeps |p| below the sweep's ceiling of 10
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        g.pressure_solve(1e-12, 300)
        p = g.download("p_dyn")
        aux = {n: g.download(n) for n in ("aux_u", "aux_v", "aux_w")}
    # The solve returns A p = -src - mu num1(i) (the source projected onto the range,
    # mu = mean of -src / num1), so one sweep with the sweep's own source moves p by at most
    # about mu num1 / denom per colour: nothing else may move.
    s2 = dict(st)
    s2.update(aux)
    s2["p_dyn"] = p.copy()
    o = OracleState(s2, config_params())
    o.pressure_sweep(n_sweeps=1, total_iter_count=0)
    op = operator(*grid)
    src = source(op, aux["aux_u"], aux["aux_v"], aux["aux_w"])
    mu = float(np.mean(-src / op["num1"][1:-1, 1:-1, None]))
    ratio = float(np.max(op["num1"] / op["denom"]))
    moved = float(np.abs(o.f["p_dyn"] - p)[1:-1, 1:-1, 1:-1].max())
    assert moved <= 2.0 * abs(mu) * ratio + 1e-8 * float(np.abs(p).max())


@pytest.mark.parametrize("grid", [(11, 21, 41), (21, 91, 181)])
def test_symmetric_source_gives_symmetric_solution(grid):
    st = perturbation(grid, 5, symmetric=True)
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        rep = g.pressure_solve(1e-10, 200)
        p = g.download("p_dyn")
    assert rep["converged"]
    assert float(np.max(np.abs(p - mirror(p)))) <= 1e-8 * float(np.max(np.abs(p)))


def test_zero_source_returns_zero():
    grid = (11, 21, 41)
    st = perturbation(grid, 6, symmetric=False)
    for n in ("aux_u", "aux_v", "aux_w"):
        st[n] = np.zeros(grid)
    with GpuAtmosphere(*grid, config_params()) as g:
        g.upload_state(st)
        rep = g.pressure_solve(1e-10, 10)
        assert rep["iterations"] == 0 and np.array_equal(g.download("p_dyn"), np.zeros(grid))
