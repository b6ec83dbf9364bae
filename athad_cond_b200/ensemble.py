"""Ensemble members and serving requests: seeded grids and condition points.

A condition point is a surface pressure p_surf [bar], a sea-surface temperature T_sea [K]
and a dry-air composition (H2O, CO2, N2 mole fractions).  As in the reference's nominal
column (test/cond_column_selftest.cpp:66-145): the surface air is saturated over the sea,
x_H2O = p_sat(T_sea) / p_surf, the rest split in the dry CO2:N2 ratio; the model constants
follow from AtmMixture::resolve (atmosphere/MixtureAtm.h:82-109) of that surface
composition (c_0 = q_H2O, co2_0 = q_CO2, R_mix, M_bg, R_bg) and of the dry composition
(c_h2o_dry_top = q_H2O); r_air = p_surf / (R_mix T_sea), so ThermoAtm::densities' surface
anchor 1e-2 r_air R_mix T_sea gives back p_surf.  T_sea is redrawn until it is at least
0.5 K below the boiling point at p_surf.

Everything is drawn from numpy's PCG64 with a fixed seed, so a member list is reproducible.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

import ctypes

from ._abi import InitConfig, Params, Precision, config_init, config_params

R_STAR = 8.314462618
M_H2O, M_CO2, M_N2 = 0.018015, 0.044010, 0.028014
T_CRIT = 647.096


def saturation_pressure(T: float) -> float:
    """Wagner & Pruss saturation line [hPa] (atmosphere/SaturationH2O.h:68-93)."""
    if T >= T_CRIT:
        return -1.0
    th = 1.0 - T / T_CRIT
    sq = math.sqrt(th)
    t3 = th * th * th
    s = (-7.85951783 * th + 1.84408259 * th * sq - 11.7866497 * t3 + 22.6807411 * t3 * sq
         - 15.9618719 * t3 * th + 1.80122502 * t3 * th * t3 * sq)
    return 220640.0 * math.exp(T_CRIT / T * s)


def boiling_point(p_hpa: float) -> float:
    """Temperature at which p_sat = p (SaturationH2O::dewPoint), by bisection."""
    lo, hi = 273.16, T_CRIT - 1e-9
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if saturation_pressure(mid) < p_hpa:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def resolve(x_h2o: float, x_co2: float, x_n2: float) -> dict:
    """AtmMixture::resolve for an H2O/CO2/N2 mixture (MixtureAtm.h:82-109)."""
    m_h2o, m_co2, m_bg = x_h2o * M_H2O, x_co2 * M_CO2, x_n2 * M_N2
    M_mean = m_h2o + m_co2 + m_bg
    M_bg = (m_bg / x_n2) if x_n2 > 0 else M_N2
    return {"M_mean": M_mean, "R_mix": R_STAR / M_mean, "q_H2O": m_h2o / M_mean,
            "q_CO2": m_co2 / M_mean, "q_bg": m_bg / M_mean, "M_bg": M_bg, "R_bg": R_STAR / M_bg}


@dataclass
class Condition:
    p_surf_bar: float
    T_sea: float
    x_dry: tuple          # (H2O, CO2, N2), renormalised
    x_surf: tuple = field(default=())
    surf: dict = field(default_factory=dict)
    dry: dict = field(default_factory=dict)
    r_air: float = 0.0


def draw_condition(rng: np.random.Generator) -> Condition:
    """p_surf ~ U[40, 100] bar; T_sea ~ U[503, 523] K redrawn until <= T_boil - 0.5 K;
    dry H2O ~ U[0.4, 2] %, CO2 ~ U[89, 95] %, N2 ~ U[5, 20] %, renormalised."""
    p_surf = float(rng.uniform(40.0, 100.0))
    t_boil = boiling_point(p_surf * 1000.0)
    while True:
        T_sea = float(rng.uniform(503.0, 523.0))
        if T_sea <= t_boil - 0.5:
            break
    x = np.array([rng.uniform(0.004, 0.02), rng.uniform(0.89, 0.95), rng.uniform(0.05, 0.20)])
    x = tuple(float(v) for v in x / x.sum())
    x_h2o_s = saturation_pressure(T_sea) / (p_surf * 1000.0)
    rest = 1.0 - x_h2o_s
    x_surf = (x_h2o_s, rest * x[1] / (x[1] + x[2]), rest * x[2] / (x[1] + x[2]))
    surf = resolve(*x_surf)
    dry = resolve(*x)
    r_air = p_surf * 1.0e5 / (surf["R_mix"] * T_sea)
    return Condition(p_surf, T_sea, x, x_surf, surf, dry, r_air)


def condition_params(cond: Condition, precision: Precision = Precision.MIXED) -> Params:
    """athad_params of a condition point (the cli/config_cond.xml values otherwise)."""
    p = config_params()
    p.precision = int(precision)
    p.p_0 = cond.p_surf_bar * 1000.0
    p.r_air = cond.r_air
    p.c_0 = cond.surf["q_H2O"]
    p.co2_0 = cond.surf["q_CO2"]
    p.c_h2o_dry_top = cond.dry["q_H2O"]
    p.R_mix = cond.surf["R_mix"]
    p.M_bg = cond.surf["M_bg"]
    p.R_bg = cond.surf["R_bg"]
    return p


def init_config(cond: Condition) -> InitConfig:
    """athad_init_config of a condition point: the sea surface at T_sea on the equator with the
    configuration's 10 K equator-to-pole contrast (513.15 / 503.15 K), the CO2 share of the
    non-water surface air; the cli/config_cond.xml values otherwise."""
    c = config_init()
    c.struct_size = ctypes.sizeof(InitConfig)
    c.t_surf_equator = cond.T_sea
    c.t_surf_pole = cond.T_sea - 10.0
    c.q_CO2 = cond.surf["q_CO2"]
    c.q_bg = cond.surf["q_bg"]
    return c


def state_params(cond: Condition) -> dict:
    """Inputs of synthetic.make_state for this condition point."""
    return {"t_surf_equator": cond.T_sea, "t_surf_pole": cond.T_sea - 10.0, "r_air": cond.r_air,
            "c_0": cond.surf["q_H2O"], "co2_0": cond.surf["q_CO2"],
            "c_h2o_dry_top": cond.dry["q_H2O"]}


def odd_uniform(rng: np.random.Generator, lo: int, hi: int) -> int:
    """An odd integer uniform over the odd values of [lo, hi] (odd jm and km keep an
    equator row and a seam meridian)."""
    lo_o = lo if lo % 2 else lo + 1
    hi_o = hi if hi % 2 else hi - 1
    return lo_o + 2 * int(rng.integers(0, (hi_o - lo_o) // 2 + 1))


@dataclass
class MemberSpec:
    index: int
    grid: tuple
    cond: Condition
    seed: int


def draw_ensemble(n: int = 64, seed: int = 20261203, im=(21, 41), jm=(61, 181), km=(121, 361)):
    """n members with uneven grids (im uniform, jm and km odd-uniform) and condition points."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(n):
        grid = (int(rng.integers(im[0], im[1] + 1)), odd_uniform(rng, *jm), odd_uniform(rng, *km))
        out.append(MemberSpec(q, grid, draw_condition(rng), seed + 1000 + q))
    return out
