"""Seeded synthetic model states with the reference's shapes and value ranges.

The reference initialises from a deterministic moist-adiabat column over a symmetric
parabolic sea-surface temperature (InitValues_Atm.cpp:466-508, 843-926; ThermoAtm.h
densities(true)).  This builder produces a state of the same shape and magnitudes without
running the reference's initialiser: a surface temperature parabola from pole to equator,
a lapse-rate column capped at the skin temperature, a hydrostatic pressure, a water column
decaying to the dry top value, CO2 well mixed in the dry air, prescribed overturning
velocities and small turbulence, forcing and condensate fields.  Everything is built from
numpy with a fixed seed.

symmetric=True builds the northern half and mirrors it (v, MC_v and aux_v change sign),
so the state is exactly north-south mirror symmetric.
"""
from __future__ import annotations

import math

import numpy as np

from ._abi import FIELD_NAMES


def layer_heights(im: int, L_atm: float = 6287.5, zeta: float = 3.0) -> np.ndarray:
    """cAtmosphereModel::init_layer_heights (cAtmosphereModel.h:441-452), float-rounded."""
    dr = 1.0 / (im - 1)
    rad = np.empty(im)
    rad[0] = 1.0
    for i in range(1, im):
        rad[i] = rad[i - 1] + dr
    hL = float(np.float32(L_atm))
    return np.array([float(np.float32((math.exp(zeta * (r - rad[0])) - 1) * hL)) for r in rad])


def make_state(im: int, jm: int, km: int, seed: int = 20261203, symmetric: bool = False,
               params: dict | None = None, amp: float = 1.0) -> dict:
    p = {"t_0": 273.15, "t_surf_equator": 513.15, "t_surf_pole": 503.15, "t_skin": 254.0,
         "u_0": 8.0, "L_atm": 6287.5, "zeta": 3.0, "c_0": 0.3464, "co2_0": 0.6233,
         "c_h2o_dry_top": 0.00423, "r_air": 40.8}
    if params:
        p.update({k: v for k, v in params.items() if k in p})
    rng = np.random.default_rng(seed)
    jh = (jm + 1) // 2 if symmetric else jm       # rows generated independently
    z = layer_heights(im, p["L_atm"], p["zeta"])   # [m]
    lat = np.linspace(90.0, -90.0, jm)[:jh]        # colatitude row j -> latitude
    phi = np.linspace(0.0, 2 * np.pi, km)
    Z = z[:, None, None]
    LAT = np.deg2rad(lat)[None, :, None]
    PHI = phi[None, None, :]

    def noise(scale):
        return scale * rng.standard_normal((im, jh, km))

    # temperature: parabola at the surface, lapse to the skin temperature
    Ts = p["t_surf_pole"] + (p["t_surf_equator"] - p["t_surf_pole"]) * (1.0 - (LAT / (np.pi / 2)) ** 2)
    T = np.maximum(p["t_skin"], Ts - 5.0e-3 * Z) + amp * 0.05 * np.cos(2 * PHI) * np.exp(-Z / 30e3)
    t = T / p["t_0"] + noise(1e-6 * amp)
    # pressure [hPa]: hydrostatic with a scale height of the mixture
    Rm = 386.0
    H = Rm * T / 9.8066
    p_surf = 1e-2 * p["r_air"] * Rm * Ts
    p_stat = p_surf * np.exp(-np.cumsum(np.concatenate([np.zeros((1,) + T.shape[1:]),
                                                         np.diff(Z, axis=0) / (0.5 * (H[1:] + H[:-1]))]), axis=0))
    p_stat = np.broadcast_to(p_stat, (im, jh, km)).copy()
    # water: saturated near the sea, decaying to the dry top
    c = np.maximum(p["c_h2o_dry_top"], p["c_0"] * np.exp(-Z / 12e3)) * (1.0 + 0.02 * np.cos(PHI) * amp)
    c = np.broadcast_to(c, (im, jh, km)) + np.abs(noise(1e-7 * amp))
    co2 = p["co2_0"] * (1.0 - c) / (1.0 - p["c_0"])
    band = np.exp(-((Z - 25e3) / 8e3) ** 2)
    cloud = np.broadcast_to(1e-4 * band * (1 + 0.5 * np.sin(3 * PHI)), (im, jh, km)) + np.abs(noise(1e-8))
    ice = np.broadcast_to(5e-5 * np.exp(-((Z - 60e3) / 10e3) ** 2), (im, jh, km)) + np.abs(noise(1e-8))
    gr = np.broadcast_to(1e-6 * band, (im, jh, km)) + np.abs(noise(1e-9))
    # velocities (non-dimensional, u_0 = 8 m/s): radial u, meridional v (south-positive,
    # antisymmetric), zonal w
    cell = np.sin(np.pi * Z / Z.max())
    u = amp * 1e-3 * cell * np.cos(3 * LAT) * (1 + 0.3 * np.cos(PHI)) + noise(1e-6 * amp)
    v = -amp * 0.2 * cell * np.sin(2 * LAT) * (1 + 0.2 * np.sin(2 * PHI)) + noise(1e-5 * amp)
    w = amp * (0.8 * np.cos(LAT) ** 2 * (1 - np.exp(-Z / 5e3)) + 0.05 * np.sin(PHI)) + noise(1e-5 * amp)
    tke = np.broadcast_to(1e-3 * np.exp(-Z / 10e3) + 1e-5, (im, jh, km)) + np.abs(noise(1e-7))
    dis = np.broadcast_to(0.5 * np.exp(-Z / 20e3) + 0.05, (im, jh, km)) + np.abs(noise(1e-4))
    nue = np.broadcast_to(1e-3 * np.exp(-Z / 8e3) + 1e-5, (im, jh, km)) + np.abs(noise(1e-7))
    p_dyn = amp * 1e-3 * np.cos(2 * LAT) * np.sin(np.pi * Z / Z.max()) * (1 + 0.5 * np.cos(PHI)) + noise(1e-6 * amp)
    t_eq = t + 0.01 * np.broadcast_to(np.cos(LAT) * np.exp(-Z / 40e3), t.shape)
    r_humid = 1e2 * p_stat / (Rm * np.broadcast_to(T, (im, jh, km)))
    S = {n: 1e-8 * np.broadcast_to(band * np.cos(PHI + k), (im, jh, km)) + noise(1e-10)
         for k, n in enumerate(["S_c", "S_r", "S_i", "S_s", "S_g", "S_v"])}
    MC = {"MC_t": 1e-7 * np.broadcast_to(band, (im, jh, km)) + noise(1e-9),
          "MC_q": -1e-8 * np.broadcast_to(band, (im, jh, km)) + noise(1e-10),
          "MC_v": 1e-8 * np.broadcast_to(np.sin(2 * LAT) * band, (im, jh, km)) + noise(1e-10),
          "MC_w": 1e-8 * np.broadcast_to(band * np.cos(PHI), (im, jh, km)) + noise(1e-10)}

    st = {"t": t, "u": u, "v": v, "w": w, "c": c, "cloud": cloud, "ice": ice, "gr": gr,
          "co2": co2, "tke": tke, "dis": dis, "p_dyn": p_dyn, "nue": nue, "t_eq": t_eq,
          "p_stat": p_stat, "r_humid": r_humid}
    st.update(S)
    st.update(MC)
    # time level n differs slightly from the current state (the saturation adjustment and
    # the boundary conditions run between storeIntermediateData3D and the RK4 step)
    for n_ in ["t", "u", "v", "w", "c", "cloud", "ice", "gr", "co2", "tke", "dis"]:
        a = st[n_]
        pert = 1e-6 * rng.standard_normal(a.shape) * (np.abs(a) + 1e-6)
        b = a + pert
        if n_ in ("c", "cloud", "ice", "gr", "tke"):
            b = np.abs(b)
        if n_ == "dis":
            b = np.maximum(b, 1e-10)
        st[n_ + "n"] = b
    st["aux_u"] = np.zeros((im, jh, km))
    st["aux_v"] = np.zeros((im, jh, km))
    st["aux_w"] = np.zeros((im, jh, km))
    # the remaining fields start at zero
    out = {}
    for name in FIELD_NAMES:
        a = st.get(name)
        if a is None:
            a = np.zeros((im, jh, km))
        a = np.array(np.broadcast_to(a, (im, jh, km)), dtype=np.float64, copy=True)
        if symmetric:
            full = np.empty((im, jm, km))
            full[:, :jh, :] = a
            sign = -1.0 if name in ("v", "vn", "MC_v", "aux_v", "v_u", "v_d") else 1.0
            full[:, jh:, :] = sign * a[:, :jm - jh, :][:, ::-1, :]
            if sign < 0 and jm % 2 == 1:
                full[:, jm // 2, :] = 0.0
            a = full
        out[name] = a
    return out


def mirror(a: np.ndarray, antisymmetric: bool = False) -> np.ndarray:
    """field(i, jm-1-j, k) (negated for the meridional components)."""
    m = a[:, ::-1, :]
    return -m if antisymmetric else m


def make_state_device(im: int, jm: int, km: int, seed: int = 20261203, params: dict | None = None,
                      device=None, amp: float = 1.0) -> dict:
    """make_state's fields built with torch on a CUDA device (a serving loop admits runs
    faster than numpy builds their states).  Same formulas and magnitudes; the noise comes
    from torch's seeded generator, so the values differ from make_state's.  Returns packed
    (im, jm, km) float64 tensors for GpuAtmosphere.upload_tensor; 2-D fields as (jm, km)."""
    import torch
    p = {"t_0": 273.15, "t_surf_equator": 513.15, "t_surf_pole": 503.15, "t_skin": 254.0,
         "u_0": 8.0, "L_atm": 6287.5, "zeta": 3.0, "c_0": 0.3464, "co2_0": 0.6233,
         "c_h2o_dry_top": 0.00423, "r_air": 40.8}
    if params:
        p.update({k: v for k, v in params.items() if k in p})
    dev = torch.device(device) if device is not None else torch.device("cuda")
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(seed))
    f64 = dict(dtype=torch.float64, device=dev)
    shape = (im, jm, km)
    z = torch.tensor(layer_heights(im, p["L_atm"], p["zeta"]), **f64)
    lat = torch.linspace(90.0, -90.0, jm, **f64)
    phi = torch.linspace(0.0, 2 * math.pi, km, **f64)
    Z = z[:, None, None]
    LAT = torch.deg2rad(lat)[None, :, None]
    PHI = phi[None, None, :]

    def noise(scale):
        return scale * torch.randn(shape, generator=gen, **f64)

    def full(a):
        return torch.broadcast_to(a, shape).contiguous()

    Ts = p["t_surf_pole"] + (p["t_surf_equator"] - p["t_surf_pole"]) * (1.0 - (LAT / (math.pi / 2)) ** 2)
    T = torch.clamp(Ts - 5.0e-3 * Z, min=p["t_skin"]) + amp * 0.05 * torch.cos(2 * PHI) * torch.exp(-Z / 30e3)
    T = full(T)
    t = T / p["t_0"] + noise(1e-6 * amp)
    Rm = 386.0
    H = Rm * T / 9.8066
    p_surf = 1e-2 * p["r_air"] * Rm * full(Ts)[0]
    dz = (Z[1:] - Z[:-1])
    steps = dz / (0.5 * (H[1:] + H[:-1]))
    cum = torch.cat([torch.zeros((1, jm, km), **f64), torch.cumsum(steps, dim=0)], dim=0)
    p_stat = p_surf[None] * torch.exp(-cum)
    c = full(torch.clamp(p["c_0"] * torch.exp(-Z / 12e3), min=p["c_h2o_dry_top"]) * (1.0 + 0.02 * torch.cos(PHI) * amp))
    c = c + torch.abs(noise(1e-7 * amp))
    co2 = p["co2_0"] * (1.0 - c) / (1.0 - p["c_0"])
    band = torch.exp(-((Z - 25e3) / 8e3) ** 2)
    cloud = full(1e-4 * band * (1 + 0.5 * torch.sin(3 * PHI))) + torch.abs(noise(1e-8))
    ice = full(5e-5 * torch.exp(-((Z - 60e3) / 10e3) ** 2)) + torch.abs(noise(1e-8))
    gr = full(1e-6 * band) + torch.abs(noise(1e-9))
    cell = torch.sin(math.pi * Z / Z.max())
    u = full(amp * 1e-3 * cell * torch.cos(3 * LAT) * (1 + 0.3 * torch.cos(PHI))) + noise(1e-6 * amp)
    v = full(-amp * 0.2 * cell * torch.sin(2 * LAT) * (1 + 0.2 * torch.sin(2 * PHI))) + noise(1e-5 * amp)
    w = full(amp * (0.8 * torch.cos(LAT) ** 2 * (1 - torch.exp(-Z / 5e3)) + 0.05 * torch.sin(PHI))) + noise(1e-5 * amp)
    tke = full(1e-3 * torch.exp(-Z / 10e3) + 1e-5) + torch.abs(noise(1e-7))
    dis = full(0.5 * torch.exp(-Z / 20e3) + 0.05) + torch.abs(noise(1e-4))
    nue = full(1e-3 * torch.exp(-Z / 8e3) + 1e-5) + torch.abs(noise(1e-7))
    p_dyn = full(amp * 1e-3 * torch.cos(2 * LAT) * torch.sin(math.pi * Z / Z.max()) * (1 + 0.5 * torch.cos(PHI))) + noise(1e-6 * amp)
    t_eq = t + 0.01 * full(torch.cos(LAT) * torch.exp(-Z / 40e3))
    r_humid = 1e2 * p_stat / (Rm * T)
    st = {"t": t, "u": u, "v": v, "w": w, "c": c, "cloud": cloud, "ice": ice, "gr": gr,
          "co2": co2, "tke": tke, "dis": dis, "p_dyn": p_dyn, "nue": nue, "t_eq": t_eq,
          "p_stat": p_stat.contiguous(), "r_humid": r_humid}
    for k_, n in enumerate(["S_c", "S_r", "S_i", "S_s", "S_g", "S_v"]):
        st[n] = full(1e-8 * band * torch.cos(PHI + k_)) + noise(1e-10)
    st["MC_t"] = full(1e-7 * band) + noise(1e-9)
    st["MC_q"] = full(-1e-8 * band) + noise(1e-10)
    st["MC_v"] = full(1e-8 * torch.sin(2 * LAT) * band) + noise(1e-10)
    st["MC_w"] = full(1e-8 * band * torch.cos(PHI)) + noise(1e-10)
    for n_ in ["t", "u", "v", "w", "c", "cloud", "ice", "gr", "co2", "tke", "dis"]:
        a = st[n_]
        b = a + 1e-6 * torch.randn(shape, generator=gen, **f64) * (torch.abs(a) + 1e-6)
        if n_ in ("c", "cloud", "ice", "gr", "tke"):
            b = torch.abs(b)
        if n_ == "dis":
            b = torch.clamp(b, min=1e-10)
        st[n_ + "n"] = b
    st["Evaporation"] = torch.full((jm, km), 20.0, **f64)
    return {k: (v.contiguous() if v.dim() == 3 else v) for k, v in st.items()}
