"""ctypes binding of the oracle (oracle/liboracle.so), the CPU checker of the tests.

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
use it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from athad_cond_b200._abi import FIELD, FIELD_NAMES, FIELD2D_NAMES, PROFILE_NAMES, InitConfig, Params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB = os.path.join(ORACLE_DIR, "liboracle.so")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
        _lib = ctypes.CDLL(LIB)
        _lib.or_params_size.restype = ctypes.c_size_t
        assert _lib.or_params_size() == ctypes.sizeof(Params), "oracle params layout differs"
        _lib.or_nfields.restype = ctypes.c_int
        assert _lib.or_nfields() == len(FIELD_NAMES)
        _lib.or_init_cfg_size.restype = ctypes.c_size_t
        assert _lib.or_init_cfg_size() == ctypes.sizeof(InitConfig), "oracle init config layout differs"
        for name in ["or_saturation_pressure", "or_sublimation_pressure", "or_latent_heat",
                     "or_dew_point"]:
            fn = getattr(_lib, name)
            fn.restype = ctypes.c_double
            fn.argtypes = [ctypes.c_double]
        _lib.or_saturation_mass_fraction.restype = ctypes.c_double
        _lib.or_saturation_mass_fraction.argtypes = [ctypes.c_double] * 3
        _lib.or_dqsat_dT.restype = ctypes.c_double
        _lib.or_dqsat_dT.argtypes = [ctypes.c_double] * 3
        _lib.or_moist_lapse.restype = ctypes.c_double
        _lib.or_moist_lapse.argtypes = [ctypes.c_double] * 6
        _lib.or_cp_of.restype = ctypes.c_double
        _lib.or_cp_of.argtypes = [ctypes.c_double] * 4
        _lib.or_R_of.restype = ctypes.c_double
        _lib.or_R_of.argtypes = [ctypes.c_double] * 3
        _lib.or_M_nonwater.restype = ctypes.c_double
        _lib.or_M_nonwater.argtypes = [ctypes.c_double] * 3
    return _lib


def update_skin_temperature(params, albedo, t_skin, relax):
    """or_update_skin_temperature: cAtmosphereModel::updateSkinTemperature on a (jm, km)
    albedo."""
    a = np.ascontiguousarray(albedo, dtype=np.float64)
    fn = lib().or_update_skin_temperature
    fn.restype = ctypes.c_double
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                   ctypes.c_double, ctypes.c_double]
    return fn(a.shape[0], a.shape[1], ctypes.byref(params), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
              t_skin, relax)


class Step(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("diffusion_ramp", ctypes.c_double),
                ("buoyancy_ramp", ctypes.c_double), ("write_diagnostics", ctypes.c_int32),
                ("pad0", ctypes.c_int32)]


def _ptrs(state: dict, names, shape):
    arr = (ctypes.POINTER(ctypes.c_double) * len(names))()
    keep = []
    for q, n in enumerate(names):
        a = state.get(n)
        if a is None:
            a = np.zeros(shape)
            state[n] = a
        assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], n
        keep.append(a)
        arr[q] = a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    return arr, keep


class OracleState:
    """Host copy of every field, advanced by the oracle in place."""

    def __init__(self, state: dict, params: Params):
        any_ = next(iter(v for k, v in state.items() if k in FIELD))
        self.shape = any_.shape
        self.params = params
        im, jm, km = self.shape
        self.f = {n: np.array(state[n], dtype=np.float64, copy=True) if n in state else np.zeros(self.shape)
                  for n in FIELD_NAMES}
        self.f2 = {n: np.array(state[n], dtype=np.float64, copy=True) if n in state else np.zeros((jm, km))
                   for n in FIELD2D_NAMES}
        self.prof = {n: np.array(state[n], dtype=np.float64, copy=True) if n in state else np.zeros(im)
                     for n in PROFILE_NAMES}

    @classmethod
    def initial(cls, im, jm, km, params: Params, cfg: InitConfig, compat=0, upto=99):
        """The reference's initial state built by the oracle (or_init_state): RunTimeSlice up
        to stage `upto` (OR_INIT_*, 99 = everything)."""
        o = cls({"t": np.zeros((im, jm, km))}, params)
        F, F2, P = o._args()
        r = lib().or_init_state(im, jm, km, ctypes.byref(params), ctypes.byref(cfg), int(compat), int(upto),
                                F, F2, P)
        assert r == 0, f"or_init_state returned {r}"
        return o

    def tropopause_layers(self, cfg: InitConfig):
        im, jm, _ = self.shape
        out = np.zeros(jm)
        lib().or_tropopause_layers(im, jm, ctypes.byref(self.params), ctypes.byref(cfg),
                                   out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def _args(self):
        self._F, self._kf = _ptrs(self.f, FIELD_NAMES, self.shape)
        self._F2, self._k2 = _ptrs(self.f2, FIELD2D_NAMES, self.shape[1:])
        self._P, self._kp = _ptrs(self.prof, PROFILE_NAMES, (self.shape[0],))
        return self._F, self._F2, self._P

    def rk4(self, dt=4e-5, diffusion_ramp=1.0, buoyancy_ramp=1.0, write_diagnostics=False, compat=0):
        F, _, P = self._args()
        im, jm, km = self.shape
        s = Step(dt, diffusion_ramp, buoyancy_ramp, int(write_diagnostics), 0)
        r = lib().or_rk4(im, jm, km, ctypes.byref(self.params), ctypes.byref(s), compat, F, P)
        assert r == 0

    def rhs_cell(self, i, j, k, dt=4e-5, diffusion_ramp=1.0, buoyancy_ramp=1.0, compat=0):
        F, _, P = self._args()
        im, jm, km = self.shape
        s = Step(dt, diffusion_ramp, buoyancy_ramp, 0, 0)
        out = (ctypes.c_double * 17)()
        lib().or_rhs_cell_at(im, jm, km, ctypes.byref(self.params), ctypes.byref(s), compat, F, P,
                             int(i), int(j), int(k), out)
        return np.array(list(out))

    def level_mean(self, compat=0):
        F, _, P = self._args()
        im, jm, km = self.shape
        lib().or_level_mean(im, jm, km, ctypes.byref(self.params), compat, F, P)

    def pressure_sweep(self, n_sweeps=1, total_iter_count=4, compat=0):
        F, _, P = self._args()
        im, jm, km = self.shape
        cnt = (ctypes.c_int64 * 2)()
        lib().or_pressure_sweep(im, jm, km, ctypes.byref(self.params), compat, n_sweeps,
                                total_iter_count, F, P, cnt)
        return int(cnt[0]), int(cnt[1])

    def project_initial_velocity(self, n_sweeps=200, total_iter_count=0, compat=0):
        F, _, P = self._args()
        im, jm, km = self.shape
        lib().or_project_initial_velocity(im, jm, km, ctypes.byref(self.params), compat, n_sweeps,
                                          total_iter_count, F, P)

    def saturation_adjust(self, compat=0):
        F, _, _ = self._args()
        im, jm, km = self.shape
        cnt = (ctypes.c_int64 * 1)()
        lib().or_saturation_adjust(im, jm, km, ctypes.byref(self.params), compat, F, cnt)
        return int(cnt[0])

    def densities(self, set_water_profile=False, compat=0):
        F, F2, P = self._args()
        im, jm, km = self.shape
        lib().or_densities(im, jm, km, ctypes.byref(self.params), compat, 1 if set_water_profile else 0,
                           F, F2, P)

    def moist_convection(self, iter_n, compat=0):
        F, F2, _ = self._args()
        im, jm, km = self.shape
        return lib().or_moist_convection(im, jm, km, ctypes.byref(self.params), compat, iter_n, F, F2)

    def moist_geometry(self, compat=0):
        """The layer heights, level steps and cos(theta_equator - theta_j) that
        moist_convection uses (or_moist_geometry)."""
        im, jm, km = self.shape
        h, s, c = np.zeros(im), np.zeros(im), np.zeros(jm)
        P = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        r = lib().or_moist_geometry(im, jm, km, ctypes.byref(self.params), compat, P(h), P(s), P(c))
        assert r == 0
        return h, s, c

    def column_geometry(self, compat=0):
        """The layer heights and the saturation adjustment's level steps (or_column_geometry)."""
        im, jm, km = self.shape
        h, s = np.zeros(im), np.zeros(im)
        P = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        assert lib().or_column_geometry(im, jm, km, ctypes.byref(self.params), compat, P(h), P(s)) == 0
        return h, s

    def store_n_level(self):
        F, _, _ = self._args()
        im, jm, km = self.shape
        lib().or_store_n_level(im, jm, km, F)

    def boundary_conditions(self):
        """or_boundary_conditions: bcRadius, apply_wall_bc, bcTheta, bcPhi."""
        F, F2, _ = self._args()
        im, jm, km = self.shape
        lib().or_boundary_conditions(im, jm, km, ctypes.byref(self.params), F, F2)

    def post_rk4_filters(self):
        """polar zonal filter of u, v, w; radial Shapiro filters (flat terrain)."""
        F, _, _ = self._args()
        im, jm, km = self.shape
        lib().or_post_rk4_filters(im, jm, km, ctypes.byref(self.params), F)

    def turbulence_run(self, compat=0):
        """or_turbulence_run: TurbulenceAtm::run; compat=1 the reference's serial sweep."""
        F, F2, _ = self._args()
        im, jm, km = self.shape
        lib().or_turbulence_run(im, jm, km, ctypes.byref(self.params), int(compat), F, F2)

    def min_max(self, name) -> dict:
        im, jm, km = self.shape
        out = (ctypes.c_double * 2)()
        idx = (ctypes.c_int * 6)()
        a = np.ascontiguousarray(self.f[name])
        lib().or_min_max(im, jm, km, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out, idx)
        return {"max": out[0], "min": out[1], "at_max": tuple(idx[0:3]), "at_min": tuple(idx[3:6])}

    def find_residuum(self) -> dict:
        """or_find_residuum: UtilsAtm::findResiduumAtm."""
        F, _, _ = self._args()
        im, jm, km = self.shape
        out = (ctypes.c_double * 3)()
        cnt = (ctypes.c_int64 * 2)()
        idx = (ctypes.c_int * 6)()
        lib().or_find_residuum(im, jm, km, F, out, cnt, idx)
        return {"residuum": out[0], "avg_abs": out[1], "avg_rel": out[2], "n_cells": cnt[0],
                "n_nonfinite": cnt[1], "at": tuple(idx[0:3]), "first_nonfinite": tuple(idx[3:6])}

    def budgets(self) -> dict:
        """or_co2_column and or_water_budget, finished as the reference's first calls finish
        them (ThermoAtm.h:1016-1031, 1126-1127): the references those calls would set."""
        F, F2, _ = self._args()
        im, jm, km = self.shape
        co2 = (ctypes.c_double * 2)()
        lib().or_co2_column(im, jm, km, ctypes.byref(self.params), F, F2, co2)
        w = (ctypes.c_double * 2)()
        qbar, abar, lev = np.zeros(im), np.zeros(im), np.zeros(im)
        dp = ctypes.POINTER(ctypes.c_double)
        lib().or_water_budget(im, jm, km, ctypes.byref(self.params), F, w, qbar.ctypes.data_as(dp),
                              abar.ctypes.data_as(dp), lev.ctypes.data_as(dp))
        q_co2 = co2[0] / co2[1] if co2[1] > 0 else 0.0
        q_h2o = w[0] / w[1] if w[1] > 0 else 0.0
        qf_num = qf_den = 0.0
        for i in range(im):
            qf_num += abar[i] * qbar[i]
            qf_den += abar[i]
        q_fixed = qf_num / qf_den if qf_den > 0 else 0.0
        levels = lev / w[1] if w[1] > 0 else np.zeros(im)
        return {"q_co2_ref": q_co2, "q_h2o_ref": q_h2o, "q_h2o_fixed_ref": q_fixed,
                "air_levels": abar, "h2o_levels": levels, "qbar": qbar}

    def water_vapour_evaporation(self):
        """or_water_vapour_evaporation: ThermoAtm::waterVapourEvaporation."""
        F, F2, _ = self._args()
        im, jm, km = self.shape
        lib().or_water_vapour_evaporation(im, jm, km, ctypes.byref(self.params), F, F2)

    def latent_sensible_heat(self, compat=0):
        """or_latent_sensible_heat: ThermoAtm::latentSensibleHeat; compat=1 the reference's
        (not mirror-exact) sin table."""
        F, _, _ = self._args()
        im, jm, km = self.shape
        lib().or_latent_sensible_heat(im, jm, km, ctypes.byref(self.params), int(compat), F)

    def stand_atm_dew_point(self, i_trop):
        """or_stand_atm_dew_point: ThermoAtm::standAtm_DewPoint_HumidRel with the rows'
        tropopause levels i_trop (the equator row's already taken from its neighbour)."""
        F, _, _ = self._args()
        im, jm, km = self.shape
        lev = (ctypes.c_int * jm)(*[int(x) for x in i_trop])
        lib().or_stand_atm_dew_point(im, jm, km, ctypes.byref(self.params), F, lev)

    def forces(self, compat=0, with_level_mean=True):
        """or_forces: ThermoAtm::forces' Coriolis and buoyancy arrays; the buoyancy reference
        the level mean of prof (or 1 without one)."""
        F, _, P = self._args()
        im, jm, km = self.shape
        tr = P[0] if with_level_mean else None
        lib().or_forces(im, jm, km, ctypes.byref(self.params), int(compat), F, tr)

    def moist_caps(self):
        F, _, _ = self._args()
        im, jm, km = self.shape
        lib().or_moist_caps(im, jm, km, ctypes.byref(self.params), F)

    def vapour_ceiling(self) -> dict:
        F, _, _ = self._args()
        im, jm, km = self.shape
        n, q, w = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
        lib().or_vapour_ceiling(im, jm, km, ctypes.byref(self.params), F, ctypes.byref(n),
                                ctypes.byref(q), ctypes.byref(w))
        return {"n_ceiling": n.value, "q_clipped": q.value, "w_air": w.value}

    def multilayer_radiation(self):
        F, F2, _ = self._args()
        im, jm, km = self.shape
        lib().or_multilayer_radiation(im, jm, km, ctypes.byref(self.params), F, F2)

    def radiative_heating(self, omega_rad=0.05):
        F, F2, _ = self._args()
        im, jm, km = self.shape
        fn = lib().or_radiative_heating
        fn.argtypes = None
        fn(im, jm, km, ctypes.byref(self.params), ctypes.c_double(omega_rad), F, F2)

    def two_cat_ice_scheme(self):
        """or_two_cat_ice_scheme: TwoCatIceScheme::run."""
        F, _, _ = self._args()
        im, jm, km = self.shape
        lib().or_two_cat_ice_scheme(im, jm, km, ctypes.byref(self.params), F)

    def ice_scheme(self, category=None):
        """or_zero/one/two/three_cat_ice_scheme: the CategoryIceScheme switch for `category`
        (default: params.category_ice_scheme; -1 runs nothing)."""
        if category is None:
            category = self.params.category_ice_scheme
        if category < 0:
            return
        F, _, _ = self._args()
        im, jm, km = self.shape
        name = ("or_zero_cat_ice_scheme", "or_one_cat_ice_scheme", "or_two_cat_ice_scheme",
                "or_three_cat_ice_scheme")[category]
        getattr(lib(), name)(im, jm, km, ctypes.byref(self.params), F)

    def damp_wiggles(self, name, compat=0):
        """or_damp_wiggles: AtomUtils::damp_wiggles; compat=1 the reference's summation order
        in the j pass, 0 the mirror-exact one of the device."""
        im, jm, km = self.shape
        a = self.f[name]
        lib().or_damp_wiggles(im, jm, km, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(compat))
