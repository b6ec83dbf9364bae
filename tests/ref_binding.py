"""ctypes binding of the reference itself, built from its sources into oracle/_ref/ by
oracle/ref/Makefile (test infrastructure: it pins the oracle)."""
from __future__ import annotations

import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def lib_path(variant: str = "pin") -> str:
    """pin: the reference (IEEE build); stock: its own Makefile flags; dropin: the IEEE build
    plus the product's C++ drop-in adapter (needs the product library)."""
    if variant == "dropin":
        return os.path.join(REF_DIR, "pin", "libathad_dropin.so")
    return os.path.join(REF_DIR, variant, "libathad_ref.so")


def available(variant: str = "pin") -> bool:
    return os.path.exists(lib_path(variant))


class Reference:
    """One cAtmosphereModel of the reference (grid fixed at 61 x 181 x 361)."""

    def __init__(self, variant: str = "pin", quiet: bool = True, threads: int | None = None):
        self.lib = ctypes.CDLL(lib_path(variant))
        L = self.lib
        L.ref_new.restype = ctypes.c_void_p
        L.ref_new.argtypes = [ctypes.c_char_p]
        for n in ["ref_init_state", "ref_rk4", "ref_pressure", "ref_satadj", "ref_store",
                  "ref_level_mean", "ref_delete", "ref_bc", "ref_post_rk4_filters",
                  "ref_turbulence_run"]:
            getattr(L, n).argtypes = [ctypes.c_void_p]
        for n in ["ref_get3", "ref_set3", "ref_get2", "ref_set2", "ref_getp", "ref_setp"]:
            getattr(L, n).argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)]
            getattr(L, n).restype = ctypes.c_int
        L.ref_project.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_densities.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_init_state_upto.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_moist.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_set_scalars.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.ref_rhs_cell.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_double)]
        L.ref_constants.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_damp_wiggles.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.ref_damp_wiggles.restype = ctypes.c_int
        self.threads = threads
        L.ref_quiet.argtypes = [ctypes.c_int]
        im, jm, km = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        L.ref_dims(ctypes.byref(im), ctypes.byref(jm), ctypes.byref(km))
        self.shape = (im.value, jm.value, km.value)
        L.ref_quiet(1 if quiet else 0)
        if threads:
            L.ref_set_threads(threads)
        self.h = L.ref_new(None)   # compiled-in defaults = cli/config_cond.xml

    def close(self):
        if self.h:
            self.lib.ref_delete(self.h)
            self.h = None

    def init_state(self, upto: int = 99):
        """RunTimeSlice's initial state, up to stage `upto` (99 = everything)."""
        self.lib.ref_init_state_upto(self.h, int(upto))

    def get(self, name):
        out = np.empty(self.shape)
        assert self.lib.ref_get3(self.h, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0, name
        return out

    def set(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == self.shape
        assert self.lib.ref_set3(self.h, name.encode(), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0, name

    def get2(self, name):
        out = np.empty(self.shape[1:])
        assert self.lib.ref_get2(self.h, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0, name
        return out

    def set2(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert self.lib.ref_set2(self.h, name.encode(), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0, name

    def getp(self, name):
        out = np.empty(self.shape[0])
        r = self.lib.ref_getp(self.h, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out if r == 0 else None

    def setp(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert self.lib.ref_setp(self.h, name.encode(), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0

    def constants(self):
        out = (ctypes.c_double * 8)()
        self.lib.ref_constants(self.h, out)
        keys = ["re_turb", "metric_r0", "shell_len", "M_bg", "R_bg", "R_mix", "dt_visc"]
        return dict(zip(keys, list(out)[:7]))

    def set_scalars(self, dt, diffusion_ramp, buoyancy_ramp, total_iter_count, iter_n):
        self.lib.ref_set_scalars(self.h, dt, diffusion_ramp, buoyancy_ramp, total_iter_count, iter_n)

    def dropin(self, what: int, arg: int = 0, wall: int = 0):
        """Run one hot-path call through the product's C++ drop-in on this model."""
        f = self.lib.dropin_run
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        f.restype = ctypes.c_int
        err = ctypes.create_string_buffer(512)
        r = f(self.h, what, arg, wall, err, 512)
        if r != 0:
            raise RuntimeError(err.value.decode())

    def resident(self, n: int, first_iter: int = 1, wall: int = 0):
        """n iterations of run_3D_loop's body through the product's device-resident drop-in
        on this model (athad_dropin::ResidentLoop); returns each iteration's residuum and
        skin temperature."""
        f = self.lib.dropin_resident
        D = ctypes.POINTER(ctypes.c_double)
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, D, D, ctypes.c_char_p, ctypes.c_int]
        f.restype = ctypes.c_int
        res, skin = np.zeros(n), np.zeros(n)
        err = ctypes.create_string_buffer(512)
        r = f(self.h, n, first_iter, wall, res.ctypes.data_as(D), skin.ctypes.data_as(D), err, 512)
        if r != 0:
            raise RuntimeError(err.value.decode())
        return res, skin

    def dropin_params(self, wall: int = 0):
        """The athad_params the C++ adapter builds from this model."""
        from athad_cond_b200._abi import Params
        p = Params()
        f = self.lib.dropin_params
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(Params)]
        f(self.h, wall, ctypes.byref(p))
        return p

    def loop_scalars(self) -> dict:
        """The model's scalars the resident loop reads."""
        out = np.zeros(6)
        f = self.lib.dropin_loop_scalars
        f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        f(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return {"dt": out[0], "buoyancy_ramp_iters": int(out[1]), "t_skin_relax": out[2],
                "checkpoint": int(out[3]), "total_iter_count": int(out[4]), "t_skin": out[5]}

    def post_rk4_filters(self):
        self.lib.ref_post_rk4_filters(self.h)

    def damp_wiggles(self, name):
        assert self.lib.ref_damp_wiggles(self.h, name.encode()) == 0, name

    def precipitation_sum(self):
        f = self.lib.ref_precipitation_sum
        f.argtypes = [ctypes.c_void_p]
        f(self.h)

    def mlr(self):
        f = self.lib.ref_mlr
        f.argtypes = [ctypes.c_void_p]
        f(self.h)

    def radiative_heating(self, omega_rad=0.05):
        f = self.lib.ref_radiative_heating
        f.argtypes = [ctypes.c_void_p, ctypes.c_double]
        f(self.h, omega_rad)

    def two_cat_ice(self):
        f = self.lib.ref_two_cat_ice
        f.argtypes = [ctypes.c_void_p]
        f(self.h)

    def ice_scheme(self, category):
        """ZeroCat/OneCat/TwoCat/ThreeCatIceScheme(*m).run() for `category` 0..3."""
        f = getattr(self.lib, ("ref_zero_cat_ice", "ref_one_cat_ice", "ref_two_cat_ice",
                               "ref_three_cat_ice")[category])
        f.argtypes = [ctypes.c_void_p]
        f(self.h)

    def skin(self, relax: float) -> float:
        """cAtmosphereModel::updateSkinTemperature with t_skin_relax = relax: the new t_skin
        (relax = 0 reads it unchanged)."""
        f = self.lib.ref_skin
        f.argtypes = [ctypes.c_void_p, ctypes.c_double]
        f.restype = ctypes.c_double
        return f(self.h, relax)

    def budgets(self, threads=1) -> dict:
        """ThermoAtm::co2Column and ::waterBudget as first calls: the references they set
        (one thread by default, so the OpenMP sums run in the serial order)."""
        im = self.shape[0]
        out = np.empty(3 + 2 * im)
        f = self.lib.ref_budgets
        f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        if threads:
            self.lib.ref_set_threads(threads)
        try:
            f(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        finally:
            if threads and self.threads:
                self.lib.ref_set_threads(self.threads)
        return {"q_co2_ref": out[0], "q_h2o_ref": out[1], "q_h2o_fixed_ref": out[2],
                "air_levels": out[3:3 + im].copy(), "h2o_levels": out[3 + im:].copy()}

    def evaporation(self):
        """ThermoAtm::waterVapourEvaporation."""
        f = self.lib.ref_evaporation
        f.argtypes = [ctypes.c_void_p]
        f(self.h)

    def latent_sensible(self):
        """ThermoAtm::latentSensibleHeat."""
        f = self.lib.ref_latent_sensible
        f.argtypes = [ctypes.c_void_p]
        f(self.h)

    def stand_atm(self):
        """ThermoAtm::standAtm_DewPoint_HumidRel."""
        f = self.lib.ref_stand_atm
        f.argtypes = [ctypes.c_void_p]
        f(self.h)

    def tropopause_layers(self):
        out = np.empty(self.shape[1])
        f = self.lib.ref_tropopause
        f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        f(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def find_residuum(self, threads=1) -> dict:
        """UtilsAtm::findResiduumAtm, read back from its printout (one thread by default, so
        the printed first non-finite cell and equal-value choices follow the serial order)."""
        out = (ctypes.c_double * 3)()
        idx = (ctypes.c_longlong * 5)()
        f = self.lib.ref_residuum
        f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong)]
        if threads:
            self.lib.ref_set_threads(threads)
        try:
            f(self.h, out, idx)
        finally:
            if threads and self.threads:
                self.lib.ref_set_threads(self.threads)
        return {"residuum": out[0], "residuum_prev": out[1], "avg_abs_8": out[2],
                "at": tuple(idx[0:3]), "n_cells": idx[3], "n_nonfinite": idx[4]}

    def budget_refs(self):
        """The model's m_q_co2_ref, m_q_h2o_ref, m_q_h2o_fixed_ref (needs the drop-in library)."""
        out = (ctypes.c_double * 3)()
        f = self.lib.dropin_budget_refs
        f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        f(self.h, out)
        return list(out)

    def residuum_old(self) -> float:
        """The model's residuum_old (needs the drop-in library)."""
        f = self.lib.dropin_residuum_old
        f.argtypes = [ctypes.c_void_p]
        f.restype = ctypes.c_double
        return f(self.h)

    def set_turb_model(self, name: str):
        f = self.lib.ref_set_turb_model
        f.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        f(self.h, name.encode())

    def turbulence_run(self, threads=None):
        """TurbulenceAtm::run; threads=1 for the serial sweep order."""
        if threads:
            self.lib.ref_set_threads(threads)
        try:
            self.lib.ref_turbulence_run(self.h)
        finally:
            if threads and self.threads:
                self.lib.ref_set_threads(self.threads)

    def bc(self):
        """BC_Atm::bcRadius, TurbulenceAtm::apply_wall_bc, bcTheta, bcPhi."""
        self.lib.ref_bc(self.h)

    def rhs_cell(self, i, j, k):
        out = (ctypes.c_double * 17)()
        self.lib.ref_rhs_cell(self.h, int(i), int(j), int(k), out)
        return np.array(list(out))
