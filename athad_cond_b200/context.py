"""Python view of one device-resident model state (an athad_ctx).

Mirrors the reference's call sites in cAtmosphereModel::run_3D_loop
(atmosphere/cAtmosphereModel.cpp:1103-1724): each method is one of the in-place physics
calls, named after the reference function it replaces.  Errors surface as AthadError with
the library's own message, as the reference's `throw` would.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import FIELD, FIELD2D, PROFILE, Status


def default_init_config() -> _abi.InitConfig:
    """athad_default_init_config: cli/config_cond.xml's initial-state members."""
    c = _abi.InitConfig()
    _abi.load_library().athad_default_init_config(ctypes.byref(c))
    return c


class AthadError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = Status(status) if status in Status._value2member_map_ else status
        super().__init__(f"{self.status!r}: {message}")


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class GpuAtmosphere:
    """Device-resident state of one grid, driven through libathad_gpu.so."""

    def __init__(self, im: int, jm: int, km: int, params: _abi.Params | None = None):
        self.lib = _abi.load_library()
        self.shape = (im, jm, km)
        self.params = params if params is not None else _abi.default_params()
        self.params.struct_size = ctypes.sizeof(_abi.Params)
        self._grid = _abi.Grid(im, jm, km)
        h = ctypes.c_void_p()
        st = self.lib.athad_create(ctypes.byref(self._grid), ctypes.byref(self.params), ctypes.byref(h))
        if st != 0:
            raise AthadError(st, "athad_create failed")
        self._h = h

    # ---- lifetime ----
    def close(self):
        if getattr(self, "_h", None):
            self.lib.athad_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int):
        if st != 0:
            raise AthadError(st, self.lib.athad_last_error(self._h).decode())

    @staticmethod
    def footprint_bytes(im: int, jm: int, km: int) -> int:
        g = _abi.Grid(im, jm, km)
        return int(_abi.load_library().athad_footprint_bytes(ctypes.byref(g)))

    def set_stream(self, cuda_stream_handle: int | None):
        self._check(self.lib.athad_set_stream(self._h, ctypes.c_void_p(cuda_stream_handle or 0)))

    def synchronize(self):
        self._check(self.lib.athad_synchronize(self._h))

    # ---- transfer ----
    def upload(self, name: str, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != self.shape:
            raise ValueError(f"{name}: shape {a.shape} != {self.shape}")
        self._check(self.lib.athad_upload(self._h, FIELD[name], _dptr(a), a.size))
        # keep the buffer alive until the (possibly asynchronous) copy has been issued
        self.synchronize()

    def upload_tensor(self, name: str, t):
        """A packed (im, jm, km) float64 CUDA tensor on this device (a state built on the
        device), copied on the context's stream."""
        if tuple(t.shape) != self.shape or not t.is_contiguous() or not t.is_cuda:
            raise ValueError(f"{name}: need a contiguous CUDA tensor of shape {self.shape}")
        self._check(self.lib.athad_upload_device(self._h, FIELD[name], ctypes.c_void_p(t.data_ptr()),
                                                 t.numel()))

    def download(self, name: str) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        self._check(self.lib.athad_download(self._h, FIELD[name], _dptr(out), out.size))
        return out

    def upload_2d(self, name: str, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self._check(self.lib.athad_upload_2d(self._h, FIELD2D[name], _dptr(a), a.size))
        self.synchronize()

    def download_2d(self, name: str) -> np.ndarray:
        out = np.empty(self.shape[1:], dtype=np.float64)
        self._check(self.lib.athad_download_2d(self._h, FIELD2D[name], _dptr(out), out.size))
        return out

    def upload_profile(self, name: str, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self._check(self.lib.athad_upload_profile(self._h, PROFILE[name], _dptr(a), a.size))
        self.synchronize()

    def download_profile(self, name: str) -> np.ndarray:
        out = np.empty(self.shape[0], dtype=np.float64)
        self._check(self.lib.athad_download_profile(self._h, PROFILE[name], _dptr(out), out.size))
        return out

    # ---- the initial state ----
    def initial_state(self, config: _abi.InitConfig | None = None):
        """cAtmosphereModel::RunTimeSlice's deterministic initial state (cAtmosphereModel.cpp:
        468-668), built on the device for this grid: every field, 2-D field and profile is
        overwritten.  config: the initial-state members (default cli/config_cond.xml)."""
        cfg = config if config is not None else default_init_config()
        cfg.struct_size = ctypes.sizeof(_abi.InitConfig)
        self._check(self.lib.athad_initial_state(self._h, ctypes.byref(cfg)))

    def upload_state(self, state: dict):
        for name, a in state.items():
            if name in FIELD:
                self.upload(name, a)
            elif name in FIELD2D:
                self.upload_2d(name, a)
            elif name in PROFILE:
                self.upload_profile(name, a)

    def device_ptr(self, name: str):
        p = ctypes.POINTER(ctypes.c_double)()
        pitch = ctypes.c_size_t()
        self._check(self.lib.athad_field_device_ptr(self._h, FIELD[name], ctypes.byref(p), ctypes.byref(pitch)))
        return ctypes.cast(p, ctypes.c_void_p).value, int(pitch.value)

    def fill(self, name: str, value: float):
        self._check(self.lib.athad_fill(self._h, FIELD[name], float(value)))

    # ---- the hot path (reference call sites of cAtmosphereModel::run_3D_loop) ----
    def storeIntermediateData3D(self):
        """UtilsAtm::storeIntermediateData3D (UtilsAtm.h:25-49)."""
        self._check(self.lib.athad_store_n_level(self._h))

    def computeLevelMeanTemperature(self):
        """RungeKutta_Atm_Turb.cpp:24-41."""
        self._check(self.lib.athad_level_mean(self._h))

    def solveRungeKutta_Atmosphere_Turb(self, dt: float, diffusion_ramp: float = 1.0,
                                        buoyancy_ramp: float = 1.0, write_diagnostics: int = 0,
                                        store_n_level: bool = False):
        """RungeKutta_Atm_Turb.cpp:44-273 (call site cAtmosphereModel.cpp:1509); with
        store_n_level the following storeIntermediateData3D is fused into the last stage.
        write_diagnostics: 1 (or True) the right-hand side's diagnostic outputs (turbulence
        production and sources, acting forces, Q_Latent, Q_Sensible), 2 the momentum budget
        terms, 3 both."""
        s = _abi.StepScalars(dt, diffusion_ramp, buoyancy_ramp, int(write_diagnostics),
                             1 if store_n_level else 0)
        self._check(self.lib.athad_rk4_step(self._h, ctypes.byref(s)))

    def PressureSolverAtm_run(self, total_iter_count: int, n_sweeps: int = 1):
        """PressureSolverAtm::run (PressureSolverAtm.h:27-669; call site cAtmosphereModel.cpp:1158)."""
        self._check(self.lib.athad_pressure_sweep(self._h, n_sweeps, total_iter_count))

    def boundary_conditions(self):
        """BC_Atm::bcRadius, TurbulenceAtm::apply_wall_bc, bcTheta, bcPhi, bcScalarSurfSur,
        bcSolidGround (call site cAtmosphereModel.cpp:1439-1446)."""
        self._check(self.lib.athad_boundary_conditions(self._h))

    def post_rk4_filters(self):
        """Polar zonal and radial Shapiro filters of u, v, w (cAtmosphereModel.cpp:1507-1520)."""
        self._check(self.lib.athad_post_rk4_filters(self._h))

    def damp_wiggles(self, name: str):
        """AtomUtils::damp_wiggles(field, i, j, k) (lib/Utils.cpp:429-531)."""
        self._check(self.lib.athad_damp_wiggles(self._h, FIELD[name]))

    def moist_caps(self):
        """precipitationSum and the source / condensate caps (cAtmosphereModel.cpp:1265-1334)."""
        self._check(self.lib.athad_moist_caps(self._h))

    def vapour_ceiling(self) -> dict:
        """c in [0, 1 - co2] (cAtmosphereModel.cpp:1369-1391); what it removed."""
        r = _abi.CeilingReport()
        self._check(self.lib.athad_vapour_ceiling(self._h, ctypes.byref(r)))
        return {"n_ceiling": r.n_ceiling, "q_clipped": r.q_clipped, "w_air": r.w_air}

    def min_max(self, name: str) -> dict:
        """searchMinMax_3D (MinMax_Atm.cpp:51-109) of one field."""
        r = _abi.MinMaxReport()
        self._check(self.lib.athad_min_max(self._h, FIELD[name], ctypes.byref(r)))
        return {"max": r.max, "min": r.min, "at_max": (r.imax, r.jmax, r.kmax),
                "at_min": (r.imin, r.jmin, r.kmin)}

    def find_residuum(self) -> dict:
        """UtilsAtm::findResiduumAtm (UtilsAtm.h:70-220): the largest rms velocity-derivative
        residual of the band i = 10..30, its cell, the grid average and the non-finite cells."""
        r = _abi.ResiduumReport()
        self._check(self.lib.athad_find_residuum(self._h, ctypes.byref(r)))
        return {"residuum": r.residuum, "residuum_prev": r.residuum_prev, "avg_abs": r.avg_abs,
                "avg_rel": r.avg_rel, "n_cells": r.n_cells, "n_nonfinite": r.n_nonfinite,
                "at": (r.i_error, r.j_error, r.k_error), "first_nonfinite": (r.i_nan, r.j_nan, r.k_nan)}

    def set_tropopause_layers(self, layers):
        """cAtmosphereModel::tropopause_layers (jm level indices) for stand_atm_dew_point."""
        a = np.ascontiguousarray(layers, dtype=np.float64)
        self._check(self.lib.athad_set_tropopause_layers(
            self._h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size))

    def stand_atm_dew_point(self):
        """ThermoAtm::standAtm_DewPoint_HumidRel (ThermoAtm.h:400-516): TempStand,
        TempDewPoint, HumidityRel."""
        self._check(self.lib.athad_stand_atm_dew_point(self._h))

    def update_skin_temperature(self, t_skin_relax: float = 0.25) -> float:
        """cAtmosphereModel::updateSkinTemperature (cAtmosphereModel.cpp:291-327): the new
        t_skin, which the context's densities use from now on."""
        out = np.zeros(1)
        self._check(self.lib.athad_update_skin_temperature(self._h, float(t_skin_relax), _dptr(out)))
        return float(out[0])

    def co2_column(self) -> dict:
        """ThermoAtm::co2Column (ThermoAtm.h:1096-1137): co2_total and the CO2 budget."""
        r = _abi.BudgetReport()
        self._check(self.lib.athad_co2_column(self._h, ctypes.byref(r)))
        return {n: getattr(r, n) for n in ("q_mean", "q_ref", "drift_pct")}

    def water_budget(self) -> dict:
        """ThermoAtm::waterBudget (ThermoAtm.h:934-1094): the water budget and the per-level
        drift from the first call."""
        r = _abi.BudgetReport()
        lev = np.zeros(self.shape[0])
        self._check(self.lib.athad_water_budget(self._h, ctypes.byref(r), _dptr(lev)))
        out = {n: getattr(r, n) for n, _ in r._fields_}
        out["level_drift"] = lev
        return out

    def water_vapour_evaporation(self):
        """ThermoAtm::waterVapourEvaporation (ThermoAtm.h:115-398): surface water vapour
        relaxed toward the sea's saturation, Evaporation and the three evaporation laws."""
        self._check(self.lib.athad_water_vapour_evaporation(self._h))

    def latent_sensible_heat(self):
        """ThermoAtm::latentSensibleHeat (ThermoAtm.h:36-112): Q_Latent, Q_Sensible."""
        self._check(self.lib.athad_latent_sensible_heat(self._h))

    def checkpoint_begin(self, names):
        """Snapshot the named fields and copy them to page-locked host arrays on a side
        stream (athad_checkpoint_begin); the arrays are valid after checkpoint_wait()."""
        import torch
        bufs = {n: torch.empty(self.shape, dtype=torch.float64, pin_memory=True) for n in names}
        ids = (ctypes.c_int32 * len(names))(*[FIELD[n] for n in names])
        ptrs = (ctypes.c_void_p * len(names))(*[bufs[n].data_ptr() for n in names])
        self._check(self.lib.athad_checkpoint_begin(self._h, ids, len(names), ptrs))
        self._ckpt = (ids, ptrs, bufs)       # kept alive until the copies are done
        return {n: b.numpy() for n, b in bufs.items()}

    def checkpoint_wait(self):
        self._check(self.lib.athad_checkpoint_wait(self._h))

    def multilayer_radiation(self):
        """MultiLayerRadiation::run (MultiLayerRadiation.h:56-388): t := radiative equilibrium."""
        self._check(self.lib.athad_multilayer_radiation(self._h))

    def radiative_heating(self, omega_rad: float = 0.05):
        """Radiation mode 2's apply_radiative_heating (cAtmosphereModel.cpp:864-879)."""
        self._check(self.lib.athad_radiative_heating(self._h, float(omega_rad)))

    def forces(self):
        """ThermoAtm::forces' Coriolis and buoyancy arrays (ThermoAtm.h:518-614; call sites
        cAtmosphereModel.cpp:635, 1419)."""
        self._check(self.lib.athad_forces(self._h))

    def two_cat_ice_scheme(self):
        """TwoCatIceScheme::run (TwoCatIceScheme.h:89-109; call site cAtmosphereModel.cpp:1238)."""
        self._check(self.lib.athad_two_cat_ice_scheme(self._h))

    def zero_cat_ice_scheme(self):
        """ZeroCatIceScheme::run (ZeroCatIceScheme.h:37-56; CategoryIceScheme 0)."""
        self._check(self.lib.athad_zero_cat_ice_scheme(self._h))

    def one_cat_ice_scheme(self):
        """OneCatIceScheme::run (OneCatIceScheme.h:50-68; CategoryIceScheme 1)."""
        self._check(self.lib.athad_one_cat_ice_scheme(self._h))

    def three_cat_ice_scheme(self):
        """ThreeCatIceScheme::run (ThreeCatIceScheme.h:70-89; CategoryIceScheme 3)."""
        self._check(self.lib.athad_three_cat_ice_scheme(self._h))

    def ice_scheme(self):
        """The CategoryIceScheme switch (cAtmosphereModel.cpp:581-596, 1230-1245) on
        params.category_ice_scheme: -1 nothing, 0..3 the schemes above."""
        self._check(self.lib.athad_ice_scheme(self._h))

    def turbulence_run(self):
        """TurbulenceAtm::run (TurbulenceAtm.h:62-79; call site cAtmosphereModel.cpp:1426)."""
        self._check(self.lib.athad_turbulence_run(self._h))

    def pressure_solve(self, rel_tol: float = 1e-10, max_iter: int = 200) -> dict:
        """The sweep's pressure equation solved to a relative residual (athad_pressure_solve)."""
        r = _abi.SolveReport()
        self._check(self.lib.athad_pressure_solve(self._h, float(rel_tol), int(max_iter), ctypes.byref(r)))
        return {"iterations": r.iterations, "converged": bool(r.converged), "rel_residual": r.rel_residual,
                "history": list(r.history)[:max(0, min(r.iterations, 64))], "levels": r.precond_levels,
                "seconds": r.seconds}

    def project_initial_velocity(self, n_sweeps: int = 200, total_iter_count: int = 0):
        """PressureSolverAtm::project_initial_velocity (PressureSolverAtm.h:686-767)."""
        self._check(self.lib.athad_project_initial_velocity(self._h, n_sweeps, total_iter_count))

    def SaturationAdjustment_run(self):
        """SaturationAdjustment::run (SaturationAdjustment.h:25-45)."""
        self._check(self.lib.athad_saturation_adjust(self._h))

    def densities(self, set_water_profile: bool = False):
        """ThermoAtm::densities (ThermoAtm.h:1436-1666)."""
        self._check(self.lib.athad_densities(self._h, 1 if set_water_profile else 0))

    def MoistConvection_run(self, iter_n: int):
        """MoistConvection::run (MoistConvection.h:106-140)."""
        self._check(self.lib.athad_moist_convection(self._h, iter_n))

    def report(self) -> dict:
        r = _abi.Report()
        self._check(self.lib.athad_get_report(self._h, ctypes.byref(r)))
        return {n: getattr(r, n) for n, _ in r._fields_}


class GpuBatch:
    """An ensemble of mixed-precision GpuAtmosphere members advanced together
    (athad_batch_* of include/athad_gpu.h): per iteration, each member's column physics at
    its own cadence and every RK4 stage of all members in one persistent launch."""

    def __init__(self, members: list, dt: float = 4e-5, diffusion_ramp: float = 1.0,
                 buoyancy_ramp_iters: int = 300, first_iter: list | None = None):
        self.lib = _abi.load_library()
        self.members = list(members)
        n = len(self.members)
        handles = (ctypes.c_void_p * n)(*[m._h.value for m in self.members])
        step = _abi.BatchStepParams(dt, diffusion_ramp, buoyancy_ramp_iters, 0)
        fi = (ctypes.c_int32 * n)(*(first_iter or [1] * n))
        h = ctypes.c_void_p()
        st = self.lib.athad_batch_create(ctypes.cast(handles, ctypes.POINTER(ctypes.c_void_p)), n,
                                         ctypes.byref(step), fi, ctypes.byref(h))
        if st != 0:
            raise AthadError(st, "athad_batch_create failed")
        self._h = h

    def _check(self, st: int):
        if st != 0:
            raise AthadError(st, self.lib.athad_batch_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self.lib.athad_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, cuda_stream_handle: int | None):
        self._check(self.lib.athad_batch_set_stream(self._h, ctypes.c_void_p(cuda_stream_handle or 0)))

    def synchronize(self):
        self._check(self.lib.athad_batch_synchronize(self._h))

    def iteration(self, graph: bool = False):
        fn = self.lib.athad_batch_iteration_graph if graph else self.lib.athad_batch_iteration
        self._check(fn(self._h))

    def member_iter(self, m: int) -> int:
        v = ctypes.c_int32()
        self._check(self.lib.athad_batch_member_iter(self._h, m, ctypes.byref(v)))
        return int(v.value)

    def set_active(self, m: int, active: bool):
        self._check(self.lib.athad_batch_set_active(self._h, m, 1 if active else 0))

    def set_shape(self, shape: int):
        self._check(self.lib.athad_batch_set_shape(self._h, shape))

    def autotune(self, reps: int = 3):
        n = int(self.lib.athad_batch_shape_count())
        ms = (ctypes.c_float * n)()
        best = ctypes.c_int32()
        self._check(self.lib.athad_batch_autotune(self._h, reps, ctypes.byref(best), ms))
        return int(best.value), [float(x) for x in ms]
