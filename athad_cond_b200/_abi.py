"""ctypes description of the C ABI in include/athad_gpu.h.

The shared library is the product; this module only describes its types and loads it.
Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from enum import IntEnum

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libathad_gpu.so")


class Status(IntEnum):
    OK = 0
    ERR_INVALID = 1
    ERR_CUDA = 2
    ERR_UNSUPPORTED = 3
    ERR_OOM = 4
    ERR_NONFINITE = 5
    ERR_TIMEOUT = 6
    ERR_NO_DEVICE = 7


class Turb(IntEnum):
    K_EPSILON = 1
    K_OMEGA = 2
    K_OMEGA_SST = 3


class Wall(IntEnum):
    MIRROR = 0
    REFERENCE = 1


class Precision(IntEnum):
    FP64 = 0
    MIXED = 1


FIELD_NAMES = [
    "t", "u", "v", "w", "c", "cloud", "ice", "gr", "co2", "tke", "dis",
    "tn", "un", "vn", "wn", "cn", "cloudn", "icen", "grn", "co2n", "tken", "disn",
    "p_dyn", "nue", "t_eq", "p_stat", "r_humid",
    "S_c", "S_r", "S_i", "S_s", "S_g", "S_v",
    "MC_t", "MC_q", "MC_v", "MC_w",
    "aux_u", "aux_v", "aux_w",
    "prod", "tke_source", "dis_source",
    "S_c_c", "P_rain", "P_snow", "P_graupel", "Precipitation",
    "r_dry",
    "s", "s_u", "s_d", "M_u", "M_d",
    "q_v_u", "q_c_u", "q_v_d",
    "u_u", "v_u", "w_u", "u_d", "v_d", "w_d",
    "E_u", "D_u", "E_d", "D_d",
    "c_u", "e_l", "e_d", "e_p", "g_p",
    "P_conv", "CloudBase", "LevelFreeSinking", "Deep_beg", "Deep_end",
    "P_rainn", "P_snown",
    "radiation", "epsilon",
    "TempStand", "TempDewPoint", "HumidityRel",
    "Q_Latent", "Q_Sensible",
    "CoriolisForce", "BuoyancyForce", "PressureGradientForce",
    "vbud_pgf", "vbud_cor", "vbud_advv", "vbud_advh", "vbud_diff", "vbud_other",
    "wbud_pgf", "wbud_cor", "wbud_advv", "wbud_advh", "wbud_diff", "wbud_other",
]
FIELD = {n: i for i, n in enumerate(FIELD_NAMES)}
NFIELDS = len(FIELD_NAMES)
PROGNOSTIC = FIELD_NAMES[0:11]
N_LEVEL = FIELD_NAMES[11:22]

FIELD2D_NAMES = ["t_top_init", "p_stat_landscape", "Evaporation", "Q_sensible_2D", "vel_star",
                 "epsilon_2D", "albedo", "Evaporation_Dalton", "Evaporation_Meyer",
                 "Evaporation_Rohwer", "c_fix", "co2_total"]
FIELD2D = {n: i for i, n in enumerate(FIELD2D_NAMES)}
PROFILE_NAMES = ["t_ref_level", "rho_base", "dlnrho_dr"]
PROFILE = {n: i for i, n in enumerate(PROFILE_NAMES)}


class Grid(ctypes.Structure):
    _fields_ = [("im", ctypes.c_int32), ("jm", ctypes.c_int32), ("km", ctypes.c_int32)]


_PARAM_INTS = [
    "turb_model", "wall_mode", "poisson_metric_fix", "anelastic", "tracer_diff_flux",
    "coriolis_nontrad", "metric_curvature", "metric_divergence",
    "convection_perturbation", "convection_mode", "iter_prec", "precision", "category_ice_scheme",
]
_PARAM_DOUBLES = [
    "metric_r0", "re_turb",
    "r_air", "g", "u_0", "cp_l", "t_0", "c_0", "L_atm", "zeta", "omega", "lamda", "lv", "ls",
    "pr_turb", "sc_WaterVapour", "sc_CO2",
    "r_Earth", "p_0", "t_00", "t_max_phys", "cloud_cap", "t_skin", "c_h2o_dry_top", "co2_0", "s_0",
    "R_Air", "R_WaterVapour",
    "M_bg", "R_bg", "R_mix",
    "abl_height", "t_000",
    "sigma", "kappa_H2O", "kappa_CO2", "kappa_bg", "geothermal_flux", "albedo_surface",
    "albedo_cloud", "rad_equator_short", "rad_pole_short", "coeff_Dalton", "r_0_water",
]


class Params(ctypes.Structure):
    _fields_ = ([("struct_size", ctypes.c_uint32)]
                + [(n, ctypes.c_int32) for n in _PARAM_INTS]
                + [(n, ctypes.c_double) for n in _PARAM_DOUBLES])

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class InitConfig(ctypes.Structure):
    """athad_init_config: the configuration members the reference's initial state reads
    beyond athad_params (cli/config_cond.xml values by default)."""
    _fields_ = [("struct_size", ctypes.c_uint32), ("n_cells_hemisphere", ctypes.c_int32),
                ("cell_amp_mode", ctypes.c_int32), ("pad0", ctypes.c_int32)] + [
        (n, ctypes.c_double) for n in ("t_surf_equator", "t_surf_pole", "tropopause_equator",
                                       "tropopause_pole", "cell_lat_scale", "co2_scale", "q_CO2",
                                       "q_bg", "vel_star_init")]


def composition(x):
    """AtmMixture::resolve (MixtureAtm.h:82-109) of the eight mole fractions x_H2O, x_CO2,
    x_N2, x_CH4, x_NH3, x_H2, x_CO, x_SO2: M_mean, R_mix, q_H2O, q_CO2, q_bg, M_bg, R_bg."""
    R_STAR, M_H2O, M_CO2 = 8.314462618, 0.018015, 0.044010
    m_H2O, m_CO2 = x[0] * M_H2O, x[1] * M_CO2
    m_bg = x[2] * 0.028014 + x[3] * 0.016043 + x[4] * 0.017031 + x[5] * 0.002016 + x[6] * 0.028010 + x[7] * 0.064066
    M_mean = m_H2O + m_CO2 + m_bg
    x_bg = x[2] + x[3] + x[4] + x[5] + x[6] + x[7]
    M_bg = (m_bg / x_bg) if x_bg > 0.0 else 0.028014
    return {"M_mean": M_mean, "R_mix": R_STAR / M_mean, "q_H2O": m_H2O / M_mean,
            "q_CO2": m_CO2 / M_mean, "q_bg": m_bg / M_mean, "M_bg": M_bg, "R_bg": R_STAR / M_bg}


CONFIG_X = (0.5578, 0.4109, 0.0313, 0.0, 0.0, 0.0, 0.0, 0.0)   # cli/config_cond.xml:77-84


def config_init() -> InitConfig:
    """cli/config_cond.xml's initial-state members (same as athad_default_init_config)."""
    c = InitConfig()
    c.struct_size = ctypes.sizeof(InitConfig)
    c.n_cells_hemisphere, c.cell_amp_mode = 5, 0
    c.t_surf_equator, c.t_surf_pole = 513.15, 503.15
    c.tropopause_equator, c.tropopause_pole = 207000.0, 195000.0
    c.cell_lat_scale, c.co2_scale, c.vel_star_init = 0.11, 1.0, 0.4
    comp = composition(CONFIG_X)
    c.q_CO2, c.q_bg = comp["q_CO2"], comp["q_bg"]
    return c


class StepScalars(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("diffusion_ramp", ctypes.c_double),
                ("buoyancy_ramp", ctypes.c_double), ("write_diagnostics", ctypes.c_int32),
                ("store_n_level", ctypes.c_int32)]


class BatchStepParams(ctypes.Structure):
    """athad_batch_step"""
    _fields_ = [("dt", ctypes.c_double), ("diffusion_ramp", ctypes.c_double),
                ("buoyancy_ramp_iters", ctypes.c_int32), ("pad0", ctypes.c_int32)]


class SolveReport(ctypes.Structure):
    """athad_solve_report"""
    _fields_ = [("iterations", ctypes.c_int32), ("converged", ctypes.c_int32),
                ("rel_residual", ctypes.c_double), ("history", ctypes.c_double * 64),
                ("precond_levels", ctypes.c_int32), ("pad0", ctypes.c_int32), ("seconds", ctypes.c_double)]


class CeilingReport(ctypes.Structure):
    """athad_ceiling_report"""
    _fields_ = [("n_ceiling", ctypes.c_int64), ("pad0", ctypes.c_int64),
                ("q_clipped", ctypes.c_double), ("w_air", ctypes.c_double)]


class MinMaxReport(ctypes.Structure):
    """athad_min_max_report"""
    _fields_ = [("max", ctypes.c_double), ("min", ctypes.c_double)] + [
        (n, ctypes.c_int32) for n in ("imax", "jmax", "kmax", "imin", "jmin", "kmin")]


class ResiduumReport(ctypes.Structure):
    """athad_residuum_report"""
    _fields_ = [("residuum", ctypes.c_double), ("residuum_prev", ctypes.c_double),
                ("avg_abs", ctypes.c_double), ("avg_rel", ctypes.c_double),
                ("n_cells", ctypes.c_int64), ("n_nonfinite", ctypes.c_int64)] + [
        (n, ctypes.c_int32) for n in ("i_error", "j_error", "k_error", "i_nan", "j_nan", "k_nan")]


class BudgetReport(ctypes.Structure):
    """athad_budget_report"""
    _fields_ = [(n, ctypes.c_double) for n in (
        "q_mean", "q_ref", "drift_pct", "q_fixed", "q_fixed_ref", "fixed_drift_pct",
        "air_now", "air_ref", "air_drift_pct")]


class Report(ctypes.Structure):
    _fields_ = [("poisson_src_cells", ctypes.c_int64), ("poisson_src_clamped", ctypes.c_int64),
                ("satadj_ceiling_hits", ctypes.c_int64), ("nonfinite_inputs", ctypes.c_int64),
                ("last_kernel_ms", ctypes.c_double)]


# name -> (restype, argtypes); every symbol include/athad_gpu.h declares
_P = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "athad_default_params": (None, [ctypes.POINTER(Params)]),
    "athad_abi_version": (ctypes.c_int32, []),
    "athad_params_size": (ctypes.c_size_t, []),
    "athad_create": (ctypes.c_int, [ctypes.POINTER(Grid), ctypes.POINTER(Params), ctypes.POINTER(_P)]),
    "athad_destroy": (ctypes.c_int, [_P]),
    "athad_last_error": (ctypes.c_char_p, [_P]),
    "athad_set_stream": (ctypes.c_int, [_P, _P]),
    "athad_synchronize": (ctypes.c_int, [_P]),
    "athad_footprint_bytes": (ctypes.c_size_t, [ctypes.POINTER(Grid)]),
    "athad_footprint_bytes_params": (ctypes.c_size_t, [ctypes.POINTER(Grid), ctypes.POINTER(Params)]),
    "athad_upload": (ctypes.c_int, [_P, ctypes.c_int, _D, ctypes.c_size_t]),
    "athad_upload_device": (ctypes.c_int, [_P, ctypes.c_int, _P, ctypes.c_size_t]),
    "athad_download": (ctypes.c_int, [_P, ctypes.c_int, _D, ctypes.c_size_t]),
    "athad_upload_2d": (ctypes.c_int, [_P, ctypes.c_int, _D, ctypes.c_size_t]),
    "athad_download_2d": (ctypes.c_int, [_P, ctypes.c_int, _D, ctypes.c_size_t]),
    "athad_upload_profile": (ctypes.c_int, [_P, ctypes.c_int, _D, ctypes.c_size_t]),
    "athad_download_profile": (ctypes.c_int, [_P, ctypes.c_int, _D, ctypes.c_size_t]),
    "athad_download_profile_async": (ctypes.c_int, [_P, ctypes.c_int, _D, ctypes.c_size_t]),
    "athad_field_device_ptr": (ctypes.c_int, [_P, ctypes.c_int, ctypes.POINTER(_D), ctypes.POINTER(ctypes.c_size_t)]),
    "athad_fill": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_double]),
    "athad_default_init_config": (None, [ctypes.POINTER(InitConfig)]),
    "athad_initial_state": (ctypes.c_int, [_P, ctypes.POINTER(InitConfig)]),
    "athad_store_n_level": (ctypes.c_int, [_P]),
    "athad_level_mean": (ctypes.c_int, [_P]),
    "athad_rk4_step": (ctypes.c_int, [_P, ctypes.POINTER(StepScalars)]),
    "athad_pressure_sweep": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32]),
    "athad_boundary_conditions": (ctypes.c_int, [_P]),
    "athad_post_rk4_filters": (ctypes.c_int, [_P]),
    "athad_damp_wiggles": (ctypes.c_int, [_P, ctypes.c_int]),
    "athad_turbulence_run": (ctypes.c_int, [_P]),
    "athad_two_cat_ice_scheme": (ctypes.c_int, [_P]),
    "athad_zero_cat_ice_scheme": (ctypes.c_int, [_P]),
    "athad_one_cat_ice_scheme": (ctypes.c_int, [_P]),
    "athad_three_cat_ice_scheme": (ctypes.c_int, [_P]),
    "athad_ice_scheme": (ctypes.c_int, [_P]),
    "athad_multilayer_radiation": (ctypes.c_int, [_P]),
    "athad_radiative_heating": (ctypes.c_int, [_P, ctypes.c_double]),
    "athad_moist_caps": (ctypes.c_int, [_P]),
    "athad_vapour_ceiling": (ctypes.c_int, [_P, _P]),
    "athad_min_max": (ctypes.c_int, [_P, ctypes.c_int, _P]),
    "athad_find_residuum": (ctypes.c_int, [_P, ctypes.POINTER(ResiduumReport)]),
    "athad_set_tropopause_layers": (ctypes.c_int, [_P, _D, ctypes.c_int32]),
    "athad_stand_atm_dew_point": (ctypes.c_int, [_P]),
    "athad_water_vapour_evaporation": (ctypes.c_int, [_P]),
    "athad_latent_sensible_heat": (ctypes.c_int, [_P]),
    "athad_update_skin_temperature": (ctypes.c_int, [_P, ctypes.c_double, _D]),
    "athad_forces": (ctypes.c_int, [_P]),
    "athad_co2_column": (ctypes.c_int, [_P, ctypes.POINTER(BudgetReport)]),
    "athad_water_budget": (ctypes.c_int, [_P, ctypes.POINTER(BudgetReport), _D]),
    "athad_checkpoint_begin": (ctypes.c_int, [_P, _P, ctypes.c_int32, _P]),
    "athad_checkpoint_wait": (ctypes.c_int, [_P]),
    "athad_pressure_solve": (ctypes.c_int, [_P, ctypes.c_double, ctypes.c_int32, ctypes.POINTER(SolveReport)]),
    "athad_project_initial_velocity": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32]),
    "athad_saturation_adjust": (ctypes.c_int, [_P]),
    "athad_densities": (ctypes.c_int, [_P, ctypes.c_int32]),
    "athad_moist_convection": (ctypes.c_int, [_P, ctypes.c_int32]),
    "athad_get_report": (ctypes.c_int, [_P, ctypes.POINTER(Report)]),
    "athad_batch_create": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int32, ctypes.POINTER(BatchStepParams),
                                          ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(_P)]),
    "athad_batch_destroy": (ctypes.c_int, [_P]),
    "athad_batch_last_error": (ctypes.c_char_p, [_P]),
    "athad_batch_set_stream": (ctypes.c_int, [_P, _P]),
    "athad_batch_synchronize": (ctypes.c_int, [_P]),
    "athad_batch_member_iter": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "athad_batch_set_active": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32]),
    "athad_batch_iteration": (ctypes.c_int, [_P]),
    "athad_batch_iteration_graph": (ctypes.c_int, [_P]),
    "athad_batch_shape_count": (ctypes.c_int32, []),
    "athad_batch_set_shape": (ctypes.c_int, [_P, ctypes.c_int32]),
    "athad_batch_autotune": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                            ctypes.POINTER(ctypes.c_float)]),
    "athad_thermo_arity": (ctypes.c_int32, [ctypes.c_int32]),
    "athad_thermo_eval": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, _D, _D]),
    "athad_density_profile_noalloc": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                     ctypes.c_size_t, _P, _P, _P]),
}
NOALLOC_MAX_ROWS = 131072
NOALLOC_MAX_IM = 1024

_lib = None


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Load libathad_gpu.so and bind every declared symbol.  Raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"athad_cond_b200: CUDA library {p} not found; run __graft_entry__.build() "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.athad_params_size() != ctypes.sizeof(Params):
        raise RuntimeError("athad_cond_b200: athad_params layout mismatch between library and bindings")
    if path is None:
        _lib = lib
    return lib


def default_params() -> Params:
    p = Params()
    load_library().athad_default_params(ctypes.byref(p))
    return p


def config_params() -> Params:
    """cli/config_cond.xml values without loading the library (same as athad_default_params)."""
    p = Params()
    p.struct_size = ctypes.sizeof(Params)
    p.turb_model = Turb.K_OMEGA_SST
    p.wall_mode = Wall.MIRROR
    p.poisson_metric_fix = 1
    p.convection_perturbation = 1
    p.convection_mode = 1
    p.iter_prec = 3
    p.category_ice_scheme = 2
    p.metric_r0 = -1.0
    p.re_turb = 0.4 * 0.1 / 1.5e-5
    vals = dict(r_air=40.8, g=9.8066, u_0=8.0, cp_l=1349.0, t_0=273.15, c_0=0.3464, L_atm=6287.5,
                zeta=3.0, omega=0.000317, lamda=0.0262, lv=2520000.0, ls=2830000.0, pr_turb=0.9,
                sc_WaterVapour=0.61, sc_CO2=0.96, r_Earth=6370.001, p_0=60000.0, t_00=236.15,
                t_max_phys=2000.0, cloud_cap=0.05, t_skin=254.0, c_h2o_dry_top=0.00423,
                co2_0=0.6233, s_0=274515.75, R_Air=296.8, R_WaterVapour=461.5, abl_height=10000.0,
                t_000=253.15, sigma=5.67028e-08, kappa_H2O=0.01, kappa_CO2=0.001, kappa_bg=1e-06,
                geothermal_flux=150.0, albedo_surface=0.08, albedo_cloud=0.5,
                rad_equator_short=298.0, rad_pole_short=0.0, coeff_Dalton=0.7, r_0_water=997.0)
    for k, v in vals.items():
        setattr(p, k, v)
    comp = composition(CONFIG_X)
    p.R_mix, p.M_bg, p.R_bg = comp["R_mix"], comp["M_bg"], comp["R_bg"]
    return p
