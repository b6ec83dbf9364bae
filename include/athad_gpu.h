/*
 * athad_gpu.h - C ABI of the B200 (sm_100a) implementation of the ATHAD_COND model
 * iteration hot path.
 *
 * The reference has no plugin or FFI interface for this path: the physics classes are
 * friends of cAtmosphereModel that mutate its public Array members in place
 * (atmosphere/cAtmosphereModel.h:52-67, 536-662).  Each entry point below replaces one
 * of those in-place calls; the reference call site it stands in for is cited beside it.
 *
 * Conventions
 *   - Host buffers are caller-owned, packed FP64, (i, j, k) order with k (longitude)
 *     fastest: exactly the element order of the reference's Array::x[i][j][k] rows
 *     (lib/Array.cpp:62-71).  n = im*jm*km for 3-D fields.
 *   - Device state is owned by the context and stays resident between calls; a caller
 *     only uploads what changed on the host and downloads what it needs to read.
 *   - Every call returns an athad_status; nothing throws across the ABI.  A failing
 *     call leaves a message readable with athad_last_error().
 *   - One host thread per context.  All work of a context is issued on one CUDA stream
 *     (its own, or the one given to athad_set_stream), so calls are ordered.
 *   - Terrain is flat (no land cells, i_topography == 0), which is the configuration
 *     the reference runs (cli/config_cond.xml, InitValues_Atm.cpp init_topography).
 */
#ifndef ATHAD_GPU_H
#define ATHAD_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ATHAD_ABI_VERSION 11

typedef enum athad_status {
    ATHAD_OK              = 0,
    ATHAD_ERR_INVALID     = 1,  /* bad argument (null pointer, size mismatch, bad id)  */
    ATHAD_ERR_CUDA        = 2,  /* a CUDA runtime call failed                          */
    ATHAD_ERR_UNSUPPORTED = 3,  /* a configuration this library does not implement     */
    ATHAD_ERR_OOM         = 4,  /* device allocation failed / budget exceeded          */
    ATHAD_ERR_NONFINITE   = 5,  /* a kernel's status word reported non-finite input    */
    ATHAD_ERR_TIMEOUT     = 6,  /* a bounded device-side wait gave up                  */
    ATHAD_ERR_NO_DEVICE   = 7   /* no CUDA device, or not an sm_100 device             */
} athad_status;

/* Grid: im radial levels, jm colatitude rows (pole to pole, both poles stored),
 * km longitudes (both seam meridians stored).  cAtmosphereModel.h:162 fixes these at
 * 61 x 181 x 361; here they are run-time values (dr = 1/(im-1), dtheta = pi/(jm-1),
 * dphi = 2 pi/(km-1), the generalisation of cAtmosphereModel.cpp:46-60). */
typedef struct athad_grid {
    int32_t im, jm, km;
} athad_grid;

/* Turbulence closures of RHS_Atm_Turb.cpp:563-721 (turb_model in the XML). */
typedef enum athad_turb_model {
    ATHAD_TURB_K_EPSILON   = 1,
    ATHAD_TURB_K_OMEGA     = 2,
    ATHAD_TURB_K_OMEGA_SST = 3
} athad_turb_model;

/* Wall distance of the k-omega-SST blending function (RHS_Atm_Turb.cpp:640-671).
 * With flat terrain the reference's scan reduces to d = min(i, j, k): it measures the
 * meridional distance from the NORTH pole only, which breaks north-south mirror
 * symmetry by construction.  MIRROR measures it from the nearer pole,
 * min(i, min(j, jm-1-j), k), and is the default; REFERENCE reproduces the reference. */
typedef enum athad_wall_mode {
    ATHAD_WALL_MIRROR    = 0,
    ATHAD_WALL_REFERENCE = 1
} athad_wall_mode;

/* Arithmetic of the RK4 step.  FP64 is the reference's arithmetic.  MIXED evaluates the
 * right-hand side and stores the stage states and the RK4 accumulator in FP32, keeps the
 * time level n and the final combination y_n + dt/6 (k1 + 2k2 + 2k3 + k4) in FP64 and
 * leaves the other entry points (Poisson, saturation adjustment, moist convection,
 * densities) in FP64.  A context's precision is fixed at creation. */
typedef enum athad_precision {
    ATHAD_PRECISION_FP64  = 0,
    ATHAD_PRECISION_MIXED = 1
} athad_precision;

/* Model constants and switches.  Every double is the cAtmosphereModel member of the
 * same name (atmosphere/AtmosphereParams.h.inc, values from cli/config_cond.xml) unless
 * noted.  athad_default_params() fills the values of cli/config_cond.xml. */
typedef struct athad_params {
    uint32_t struct_size;        /* sizeof(athad_params), checked by athad_create     */
    int32_t  turb_model;         /* athad_turb_model                                  */
    int32_t  wall_mode;          /* athad_wall_mode                                   */
    int32_t  poisson_metric_fix; /* ATM_POISSON_METRIC_FIX, default 1 (PressureSolverAtm.h:173) */
    int32_t  anelastic;          /* ATM_ANELASTIC, default 0 (PressureSolverAtm.h:92)  */
    int32_t  tracer_diff_flux;   /* ATM_TRACER_DIFF_FLUX, default 0 (RHS_Atm_Turb.cpp:906) */
    int32_t  coriolis_nontrad;   /* ATOM_CORIOLIS_NONTRAD, default 0 (lib/Utils.h:54)  */
    int32_t  metric_curvature;   /* ATOM_METRIC_CURVATURE, default 0 (lib/Utils.h:92)  */
    int32_t  metric_divergence;  /* ATOM_METRIC_DIVERGENCE, default 0 (lib/Utils.h:98) */
    int32_t  convection_perturbation; /* XML, 1 */
    int32_t  convection_mode;    /* XML, 1 */
    int32_t  iter_prec;          /* XML, 3 */
    int32_t  precision;          /* athad_precision of the RK4 step (no counterpart in
                                  * the reference, which is FP64 only); default FP64 */
    int32_t  category_ice_scheme;/* XML CategoryIceScheme, 2 (cli/config_cond.xml:18): the
                                  * scheme athad_ice_scheme runs, -1 (none) or 0..3 */
    /* metric radius in rad.z units; 0 = off.  The reference default (ATM_METRIC_RADIUS
     * unset) is r_Earth*1e3/metricShellLength() (cAtmosphereModel.cpp:382-399); the
     * value 0 reproduces ATM_METRIC_RADIUS=0. */
    double metric_r0;
    double re_turb;              /* TurbulenceAtm.h:35: 0.4 * 0.1 / 1.5e-5            */
    double r_air, g, u_0, cp_l, t_0, c_0, L_atm, zeta, omega, lamda, lv, ls;
    double pr_turb, sc_WaterVapour, sc_CO2;
    double r_Earth, p_0, t_00, t_max_phys, cloud_cap, t_skin, c_h2o_dry_top, co2_0, s_0;
    double R_Air, R_WaterVapour;
    /* composition resolved from the configured mole fractions, AtmMixture::resolve
     * (MixtureAtm.h:82-109), i.e. cAtmosphereModel::m_comp */
    double M_bg, R_bg, R_mix;
    double abl_height;           /* XML abl_height [m], 10000 (cli/config_cond.xml:76):
                                  * the eddy-viscosity ceiling of TurbulenceAtm::clamp_nue */
    double t_000;                /* XML t_000 [K], 253.15 (cli/config_cond.xml:102): the
                                  * snow-flux floor temperature of TwoCatIceScheme */
    /* MultiLayerRadiation (cli/config_cond.xml:29-37, 66-67; cAtmosphereDefaults.cpp.inc) */
    double sigma;                /* Stefan-Boltzmann constant, 5.67028e-8              */
    double kappa_H2O, kappa_CO2, kappa_bg;  /* grey LW mass absorption [m2/kg]          */
    double geothermal_flux;      /* [W/m2], 150                                          */
    double albedo_surface, albedo_cloud;
    double rad_equator_short, rad_pole_short;   /* TOA short-wave insolation [W/m2]     */
    double coeff_Dalton;         /* XML coeff_Dalton, 0.7 (cli/config_cond.xml:54): the
                                  * Dalton evaporation coefficient (AtomUtils::C_Dalton)   */
    double r_0_water;            /* XML r_0_water [kg/m3], 997 (cAtmosphereDefaults.cpp.inc:33):
                                  * the rain drop density of ThreeCatIceScheme            */
} athad_params;

/* 3-D fields, one per cAtmosphereModel Array member of the same name. */
typedef enum athad_field {
    /* prognostic state (current level) */
    ATHAD_T = 0, ATHAD_U, ATHAD_V, ATHAD_W, ATHAD_C, ATHAD_CLOUD, ATHAD_ICE, ATHAD_GR,
    ATHAD_CO2, ATHAD_TKE, ATHAD_DIS,
    /* time level n (storeIntermediateData3D, UtilsAtm.h:25-49) */
    ATHAD_TN, ATHAD_UN, ATHAD_VN, ATHAD_WN, ATHAD_CN, ATHAD_CLOUDN, ATHAD_ICEN, ATHAD_GRN,
    ATHAD_CO2N, ATHAD_TKEN, ATHAD_DISN,
    /* inputs of the right-hand side */
    ATHAD_P_DYN, ATHAD_NUE, ATHAD_T_EQ, ATHAD_P_STAT, ATHAD_R_HUMID,
    ATHAD_S_C, ATHAD_S_R, ATHAD_S_I, ATHAD_S_S, ATHAD_S_G, ATHAD_S_V,
    ATHAD_MC_T, ATHAD_MC_Q, ATHAD_MC_V, ATHAD_MC_W,
    /* provisional velocity (RHS_Atm_Turb.cpp:1077-1079), source of the Poisson solve */
    ATHAD_AUX_U, ATHAD_AUX_V, ATHAD_AUX_W,
    /* turbulence diagnostics written by the last RK4 stage (RHS_Atm_Turb.cpp:551, 628) */
    ATHAD_PROD, ATHAD_TKE_SOURCE, ATHAD_DIS_SOURCE,
    /* saturation adjustment / microphysics fields (SaturationAdjustment.h,
     * IceSchemeCommon.h:121-190) */
    ATHAD_S_C_C, ATHAD_P_RAIN, ATHAD_P_SNOW, ATHAD_P_GRAUPEL, ATHAD_PRECIPITATION,
    /* densities (ThermoAtm.h:1436-1666) */
    ATHAD_R_DRY,
    /* moist convection (MoistConvection.h) */
    ATHAD_MC_S, ATHAD_MC_S_U, ATHAD_MC_S_D, ATHAD_M_U, ATHAD_M_D,
    ATHAD_Q_V_U, ATHAD_Q_C_U, ATHAD_Q_V_D,
    ATHAD_U_U, ATHAD_V_U, ATHAD_W_U, ATHAD_U_D, ATHAD_V_D, ATHAD_W_D,
    ATHAD_E_U, ATHAD_D_U, ATHAD_E_D, ATHAD_D_D,
    ATHAD_C_U, ATHAD_E_L, ATHAD_E_DD, ATHAD_E_P, ATHAD_G_P,
    ATHAD_P_CONV, ATHAD_CLOUD_BASE, ATHAD_LEVEL_FREE_SINKING, ATHAD_DEEP_BEG, ATHAD_DEEP_END,
    /* precipitation fluxes of the time level n (storeIntermediateData3D, UtilsAtm.h:41-42),
     * the ice scheme's starting fluxes (TwoCatIceScheme.h:149-153) */
    ATHAD_P_RAINN, ATHAD_P_SNOWN,
    /* MultiLayerRadiation outputs (MultiLayerRadiation.h): upward long-wave flux per layer
     * [W/m2] and the layer emissivity */
    ATHAD_RADIATION, ATHAD_EPSILON,
    /* standAtm_DewPoint_HumidRel outputs (ThermoAtm.h:400-516): the standard-atmosphere
     * temperature [deg C], the dew point [deg C] and the relative humidity [%] */
    ATHAD_TEMP_STAND, ATHAD_TEMP_DEW_POINT, ATHAD_HUMIDITY_REL,
    /* latentSensibleHeat outputs (ThermoAtm.h:36-112), overwritten in the interior by the
     * right-hand side's own heat diagnostics on athad_rk4_step's diagnostic steps
     * (RHS_Atm_Turb.cpp:471-491) */
    ATHAD_Q_LATENT, ATHAD_Q_SENSIBLE,
    /* the right-hand side's acting forces (RHS_Atm_Turb.cpp:447-456), written on diagnostic
     * steps */
    ATHAD_CORIOLIS_FORCE, ATHAD_BUOYANCY_FORCE, ATHAD_PRESSURE_GRADIENT_FORCE,
    /* the terms of rhs_v and rhs_w (pressure gradient, Coriolis, vertical and horizontal
     * advection, diffusion, the rest), written on momentum-budget steps
     * (RHS_Atm_Turb.cpp:1031-1057, vbud_* and wbud_*) */
    ATHAD_VBUD_PGF, ATHAD_VBUD_COR, ATHAD_VBUD_ADVV, ATHAD_VBUD_ADVH, ATHAD_VBUD_DIFF, ATHAD_VBUD_OTHER,
    ATHAD_WBUD_PGF, ATHAD_WBUD_COR, ATHAD_WBUD_ADVV, ATHAD_WBUD_ADVH, ATHAD_WBUD_DIFF, ATHAD_WBUD_OTHER,
    ATHAD_NFIELDS
} athad_field;

/* 2-D (jm x km) fields. */
typedef enum athad_field2d {
    ATHAD_2D_T_TOP_INIT = 0,        /* cAtmosphereModel::t_top_init                  */
    ATHAD_2D_P_STAT_LANDSCAPE,      /* Array_2D p_stat_landscape                      */
    ATHAD_2D_EVAPORATION,           /* Array_2D Evaporation (MoistConvection input)   */
    ATHAD_2D_Q_SENSIBLE,            /* Array_2D Q_sensible_2D (MoistConvection input) */
    ATHAD_2D_VEL_STAR,              /* Array_2D vel_star, friction velocity [m/s]
                                     * (TurbulenceAtm::compute_vel_star; wall BC input) */
    ATHAD_2D_EPSILON,               /* Array_2D epsilon_2D, surface-layer emissivity     */
    ATHAD_2D_ALBEDO,                /* Array_2D albedo (MultiLayerRadiation)             */
    /* waterVapourEvaporation (ThermoAtm.h:115-398) outputs: the three evaporation laws
     * [mm/d] and the surface water vapour before the update */
    ATHAD_2D_EVAPORATION_DALTON, ATHAD_2D_EVAPORATION_MEYER, ATHAD_2D_EVAPORATION_ROHWER,
    ATHAD_2D_C_FIX,
    ATHAD_2D_CO2_TOTAL,             /* Array_2D co2_total, the column CO2 path [kg/m2]   */
    ATHAD_NFIELDS2D
} athad_field2d;

/* 1-D (im) profiles. */
typedef enum athad_profile {
    ATHAD_PROF_T_REF_LEVEL = 0,     /* computeLevelMeanTemperature, RK4.cpp:24-41     */
    ATHAD_PROF_RHO_BASE,            /* m_rho_base, ThermoAtm.h:1629-1646               */
    ATHAD_PROF_DLNRHO_DR,           /* m_dlnrho_dr, ThermoAtm.h:1652-1659              */
    ATHAD_NPROFILES
} athad_profile;

/* Per-iteration scalars of run_3D_loop (cAtmosphereModel.cpp:1109-1131). */
typedef struct athad_step_scalars {
    double dt;               /* dt = dt_visc (or dt_inviscid in the spin-up)           */
    double diffusion_ramp;   /* diffusion_ramp in [0,1]                                */
    double buoyancy_ramp;    /* min(1, total_iter_count / 300)                         */
    int32_t write_diagnostics; /* bit 0: store the right-hand side's diagnostic outputs of
                                * stage 4 - prod, tke_source, dis_source, the acting forces
                                * and Q_Latent, Q_Sensible in the interior cells (the
                                * reference writes them in every call; they are output
                                * only); bit 1: the momentum budget terms vbud_*, wbud_*
                                * (the reference's checkpoint iterations,
                                * cAtmosphereModel.cpp:1502-1503)                       */
    int32_t store_n_level;   /* 1: storeIntermediateData3D (UtilsAtm.h:25-49) fused into
                              * the last stage (the precipitation fluxes copied right
                              * after it): the caller runs nothing between the RK4 step
                              * and the time-level copy (no counterpart in the reference,
                              * which copies in a separate pass) */
} athad_step_scalars;

/* Counters a call leaves behind (read with athad_get_report). */
typedef struct athad_report {
    int64_t poisson_src_cells;     /* fluid cells of the last pressure call, summed over
                                    * its sweeps                                          */
    int64_t poisson_src_clamped;   /* of which the divergence source hit p_dyn_cap (the
                                    * pressure solve's sources are not counted)          */
    int64_t satadj_ceiling_hits;   /* c > 1 - co2 clamps in clampAndFade                  */
    int64_t nonfinite_inputs;      /* non-finite values of t seen by the last level mean (every
                                    * athad_rk4_step forms one from its input t)           */
    double  last_kernel_ms;        /* device time of the last athad_rk4_step (CUDA events on
                                    * the context's stream); 0 before the first            */
} athad_report;

/* What the vapour ceiling removed in one call (cAtmosphereModel.cpp:1369-1391). */
typedef struct athad_ceiling_report {
    int64_t n_ceiling;             /* cells where c was lowered to 1 - co2                 */
    int64_t pad0;
    double  q_clipped;             /* sum of the removed mass fraction x layer air mass [kg/m2] */
    double  w_air;                 /* sum of the layer air masses [kg/m2]                  */
} athad_ceiling_report;

/* cAtmosphereModel::searchMinMax_3D (MinMax_Atm.cpp:51-109): the largest and smallest
 * finite value of a field and the first cell in (i, j, k) order holding each; 0 at (0, 0, 0)
 * where the field has none. */
typedef struct athad_min_max_report {
    double  max, min;
    int32_t imax, jmax, kmax, imin, jmin, kmin;
} athad_min_max_report;

/* UtilsAtm::findResiduumAtm (UtilsAtm.h:70-220): the rms of the three normal velocity
 * derivatives over the band i = 10..30, j and k interior. */
typedef struct athad_residuum_report {
    double  residuum;              /* largest finite cell residual (0 if none is above 0)    */
    double  residuum_prev;         /* the previous call's residuum (residuum_old; 1e-5 before
                                    * the first call, cAtmosphereModel.h:164)              */
    double  avg_abs;               /* grid-average residual of the finite cells           */
    double  avg_rel;               /* avg_abs / residuum (0 if residuum is 0)              */
    int64_t n_cells;               /* finite cells of the band                            */
    int64_t n_nonfinite;           /* non-finite residuals, left out of the average        */
    int32_t i_error, j_error, k_error;   /* cell of the residuum: the smallest (i, j, k) on
                                          * equal values; 0, 0, 0 if none                 */
    int32_t i_nan, j_nan, k_nan;   /* first non-finite residual in (j, k, i) order; -1 if none */
} athad_residuum_report;

/* The global mass budgets of ThermoAtm::co2Column (ThermoAtm.h:1096-1137) and
 * ::waterBudget (:934-1094): the cos-latitude-weighted, air-mass-weighted mean mass fraction
 * of the species and its drift from the context's first call (the reference's m_q_co2_ref /
 * m_q_h2o_ref), summed in FP64 in a fixed order. */
typedef struct athad_budget_report {
    double q_mean, q_ref, drift_pct;   /* mean, first call's mean, 100 (q_mean / q_ref - 1)  */
    double q_fixed, q_fixed_ref, fixed_drift_pct;  /* water: the level means weighted by the
                                        * first call's level air masses, and its drift       */
    double air_now, air_ref, air_drift_pct;        /* water: total air mass and its drift   */
} athad_budget_report;

typedef struct athad_ctx athad_ctx;

/* ---- lifetime -------------------------------------------------------------- */

/* Fill p with the cli/config_cond.xml values and the reference's default switches. */
void athad_default_params(athad_params* p);
int32_t athad_abi_version(void);
size_t athad_params_size(void);

/* Create a context on the current CUDA device; allocates every field once.  Grids:
 * 4 <= im <= 1024, 5 <= jm <= 6144, km >= 5 (ATHAD_ERR_INVALID otherwise). */
athad_status athad_create(const athad_grid* grid, const athad_params* params, athad_ctx** out);
athad_status athad_destroy(athad_ctx* ctx);
const char*  athad_last_error(const athad_ctx* ctx);
/* Issue all further work on this stream (a cudaStream_t passed as void*); NULL = the
 * context's own stream. */
athad_status athad_set_stream(athad_ctx* ctx, void* cuda_stream);
athad_status athad_synchronize(athad_ctx* ctx);
/* Device bytes held by a context of this grid (admission by HBM footprint). */
size_t athad_footprint_bytes(const athad_grid* grid);
/* The same for a context created with these params (the mixed-precision step holds its
 * FP32 buffers in addition); 0 for an invalid grid or precision.  No counterpart in the
 * reference. */
size_t athad_footprint_bytes_params(const athad_grid* grid, const athad_params* params);

/* ---- state transfer --------------------------------------------------------- */

athad_status athad_upload(athad_ctx* ctx, athad_field f, const double* host, size_t n);
/* The same from a packed (i,j,k) buffer already in this device's memory (a state built on
 * the device); ordered on the context's stream.  No counterpart in the reference. */
athad_status athad_upload_device(athad_ctx* ctx, athad_field f, const double* device_src, size_t n);
athad_status athad_download(athad_ctx* ctx, athad_field f, double* host, size_t n);
athad_status athad_upload_2d(athad_ctx* ctx, athad_field2d f, const double* host, size_t n);
athad_status athad_download_2d(athad_ctx* ctx, athad_field2d f, double* host, size_t n);
athad_status athad_upload_profile(athad_ctx* ctx, athad_profile f, const double* host, size_t n);
athad_status athad_download_profile(athad_ctx* ctx, athad_profile f, double* host, size_t n);
/* athad_download_profile without the wait: the copy is enqueued on the context's stream and
 * the call returns.  host should be page-locked (into pageable memory CUDA completes the copy
 * before the call returns) and must stay valid until the stream has passed the copy
 * (athad_synchronize, or an event the caller records on the stream after the call); the
 * caller reads it only then.  A loop that reads each step's profile one step later keeps
 * the device busy while the host enqueues the next step. */
athad_status athad_download_profile_async(athad_ctx* ctx, athad_profile f, double* host, size_t n);
/* Device address and row pitch (in elements, >= km) of a field: element (i,j,k) is at
 * ptr[(i*jm + j)*pitch + k].  For zero-copy adapters and device-side consumers. */
athad_status athad_field_device_ptr(athad_ctx* ctx, athad_field f, double** ptr, size_t* pitch);
/* Fill a field with a constant on the device. */
athad_status athad_fill(athad_ctx* ctx, athad_field f, double value);

/* ---- the initial state --------------------------------------------------------- */

/* The configuration members the reference's initial state reads beyond athad_params
 * (cAtmosphereModel members of the same name; athad_default_init_config fills the values of
 * cli/config_cond.xml). */
typedef struct athad_init_config {
    uint32_t struct_size;        /* sizeof(athad_init_config)                             */
    int32_t  n_cells_hemisphere; /* prescribed circulation cells per hemisphere, 5        */
    int32_t  cell_amp_mode;      /* 0: unscaled amplitudes; 1, 2: scaled with cell_lat_scale */
    int32_t  pad0;
    double   t_surf_equator;     /* sea-surface temperature at the equator [K], 513.15   */
    double   t_surf_pole;        /* ... at the poles [K], 503.15                          */
    double   tropopause_equator; /* top of the convective column at the equator [m], 207000 */
    double   tropopause_pole;    /* ... at the poles [m], 195000                          */
    double   cell_lat_scale;     /* Hadley edge as a fraction of Earth's 30 degrees, 0.11 */
    double   co2_scale;          /* multiplier of the CO2 field, 1                        */
    double   q_CO2, q_bg;        /* mass fractions of CO2 and the background gas of the
                                  * configured composition (AtmMixture::resolve, m_comp):
                                  * co2Atmosphere's dry-air CO2 share q_CO2 / (q_CO2 + q_bg) */
    double   vel_star_init;      /* resetArrays' friction velocity [m/s], 0.4              */
} athad_init_config;

void athad_default_init_config(athad_init_config* c);

/* The reference's deterministic initial state, cAtmosphereModel::RunTimeSlice for Ma = 0
 * (cAtmosphereModel.cpp:468-668), built on the device for this context's grid, followed by
 * run_3D_loop's Held-Suarez target t_eq := t (:750-753): resetArrays, the tropopause levels,
 * the prescribed Hadley/Ferrel velocities (VelocityInitializer.h:23-105), the symmetric
 * parabolic sea-surface temperature with the dry adiabat (InitValues_Atm.cpp:466-620), the
 * saturated water profile (:843-926), two passes of co2Atmosphere and densities(true), the
 * cloud and ice profile (:930-1117), the saturation adjustment, the ice scheme, the moist
 * convection, the turbulence initialisation, the diagnosis block (with ThermoAtm::forces'
 * Coriolis and buoyancy arrays), the boundary conditions and the 200-sweep initial
 * projection, with every damp_wiggles between them.  Overwrites every field, 2-D field and
 * profile, the tropopause levels and the budgets' first-call references; leaves out the
 * outputs no field reads (precipitableWater, standAtm_DewPoint_HumidRel).  Rows are evaluated on the northern half and mirrored, so the
 * state is exactly north-south symmetric; the anchor row of latitude phi is
 * lround((90 - phi) (jm - 1) / 180), the reference's row at jm = 181.  Waits for the device. */
athad_status athad_initial_state(athad_ctx* ctx, const athad_init_config* config);

/* ---- the hot path ----------------------------------------------------------- */

/* storeIntermediateData3D(1.0) (UtilsAtm.h:25-49; call sites cAtmosphereModel.cpp:667,
 * 1647): tn..disn := t..dis and P_rainn, P_snown := P_rain, P_snow. */
athad_status athad_store_n_level(athad_ctx* ctx);

/* cAtmosphereModel::computeLevelMeanTemperature (RungeKutta_Atm_Turb.cpp:24-41):
 * fills the t_ref_level profile from t.  Mirror-symmetric, deterministic order. */
athad_status athad_level_mean(athad_ctx* ctx);

/* cAtmosphereModel::solveRungeKutta_Atmosphere_Turb (RungeKutta_Atm_Turb.cpp:44-273)
 * with RHS_Atmosphere_Turb (RHS_Atm_Turb.cpp:31-1080); call site
 * cAtmosphereModel.cpp:1509.  Computes t_ref_level, then the four RK4 stages over the
 * interior cells with Jacobi stage semantics (every stage reads the previous stage's
 * state everywhere).  Updates t..dis, aux_u/v/w and, with write_diagnostics, the stage-4
 * prod/tke_source/dis_source. */
athad_status athad_rk4_step(athad_ctx* ctx, const athad_step_scalars* s);

/* PressureSolverAtm::run (PressureSolverAtm.h:27-669); call site
 * cAtmosphereModel.cpp:1158.  n_sweeps red-black Gauss-Seidel sweeps of the pressure
 * Poisson equation with the source from aux_u/v/w, each followed by the boundary
 * conditions and the |p_dyn| ceiling.  total_iter_count selects the ceiling (10, or 3
 * after iteration 300). */
athad_status athad_pressure_sweep(athad_ctx* ctx, int32_t n_sweeps, int32_t total_iter_count);

/* PressureSolverAtm::project_initial_velocity (PressureSolverAtm.h:686-767); call site
 * cAtmosphereModel.cpp:665. */
/* Result of athad_pressure_solve. */
typedef struct athad_solve_report {
    int32_t iterations;        /* conjugate-gradient iterations                              */
    int32_t converged;         /* rel_residual <= rel_tol                                    */
    double  rel_residual;      /* ||b - A p||_2 / ||b||_2 at the end: b the projected source,
                                * A the sweep's operator with its boundary conditions (FP64) */
    double  history[64];       /* relative residual after iteration n (n <= 64)              */
    int32_t precond_levels;    /* multigrid levels of the FP32 preconditioner                */
    int32_t pad0;
    double  seconds;           /* device time of the solve                                   */
} athad_solve_report;

/* Solve the pressure-Poisson equation of the sweep to a relative residual: the fixed point
 * of PressureSolverAtm::run's red-black relaxation (PressureSolverAtm.h:225-552) for the
 * current aux_u/v/w, with the same clamped divergence source and boundary conditions,
 * without the |p| ceiling.  FP64 conjugate gradients preconditioned by an FP32 multigrid
 * V-cycle; the source is projected onto the operator's range (the operator has the
 * constants as its null space) and p_dyn is returned with zero interior mean.  The
 * multigrid hierarchy is allocated on the first call and kept by the context.  Not
 * supported with the anelastic term (ATHAD_ERR_UNSUPPORTED).  The reference has no such
 * call: it relaxes one sweep per call (athad_pressure_sweep). */
athad_status athad_pressure_solve(athad_ctx* ctx, double rel_tol, int32_t max_iter,
                                  athad_solve_report* report);
/* The per-iteration boundary conditions of cAtmosphereModel.cpp:1439-1446 for flat
 * terrain: BC_Atm::bcRadius (BC_Atm.h:556-746), TurbulenceAtm::apply_wall_bc
 * (TurbulenceAtm.h:109-147; reads the 2-D field ATHAD_2D_VEL_STAR), BC_Atm::bcTheta
 * (:750-796), BC_Atm::bcPhi (:803-918), BC_Atm::bcScalarSurfSur and BC_Atm::bcSolidGround
 * (without land only bcSolidGround's value limits over every cell act, :470-545: c, cloud,
 * ice, tke, dis >= 0; tke, dis, nue, prod, tke_source, dis_source, u, v, w and their time
 * level n bounded, non-finite values replaced), on the fields the context holds. */
athad_status athad_boundary_conditions(athad_ctx* ctx);
/* The filters after the RK4 step (cAtmosphereModel.cpp:1507-1520), flat terrain:
 * AtomUtils::polar_zonal_filter of u, v, w (lib/Utils.cpp:542-611), radial_shapiro_filter
 * of u (:831-873), radial_shapiro_filter_ho of v, w (:884-940); the orographic,
 * steep-massif and coastal filters change nothing without land.  Grids with km > 3072 are
 * rejected. */
athad_status athad_post_rk4_filters(athad_ctx* ctx);
/* AtomUtils::damp_wiggles(field, along i, j and k; strength 1, one pass), lib/Utils.cpp:
 * 429-531: what the moist iteration applies to t, ice, c and cloud after the saturation
 * adjustment (cAtmosphereModel.cpp:1225-1228).  Uses the RK4 stage buffers as scratch. */
athad_status athad_damp_wiggles(athad_ctx* ctx, athad_field field);
/* TurbulenceAtm(*this).run() (TurbulenceAtm.h:62-79; call sites cAtmosphereModel.cpp:614, 1426),
 * flat terrain: compute_vel_star into ATHAD_2D_VEL_STAR, compute_sources with the
 * configured closure (prod, nue, tke_source, dis_source; the floors of tke and dis) and
 * clamp_nue (the eddy-viscosity ceiling athad_params.abl_height).  Every cell reads the
 * state before the call: the reference's in-place sweep lets a cell see the floored tke/dis
 * of the neighbours visited before it, which differs only where a floor binds there. */
athad_status athad_turbulence_run(athad_ctx* ctx);
/* TwoCatIceScheme(*this).run() (TwoCatIceScheme.h:89-109; the configuration's
 * CategoryIceScheme = 2, call sites cAtmosphereModel.cpp:589, 1238), flat terrain: the
 * falling rain and snow restarted from ATHAD_P_RAINN/ATHAD_P_SNOWN, the COSMO sources and
 * sinks S_v, S_c, S_i, S_r, S_s (reading S_c_c), the capped fluxes P_rain, P_snow and
 * Precipitation, and their boundary extrapolation; cells where no condensed phase can exist
 * evaporate their condensate (IceSchemeCommon.h:121-190). */
athad_status athad_two_cat_ice_scheme(athad_ctx* ctx);
/* ZeroCatIceScheme(*this).run() (ZeroCatIceScheme.h:37-56; CategoryIceScheme = 0), flat
 * terrain: rain only.  Kessler autoconversion above 0.5 g/kg, accretion and evaporation give
 * S_v, S_c and S_r; the rain flux is integrated top-down from S_r of the cell above, uncapped;
 * P_snow keeps its restart value; P_rain is extrapolated with the seam average, P_snow
 * without.  Up to two passes per column until the rain flux at i = 23 settles, so the grid
 * needs im >= 24 (the reference reads level 23 whatever the grid; ATHAD_ERR_UNSUPPORTED
 * below). */
athad_status athad_zero_cat_ice_scheme(athad_ctx* ctx);
/* OneCatIceScheme(*this).run() (OneCatIceScheme.h:50-68; CategoryIceScheme = 1), flat
 * terrain: rain and snow with the COSMO one-category rates; snow grows through the shared
 * ice throttle (IceSchemeCommon.h:203-237); fluxes capped at 3e-3 kg/(m2 s).  The reference
 * walks the columns in one serial order (k outer, j inner) and keeps the autoconversion rate
 * S_au from the last cell with cloud water where a cell has none, across columns; the library
 * resolves that carry with a scan over the columns in the same order, so the result is the
 * reference's.  The carry before the first cloudy cell of the grid, uninitialised in the
 * reference, is 0 here.  im >= 24 as for athad_zero_cat_ice_scheme. */
athad_status athad_one_cat_ice_scheme(athad_ctx* ctx);
/* ThreeCatIceScheme(*this).run() (ThreeCatIceScheme.h:70-89; CategoryIceScheme = 3), flat
 * terrain: rain, snow and graupel, the fluxes normalised by the surface flux (floored at
 * 1e-6), the shared ice throttle, capped at 3e-3 kg/(m2 s); all three fluxes extrapolated
 * with the seam average.  im >= 24 as for athad_zero_cat_ice_scheme. */
athad_status athad_three_cat_ice_scheme(athad_ctx* ctx);
/* The switch of cAtmosphereModel.cpp:581-596 and 1230-1245 on athad_params.
 * category_ice_scheme: -1 runs nothing, 0..3 the schemes above. */
athad_status athad_ice_scheme(athad_ctx* ctx);
/* MultiLayerRadiation(*this).run() (MultiLayerRadiation.h:56-388; call sites
 * cAtmosphereModel.cpp:831-1007), flat terrain: per (j, k) column the grey long-wave
 * emissivities, four radiative-equilibrium sweeps and the surface energy balance.  Writes t
 * (the radiative equilibrium), ATHAD_RADIATION, ATHAD_EPSILON, ATHAD_2D_EPSILON and
 * ATHAD_2D_ALBEDO.  Uses RK4 stage buffers as scratch. */
athad_status athad_multilayer_radiation(athad_ctx* ctx);
/* Radiation mode 2 (cAtmosphereModel.cpp:799, 1655-1656): apply_radiative_heating
 * (:864-879), t := t (1 - omega_rad) + MultiLayerRadiation(t) omega_rad; the reference's
 * omega_rad is 0.05 (:801). */
athad_status athad_radiative_heating(athad_ctx* ctx, double omega_rad);
/* The moist iteration's bookkeeping after the moist convection: UtilsAtm::precipitationSum
 * (UtilsAtm.h:51-65; Precipitation = P_rain + P_snow + P_graupel + P_conv), the caps of the
 * microphysics sources S_v, S_c, S_i, S_r, S_s, S_g, S_c_c at +-1e-3 with non-finite values
 * set to 0 (cAtmosphereModel.cpp:1277-1297), and of cloud + ice at cloud_cap with c, cloud,
 * ice made finite, non-negative and c <= 1 - co2 (:1310-1334). */
athad_status athad_moist_caps(athad_ctx* ctx);
/* Water vapour's ceiling (cAtmosphereModel.cpp:1369-1391): c >= 0 and c <= 1 - co2 in every
 * cell.  With out non-NULL the call waits for the device and reports the clamped cells, the
 * air-mass-weighted water removed and the air mass (summed in a fixed order; the reference
 * accumulates m_q_h2o_clipped += q_clipped / w_air). */
athad_status athad_vapour_ceiling(athad_ctx* ctx, athad_ceiling_report* out);

/* ---- diagnostics and checkpoints ----------------------------------------------- */

/* searchMinMax_3D of one field (the values before the reference's unit conversion and
 * printing, MinMax_Atm.cpp:96-108).  Waits for the device.  Uses an RK4 stage buffer as
 * scratch. */
athad_status athad_min_max(athad_ctx* ctx, athad_field f, athad_min_max_report* out);
/* Checkpoint without stalling the model (the data of save_state, FileIO_Atm.cpp:293-356):
 * the n fields are snapshot on the device in stream order, then copied into the caller's
 * host arrays (packed (i, j, k), im*jm*km doubles each; page-locked memory makes the copy
 * asynchronous) on a side stream while later calls proceed.  The host arrays must stay valid
 * until athad_checkpoint_wait returns.  The first call, and a call with more fields than
 * before, allocates the snapshot (n fields of device memory outside the context's slab). */
/* UtilsAtm::findResiduumAtm (UtilsAtm.h:70-220; call sites cAtmosphereModel.cpp:668,
 * 1645, the end of every iteration of run_3D_loop).  The band is i = 10..30 as in the reference,
 * which needs im >= 32; on smaller grids it ends at im - 2 (and is empty for im < 12).  The
 * sum behind the average runs in a fixed order.  Waits for the device.  Uses an RK4 stage
 * buffer as scratch. */
athad_status athad_find_residuum(athad_ctx* ctx, athad_residuum_report* out);
/* The tropopause level of each colatitude row (cAtmosphereModel::tropopause_layers, built
 * by init_tropopause_layers, InitValues_Atm.cpp:330-401): jm values, each a level index in
 * [0, im-1].  Needed once before athad_stand_atm_dew_point. */
athad_status athad_set_tropopause_layers(athad_ctx* ctx, const double* layers, int32_t n);
/* ThermoAtm::standAtm_DewPoint_HumidRel (ThermoAtm.h:400-516; call sites
 * cAtmosphereModel.cpp:636, 1420), flat terrain: ATHAD_TEMP_STAND, ATHAD_TEMP_DEW_POINT
 * (SaturationH2O::dewPoint's 60-step bisection of the IAPWS curve at the exact vapour
 * pressure x_H2O p) and ATHAD_HUMIDITY_REL.  The reference takes the equator row's
 * tropopause from its neighbour by the literal row index 90; here that is the equator row
 * (jm-1)/2, the same row at jm = 181 and mirror-symmetric on every grid. */
athad_status athad_stand_atm_dew_point(athad_ctx* ctx);
/* ThermoAtm::waterVapourEvaporation (ThermoAtm.h:115-398; call sites
 * cAtmosphereModel.cpp:637, 1421), flat terrain: the sea surface as a saturation boundary.
 * Per (j, k) column below the critical temperature, the surface water vapour relaxes toward
 * the sea's saturation mass fraction and the change spreads over levels 1-3 with weights
 * e^-i, capped at each level's saturation; the Dalton, Meyer and Rohwer evaporation rates of
 * the saturation deficit are reported (ATHAD_2D_EVAPORATION = Dalton's).  The reference's
 * Earth branch after this block is unreachable and not built. */
athad_status athad_water_vapour_evaporation(athad_ctx* ctx);
/* ThermoAtm::latentSensibleHeat (ThermoAtm.h:36-112; call sites cAtmosphereModel.cpp:638,
 * 1422): Q_Latent zeroed at the surface, Q_Sensible = cp_l t_0 |grad t| / sqrt(3) in the
 * interior. */
athad_status athad_latent_sensible_heat(athad_ctx* ctx);
/* cAtmosphereModel::updateSkinTemperature (cAtmosphereModel.cpp:291-327; called after the
 * radiative heating of radiation mode 2, :1661) with planetaryShortWave (:236-265): the
 * optically thin top's skin temperature relaxed by t_skin_relax (XML, 0.25) toward
 * ((absorbed short wave + geothermal flux) / sigma)^(1/4), the absorbed short wave being the
 * cos-latitude mean of (1 - albedo) times the pole-to-equator insolation profile, from
 * ATHAD_2D_ALBEDO.  Changes the context's t_skin (read by athad_densities); t_skin, if not
 * NULL, receives it.  Nothing changes where the reference returns early (t_skin_relax <= 0,
 * no positive albedo, no positive absorbed flux).  Waits for the device. */
athad_status athad_update_skin_temperature(athad_ctx* ctx, double t_skin_relax, double* t_skin);
/* ThermoAtm::forces (ThermoAtm.h:518-614; call sites cAtmosphereModel.cpp:635, 1419): the
 * two arrays it shares with the right-hand side's outputs, ATHAD_CORIOLIS_FORCE and
 * ATHAD_BUOYANCY_FORCE of the interior cells (its centrifugal and pressure-gradient arrays
 * are output only and not held).  The buoyancy reference is the level-mean temperature
 * once one exists (an athad_rk4_step, athad_level_mean or an upload of
 * ATHAD_PROF_T_REF_LEVEL since the context's creation or initial state), else 1, as the
 * reference's empty t_ref_level gives before its first RK4 step. */
athad_status athad_forces(athad_ctx* ctx);
/* ThermoAtm::co2Column (ThermoAtm.h:1096-1137; call sites cAtmosphereModel.cpp:632, 1416):
 * ATHAD_2D_CO2_TOTAL and the CO2 budget.  Waits for the device. */
athad_status athad_co2_column(athad_ctx* ctx, athad_budget_report* out);
/* ThermoAtm::waterBudget (ThermoAtm.h:934-1094; call sites cAtmosphereModel.cpp:633, 1216,
 * 1417): the water budget (c + cloud + ice + graupel); level_drift, if not NULL, receives the
 * im per-level drifts of the water mass fraction from the first call (the reference prints
 * the six largest).  Waits for the device. */
athad_status athad_water_budget(athad_ctx* ctx, athad_budget_report* out, double* level_drift);
athad_status athad_checkpoint_begin(athad_ctx* ctx, const int32_t* fields, int32_t n, double* const* hosts);
athad_status athad_checkpoint_wait(athad_ctx* ctx);
athad_status athad_project_initial_velocity(athad_ctx* ctx, int32_t n_sweeps,
                                            int32_t total_iter_count);

/* SaturationAdjustment::run (SaturationAdjustment.h:25-45); call sites
 * cAtmosphereModel.cpp:574, 1218. */
athad_status athad_saturation_adjust(athad_ctx* ctx);

/* ThermoAtm::densities (ThermoAtm.h:1436-1666); call sites cAtmosphereModel.cpp:567
 * (set_water_profile = 1), 634, 1418. */
athad_status athad_densities(athad_ctx* ctx, int32_t set_water_profile);

/* MoistConvection::run (MoistConvection.h:106-140); call sites cAtmosphereModel.cpp:599,
 * 1247. */
athad_status athad_moist_convection(athad_ctx* ctx, int32_t iter_n);

/* Counters of the last calls. */
athad_status athad_get_report(athad_ctx* ctx, athad_report* out);

/* ---- ensembles: batched iteration of many contexts ----------------------------
 * No counterpart in the reference, which runs one grid per process.  A batch advances
 * mixed-precision contexts (members, each with its own grid and parameters) together on
 * one stream: every member's column physics at its own cadence, the level mean of all
 * members in one launch, each RK4 stage of all members in one persistent launch, the
 * time-level copy (storeIntermediateData3D) fused into the last stage.  The members stay
 * ordinary contexts: upload/download work on them between batch calls (on the batch's
 * stream order: call athad_batch_synchronize first).  A member's result is bit-for-bit
 * the result of the same iterations run on it alone through athad_rk4_step and friends
 * with the same scalars. */
typedef struct athad_batch athad_batch;

typedef struct athad_batch_step {
    double  dt;                   /* non-dimensional time step (dt_visc, cli/config_cond.xml: 4e-5) */
    double  diffusion_ramp;       /* 1 */
    int32_t buoyancy_ramp_iters;  /* buoyancy ramp of iteration n = min(1, n / this); 300 */
    int32_t pad0;
} athad_batch_step;

/* members: n_members distinct MIXED contexts on the current device; first_iter: each
 * member's next iteration number (NULL = all 1).  The batch holds small device tables
 * only.  Creation waits for the work already queued on the members' streams (an initial
 * state being built, an upload), since the batch runs the members on its own streams. */
athad_status athad_batch_create(athad_ctx* const* members, int32_t n_members,
                                const athad_batch_step* step, const int32_t* first_iter,
                                athad_batch** out);
athad_status athad_batch_destroy(athad_batch* b);
const char*  athad_batch_last_error(const athad_batch* b);
athad_status athad_batch_set_stream(athad_batch* b, void* cuda_stream);
athad_status athad_batch_synchronize(athad_batch* b);
/* A member's next iteration number. */
athad_status athad_batch_member_iter(const athad_batch* b, int32_t member, int32_t* next_iter);
/* An inactive member is skipped by every launch (its state and counter stay). */
athad_status athad_batch_set_active(athad_batch* b, int32_t member, int32_t active);
/* One model iteration of every active member (cadence of cAtmosphereModel.cpp:1156-1509). */
athad_status athad_batch_iteration(athad_batch* b);
/* The same iteration replayed from a CUDA graph, captured on first use for the current
 * cadence pattern of the members (at most a few per batch). */
athad_status athad_batch_iteration_graph(athad_batch* b);
/* Tile shapes of the persistent RK4 kernel; athad_batch_autotune times RK4 stages 1-3 of
 * the whole batch once per shape (reps repetitions, model state unchanged), keeps the
 * fastest and reports each shape's milliseconds per stage triple. */
int32_t      athad_batch_shape_count(void);
athad_status athad_batch_set_shape(athad_batch* b, int32_t shape);
athad_status athad_batch_autotune(athad_batch* b, int32_t reps, int32_t* best_shape,
                                  float* ms_per_shape);

/* ---- the device thermodynamics, for the known-answer tests ---------------------- */

/* The saturation and mixture functions the column kernels evaluate on the device
 * (SaturationH2O.h:68-303, MixtureAtm.h:123-225), evaluated on the GPU for n input tuples so
 * the reference's self-test values (test/saturation_selftest.cpp,
 * test/cond_column_selftest.cpp) can be checked against the device code.  Arguments per
 * function, in order: */
typedef enum athad_thermo_fn {
    ATHAD_THERMO_SATURATION_PRESSURE = 1,      /* T -> p_sat [hPa] (-1 where none)          */
    ATHAD_THERMO_SUBLIMATION_PRESSURE,         /* T -> p_subl [hPa]                         */
    ATHAD_THERMO_LATENT_HEAT,                  /* T -> L [J/kg]                             */
    ATHAD_THERMO_SATURATION_MASS_FRACTION,     /* E, p, M_other -> q_sat                    */
    ATHAD_THERMO_DEW_POINT,                    /* e [hPa] -> T_dew [K]                      */
    ATHAD_THERMO_CP_OF,                        /* c, co2, T, M_bg -> cp [J/(kg K)]          */
    ATHAD_THERMO_M_NONWATER,                   /* c, co2, M_bg -> M [kg/mol]                */
    ATHAD_THERMO_MOIST_LAPSE,                  /* T, p, M_other, cp, R_mix, g -> lapse [K/m] */
    ATHAD_THERMO_R_OF,                         /* c, co2, R_bg -> R [J/(kg K)]              */
    ATHAD_THERMO_SATURATION_MASS_FRACTION_AT,  /* T, p, M_other -> q_sat                    */
    ATHAD_THERMO_DQSAT_DT                      /* T, p, M_other -> dq_sat/dT [1/K]          */
} athad_thermo_fn;
/* Inputs per tuple (0 for an unknown function). */
int32_t athad_thermo_arity(int32_t fn);
/* in: n tuples of athad_thermo_arity(fn) doubles (host memory); out: n doubles (host).
 * Synchronous; allocates device memory for the call. */
athad_status athad_thermo_eval(int32_t fn, int32_t n, const double* in, double* out);

/* ---- allocation-free entry point --------------------------------------------- */

/* Largest grid athad_density_profile_noalloc accepts: im*jm (i, j) rows, im levels. */
#define ATHAD_NOALLOC_MAX_ROWS 131072
#define ATHAD_NOALLOC_MAX_IM   1024

/* No counterpart in the reference: an addition for callers that cannot allocate device
 * memory when they need this result (a host that reserved its whole HBM budget up front,
 * a real-time loop that cannot afford cudaMalloc's implicit synchronisation, a caller
 * whose device buffers come from another runtime).  It computes what athad_densities
 * leaves in ATHAD_PROF_RHO_BASE and ATHAD_PROF_DLNRHO_DR - the cos-latitude horizontal
 * mean of the density and d ln(rho_bar)/d rad.z - from a density field the caller holds on
 * the device (element (i,j,k) at r_humid[(i*jm + j)*pitch + k]) into two caller-provided
 * device arrays of im doubles, on the given stream (a cudaStream_t, NULL = default
 * stream), without a context and without allocating: its scratch is a fixed device array
 * of 2 * ATHAD_NOALLOC_MAX_ROWS doubles (2 MiB) that every GPU loading the library keeps
 * until exit.  Grids beyond im*jm > ATHAD_NOALLOC_MAX_ROWS or im > ATHAD_NOALLOC_MAX_IM are
 * rejected with ATHAD_ERR_INVALID.  The first call on a device looks up the scratch
 * address (make it before any stream capture) and keeps it for the life of the process:
 * cudaDeviceReset between calls is not supported.  All calls share the scratch, so calls
 * that overlap on the GPU race; calls ordered on one stream do not.  A CUDA error pending
 * from earlier work is reported as ATHAD_ERR_CUDA without launching.  Asynchronous: the
 * outputs are ready when the stream is. */
athad_status athad_density_profile_noalloc(const double* r_humid, int32_t im, int32_t jm,
                                           int32_t km, size_t pitch, double* rho_base,
                                           double* dlnrho_dr, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* ATHAD_GPU_H */
