/*
 * athad_oracle.h - CPU restatement of the ATHAD_COND model-iteration hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is what the CUDA path is compared against; it
 * is never linked into, loaded by or called from the product.  Only tests/, the smoke()
 * entry point and the cpu_baseline leg of bench.py use it.
 *
 * Plain C99, FP64, compiled without -ffast-math and with -ffp-contract=off so every
 * operation rounds as written.  Each function cites the reference file:line it follows.
 *
 * Two semantics are available through the `compat` argument:
 *   compat = 0  the semantics the CUDA path implements: Jacobi RK4 stages, trig tables
 *               and theta second differences written so that the result is exactly
 *               north-south mirror symmetric, a pairwise (mirror-invariant) level mean.
 *   compat = 1  the reference's own semantics, operation for operation: the in-place,
 *               cell-by-cell RK4 sweep of RungeKutta_Atm_Turb.cpp:99-266 in serial order
 *               (OMP_NUM_THREADS=1), the reference's trig tables and expression order.
 *               Used to pin this restatement against the reference built from source.
 *
 * The field pointers are packed host arrays in (i, j, k) order, k fastest, indexed by
 * the athad_field enumeration of include/athad_gpu.h (re-declared here as plain ints so
 * this file does not include product headers).
 */
#ifndef ATHAD_ORACLE_H
#define ATHAD_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_params {
    uint32_t struct_size;
    int32_t  turb_model, wall_mode, poisson_metric_fix, anelastic, tracer_diff_flux;
    int32_t  coriolis_nontrad, metric_curvature, metric_divergence;
    int32_t  convection_perturbation, convection_mode, iter_prec, precision;   /* precision: unused by the oracle (FP64) */
    int32_t  category_ice_scheme;
    double metric_r0, re_turb;
    double r_air, g, u_0, cp_l, t_0, c_0, L_atm, zeta, omega, lamda, lv, ls;
    double pr_turb, sc_WaterVapour, sc_CO2;
    double r_Earth, p_0, t_00, t_max_phys, cloud_cap, t_skin, c_h2o_dry_top, co2_0, s_0;
    double R_Air, R_WaterVapour;
    double M_bg, R_bg, R_mix;
    double abl_height, t_000;
    double sigma, kappa_H2O, kappa_CO2, kappa_bg, geothermal_flux, albedo_surface, albedo_cloud;
    double rad_equator_short, rad_pole_short;
    double coeff_Dalton;
    double r_0_water;
} or_params;

typedef struct or_step {
    double dt, diffusion_ramp, buoyancy_ramp;
    int32_t write_diagnostics, pad0;
} or_step;

/* field ids, identical numbering to athad_field */
enum {
    OF_T = 0, OF_U, OF_V, OF_W, OF_C, OF_CLOUD, OF_ICE, OF_GR, OF_CO2, OF_TKE, OF_DIS,
    OF_TN, OF_UN, OF_VN, OF_WN, OF_CN, OF_CLOUDN, OF_ICEN, OF_GRN, OF_CO2N, OF_TKEN, OF_DISN,
    OF_P_DYN, OF_NUE, OF_T_EQ, OF_P_STAT, OF_R_HUMID,
    OF_S_C, OF_S_R, OF_S_I, OF_S_S, OF_S_G, OF_S_V,
    OF_MC_T, OF_MC_Q, OF_MC_V, OF_MC_W,
    OF_AUX_U, OF_AUX_V, OF_AUX_W,
    OF_PROD, OF_TKE_SOURCE, OF_DIS_SOURCE,
    OF_S_C_C, OF_P_RAIN, OF_P_SNOW, OF_P_GRAUPEL, OF_PRECIPITATION,
    OF_R_DRY,
    OF_MC_S, OF_MC_S_U, OF_MC_S_D, OF_M_U, OF_M_D,
    OF_Q_V_U, OF_Q_C_U, OF_Q_V_D,
    OF_U_U, OF_V_U, OF_W_U, OF_U_D, OF_V_D, OF_W_D,
    OF_E_U, OF_D_U, OF_E_D, OF_D_D,
    OF_C_U, OF_E_L, OF_E_DD, OF_E_P, OF_G_P,
    OF_P_CONV, OF_CLOUD_BASE, OF_LEVEL_FREE_SINKING, OF_DEEP_BEG, OF_DEEP_END,
    OF_P_RAINN, OF_P_SNOWN,
    OF_RADIATION, OF_EPSILON,
    OF_TEMP_STAND, OF_TEMP_DEW_POINT, OF_HUMIDITY_REL,
    OF_Q_LATENT, OF_Q_SENSIBLE,
    OF_CORIOLIS_FORCE, OF_BUOYANCY_FORCE, OF_PRESSURE_GRADIENT_FORCE,
    OF_VBUD_PGF, OF_VBUD_COR, OF_VBUD_ADVV, OF_VBUD_ADVH, OF_VBUD_DIFF, OF_VBUD_OTHER,
    OF_WBUD_PGF, OF_WBUD_COR, OF_WBUD_ADVV, OF_WBUD_ADVH, OF_WBUD_DIFF, OF_WBUD_OTHER,
    OF_NFIELDS
};
enum { OF2_T_TOP_INIT = 0, OF2_P_STAT_LANDSCAPE, OF2_EVAPORATION, OF2_Q_SENSIBLE, OF2_VEL_STAR,
       OF2_EPSILON, OF2_ALBEDO, OF2_EVAPORATION_DALTON, OF2_EVAPORATION_MEYER,
       OF2_EVAPORATION_ROHWER, OF2_C_FIX, OF2_CO2_TOTAL, OF2_N };
enum { OFP_T_REF_LEVEL = 0, OFP_RHO_BASE, OFP_DLNRHO_DR, OFP_N };

size_t or_params_size(void);
int    or_nfields(void);

/* computeLevelMeanTemperature, RungeKutta_Atm_Turb.cpp:24-41 */
void or_level_mean(int im, int jm, int km, const or_params* p, int compat,
                   double* const* f, double* const* prof);

/* solveRungeKutta_Atmosphere_Turb + RHS_Atmosphere_Turb, RungeKutta_Atm_Turb.cpp:44-273,
 * RHS_Atm_Turb.cpp:31-1080.  Returns 0, or -1 on a configuration the restatement does
 * not cover. */
int or_rk4(int im, int jm, int km, const or_params* p, const or_step* s, int compat,
           double* const* f, double* const* prof);

void or_rhs_cell_at(int im, int jm, int km, const or_params* p, const or_step* s, int compat,
                    double* const* f, double* const* prof, int i, int j, int k, double* out);

/* PressureSolverAtm::run, PressureSolverAtm.h:27-594.  counters[0] = fluid cells,
 * counters[1] = clamped sources (may be NULL). */
void or_pressure_sweep(int im, int jm, int km, const or_params* p, int compat,
                       int n_sweeps, int total_iter_count, double* const* f,
                       double* const* prof, int64_t* counters);

/* PressureSolverAtm::project_initial_velocity, PressureSolverAtm.h:686-767 */
void or_project_initial_velocity(int im, int jm, int km, const or_params* p, int compat,
                                 int n_sweeps, int total_iter_count, double* const* f,
                                 double* const* prof);

/* SaturationAdjustment::run, SaturationAdjustment.h:25-459.  counters[0] = ceiling hits */
void or_saturation_adjust(int im, int jm, int km, const or_params* p, int compat,
                          double* const* f, int64_t* counters);

/* the layer heights [im] and SaturationAdjustment's level steps [im] (computeSteps,
 * SaturationAdjustment.h:56-60: float differences) that the two column passes use */
int or_column_geometry(int im, int jm, int km, const or_params* p, int compat, double* height,
                       double* step_f);

/* ThermoAtm::densities, ThermoAtm.h:1436-1666 */
void or_densities(int im, int jm, int km, const or_params* p, int compat,
                  int set_water_profile, double* const* f, double* const* f2,
                  double* const* prof);

/* MoistConvection::run, MoistConvection.h:106-140 */
int or_moist_convection(int im, int jm, int km, const or_params* p, int compat, int iter_n,
                        double* const* f, double* const* f2);
/* the geometry or_moist_convection uses: layer heights [im], level steps [im] (double
 * differences, MoistConvection.h:300-309) and cos(theta_equator - theta_j) [jm] (:239) */
int or_moist_geometry(int im, int jm, int km, const or_params* p, int compat, double* height,
                      double* step, double* cose);

/* the per-iteration boundary conditions, cAtmosphereModel.cpp:1439-1446: BC_Atm::bcRadius,
 * TurbulenceAtm::apply_wall_bc, BC_Atm::bcTheta, BC_Atm::bcPhi, BC_Atm::bcScalarSurfSur and
 * BC_Atm::bcSolidGround (flat terrain: the value limits of BC_Atm.h:470-545) */
void or_boundary_conditions(int im, int jm, int km, const or_params* p, double* const* f,
                            double* const* f2);

/* the filters after the RK4 step (cAtmosphereModel.cpp:1507-1520): polar zonal filter of
 * u, v, w; radial Shapiro filter of u; 4th-order radial Shapiro filter of v, w (flat
 * terrain) */
void or_post_rk4_filters(int im, int jm, int km, const or_params* p, double* const* f);
/* AtomUtils::damp_wiggles(field, along i, j, k), lib/Utils.cpp:429-531 */
void or_damp_wiggles(int im, int jm, int km, double* field, int compat);
int  or_polar_passes(int jm, int j, const double* sin_w);

/* TurbulenceAtm::run, TurbulenceAtm.h:62-79 (compute_vel_star, compute_sources with the
 * k-epsilon, k-omega or k-omega SST closure, clamp_nue), flat terrain.  compat = 1: the
 * reference's serial in-place sweep (j, k, i loops; a cell reads the floored tke/dis of the
 * neighbours processed before it); compat = 0: every cell reads the values before the call
 * (the device form). */
void or_turbulence_run(int im, int jm, int km, const or_params* p, int compat,
                       double* const* f, double* const* f2);

/* TwoCatIceScheme::run, TwoCatIceScheme.h:89-109 (initArrays, computeColumns,
 * applyBoundaryConditions; applyTopography does nothing without land), flat terrain */
void or_two_cat_ice_scheme(int im, int jm, int km, const or_params* p, double* const* f);
/* ZeroCatIceScheme::run, OneCatIceScheme::run, ThreeCatIceScheme::run (im >= 24: the
 * schemes read level 23); or_ice_scheme: the CategoryIceScheme switch (-1 .. 3) */
void or_zero_cat_ice_scheme(int im, int jm, int km, const or_params* p, double* const* f);
void or_one_cat_ice_scheme(int im, int jm, int km, const or_params* p, double* const* f);
void or_three_cat_ice_scheme(int im, int jm, int km, const or_params* p, double* const* f);
void or_ice_scheme(int im, int jm, int km, const or_params* p, double* const* f);

/* MultiLayerRadiation::run (MultiLayerRadiation.h:56-388): t := the radiative equilibrium;
 * radiation, epsilon, epsilon_2D, albedo.  or_radiative_heating: radiation mode 2's
 * apply_radiative_heating (cAtmosphereModel.cpp:864-879), t := t (1 - omega) + RE omega. */
void or_multilayer_radiation(int im, int jm, int km, const or_params* p, double* const* f,
                             double* const* f2);
void or_radiative_heating(int im, int jm, int km, const or_params* p, double omega_rad,
                          double* const* f, double* const* f2);

/* the moist iteration's caps (UtilsAtm.h:51-65, cAtmosphereModel.cpp:1277-1334) and the
 * vapour ceiling (:1369-1391) with its sums in the reference's serial order */
void or_moist_caps(int im, int jm, int km, const or_params* p, double* const* f);
void or_vapour_ceiling(int im, int jm, int km, const or_params* p, double* const* f,
                       int64_t* n_ceiling, double* q_clipped, double* w_air);

/* searchMinMax_3D, MinMax_Atm.cpp:51-109 */
void or_min_max(int im, int jm, int km, const double* x, double* out, int* idx);

/* UtilsAtm::findResiduumAtm (UtilsAtm.h:70-220) over the band i = 10 .. min(30, im-2):
 * out = residuum (largest finite residual, 0 if none above 0), grid-average residual,
 * average / residuum; cnt = finite cells, non-finite cells; idx = i, j, k of the residuum
 * (smallest (i, j, k) on ties; 0, 0, 0 if none) and of the first non-finite residual in the
 * serial (j, k, i) order (-1, -1, -1 if none). */
void or_find_residuum(int im, int jm, int km, double* const* f, double* out, int64_t* cnt, int* idx);

/* ThermoAtm::standAtm_DewPoint_HumidRel (ThermoAtm.h:400-516), flat terrain: TempStand,
 * TempDewPoint, HumidityRel.  i_trop[j] = the tropopause level the row uses (the equator
 * row already given its neighbour's value). */
void or_stand_atm_dew_point(int im, int jm, int km, const or_params* p, double* const* f,
                            const int* i_trop);

/* ThermoAtm::waterVapourEvaporation (ThermoAtm.h:115-398) and ::latentSensibleHeat
 * (:36-112), flat terrain */
void or_water_vapour_evaporation(int im, int jm, int km, const or_params* p, double* const* f,
                                 double* const* f2);
void or_latent_sensible_heat(int im, int jm, int km, const or_params* p, int compat, double* const* f);

/* cAtmosphereModel::updateSkinTemperature (cAtmosphereModel.cpp:291-327) with
 * planetaryShortWave (:236-265) from the albedo [jm][km]: the new t_skin */
double or_update_skin_temperature(int jm, int km, const or_params* p, const double* albedo,
                                  double t_skin, double t_skin_relax);

/* ThermoAtm::co2Column (ThermoAtm.h:1096-1137): co2_total and the mass-weighted mean q_CO2,
 * in the reference's serial (j, k, i) order; out = w_num, w_den. */
void or_co2_column(int im, int jm, int km, const or_params* p, double* const* f, double* const* f2,
                   double* out);
/* ThermoAtm::waterBudget (ThermoAtm.h:934-1094), the sums before the reference's first-call
 * bookkeeping: out = w_num, w_den; qbar, abar, lev [im] */
void or_water_budget(int im, int jm, int km, const or_params* p, double* const* f, double* out,
                     double* qbar, double* abar, double* lev);

/* the per-iteration boundary conditions without (wall_bc = 0) or with (1) the turbulence wall
 * values; RunTimeSlice's boundary conditions (cAtmosphereModel.cpp:651-653) have none.
 * or_turb_wall_bc: TurbulenceAtm::apply_wall_bc alone (TurbulenceAtm.h:109-147). */
void or_boundary_conditions_ex(int im, int jm, int km, const or_params* p, double* const* f,
                               double* const* f2, int wall_bc);
void or_turb_wall_bc(int im, int jm, int km, const or_params* p, double* const* f, double* const* f2);

/* The reference's deterministic initial state (cAtmosphereModel::RunTimeSlice, Ma = 0,
 * cAtmosphereModel.cpp:468-668, then run_3D_loop's t_eq := t, :750-753): the configuration
 * members it reads beyond or_params, laid out as athad_init_config. */
typedef struct or_init_cfg {
    uint32_t struct_size;
    int32_t  n_cells_hemisphere, cell_amp_mode, pad0;
    double   t_surf_equator, t_surf_pole, tropopause_equator, tropopause_pole;
    double   cell_lat_scale, co2_scale, q_CO2, q_bg, vel_star_init;
} or_init_cfg;
/* stages of or_init_state's `upto`, in the reference's order */
enum { OR_INIT_VELOCITY = 1, OR_INIT_TEMPERATURE, OR_INIT_WATER, OR_INIT_CLOUD, OR_INIT_SATADJ,
       OR_INIT_ICE, OR_INIT_MOIST, OR_INIT_TURBULENCE, OR_INIT_DIAGNOSE, OR_INIT_BC,
       OR_INIT_PROJECT, OR_INIT_ALL };
size_t or_init_cfg_size(void);
/* init_tropopause_layers (InitValues_Atm.cpp:330-401): jm levels */
void or_tropopause_layers(int im, int jm, const or_params* p, const or_init_cfg* c, double* levels);
/* every field, 2-D field and profile is overwritten; returns 0, -1 on a bad config */
int or_init_state(int im, int jm, int km, const or_params* p, const or_init_cfg* c, int compat, int upto,
                  double* const* f, double* const* f2, double* const* prof);

/* ThermoAtm::forces (ThermoAtm.h:518-614): CoriolisForce and BuoyancyForce of the interior
 * cells; t_ref the level-mean temperature, NULL before the first RK4 step (reference 1) */
void or_forces(int im, int jm, int km, const or_params* p, int compat, double* const* f,
               const double* t_ref);

/* storeIntermediateData3D, UtilsAtm.h:25-49 */
void or_store_n_level(int im, int jm, int km, double* const* f);

/* Thermodynamics (SaturationH2O.h, MixtureAtm.h), exposed for the known-answer tests. */
double or_saturation_pressure(double T);
double or_sublimation_pressure(double T);
double or_latent_heat(double T);
double or_saturation_mass_fraction(double E, double p, double M_other);
double or_dew_point(double e);
double or_dqsat_dT(double T, double p, double M_other);
double or_moist_lapse(double T, double p, double M_other, double cp, double R_mix, double g);
double or_cp_of(double c, double co2, double T, double M_bg);
double or_R_of(double c, double co2, double R_bg);
double or_M_nonwater(double c, double co2, double M_bg);
double or_x_H2O_of(double c, double co2, double M_bg);
void   or_resolve(const double* x8, double* out7);   /* M_mean, R_mix, q_H2O, q_CO2, q_bg, M_bg, R_bg */

#ifdef __cplusplus
}
#endif
#endif
