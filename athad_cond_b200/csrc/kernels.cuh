// kernels.cuh - launch interface of the sm_100a kernels of the ATHAD_COND hot path.
// Every launcher issues on the given stream and returns without synchronising.
#pragma once

#include "common.cuh"

// The RK4 stage launches (single grid, both forms) walk the radial planes forward in the odd
// stages and backward in the even ones, so that a stage starts on the planes the stage
// before it wrote last; measured 0.6 % on the mixed step, neutral on FP64.
#ifndef ATHAD_RK4_SERPENTINE
#define ATHAD_RK4_SERPENTINE 1
#endif

namespace athad {

// Argument block of the RK4 stage kernels.  Field pointers are pitched device arrays.
struct RK4Args {
    Dims d;
    const GeoIJ* geo;          // [im*jm]
    const double* t_ref;       // [im]   level-mean temperature
    const double* dlnrho;      // [im]   d ln rho_bar / d rad.z
    const double* Yin[11];     // stage state read (stencil)
    double*       Yout[11];    // stage state written
    const double* Yn[11];      // time level n
    double*       K[11];       // RK4 accumulator k1 + 2 k2 + 2 k3
    double*       Ybnd[11];    // stage 1 only: second stage buffer that receives the boundary
    double*       Yn_store[11];    // store_n: stage 4 also writes the new time level n here
    const double* p_dyn;
    const double* nue;
    const double* t_eq;
    const double* p_stat;
    const double* r_humid;
    const double* S_c; const double* S_r; const double* S_i; const double* S_s;
    const double* S_g; const double* S_v;
    const double* MC_t; const double* MC_q; const double* MC_v; const double* MC_w;
    double* aux_u; double* aux_v; double* aux_w;
    double* prod; double* tke_source; double* dis_source;
    // constants
    double inv_2dr, inv_2dthe, inv_2dphi, inv_dr2, inv_dthe2, inv_dphi2;
    double dt, half_dt, dt_sixth, diffusion_ramp, buoyancy_ramp, tke_max_nd, force_nd;
    double coeff_energy_p, coeff_energy, coeff_MC_vel, coeff_MC_q, coeff_MC_t;
    double lv, ls, g, u_0, L_atm, re_turb, pr_turb, sc_WaterVapour, sc_CO2;
    // launch constants the reference evaluates per cell from the same operands (hoisted,
    // values identical): 1/re_turb, 1000/(u_0 L_atm), 1.5e-5/(u_0 L_atm), the tracer
    // diffusivities, the buoyancy prefactor buoyancy_ramp*1*g*dt/u_0 and the drag
    // prefactor (1/86400)*L_atm/u_0*dt
    double inv_re, nue_max, nue_air_nd, diff_prec_re_inv, diff_co2_re_inv, buoy_pref, drag_pref;
    int turb_model, wall_mode, nontrad, curvature, tracer_diff_flux, write_diag;
    int store_n;               // fuse storeIntermediateData3D into stage 4
};

// The right-hand side's diagnostic outputs (k_rhsdiag.cu): out[0..2] CoriolisForce,
// BuoyancyForce, PressureGradientForce, [3..4] Q_Latent, Q_Sensible (flags bit 0),
// [5..10] vbud_*, [11..16] wbud_* (flags bit 1); the last stage's input state in FP64 or FP32.
struct RhsDiagArgs {
    Dims d;
    const GeoIJ* geo;
    const double* t_ref;
    const double* p_dyn; const double* nue; const double* MC_v; const double* MC_w;
    const double* Y64[11];      // the state read: FP64 (Y32[0] null) or FP32 stage buffers
    const float* Y32[11];
    double* out[17];
    double inv_2dr, inv_2dthe, inv_2dphi, inv_dr2, inv_dthe2, inv_dphi2;
    double coeff_Coriolis, coeff_buoy, coeff_u_p, coeff_L, coeff_S, t_0;
    double inv_re, diffusion_ramp, drag_pref, force_nd, coeff_MC_vel;
    int nontrad, flags;
};
void launch_rhs_diagnostics(const RhsDiagArgs& a, cudaStream_t st);

void launch_level_mean(const Dims& d, const double* t, const double* sin_w, double* out,
                       double* row_sum, cudaStream_t st, unsigned long long* nonfinite = nullptr);
void launch_rk4_stage(int stage, const RK4Args& a, cudaStream_t st);

// Mixed-precision RK4 step (k_rk4m.cu).  FP32 geometry factors (rounded from GeoIJ, so
// still mirror-exact) and the packed FP32 forcing fields stage 1 writes.
struct GeoF {
    float exp_rm, exp_2_rm, sinthe, costhe, inv_rm, inv_rm2, inv_rmsinthe, inv_rm2sinthe,
          inv_rm2sinthe2, costhe_inv_rm2sinthe, two_over_rm_exp, v_metric, cos4lat, pad;
};
enum {
    ATHAD_MF_P = 0,   // p_dyn (read as a stencil)
    ATHAD_MF_NUE,     // nue
    ATHAD_MF_QT,      // moist-convective and latent heating of t
    ATHAD_MF_KT,      // Held-Suarez rate k_T * L_atm / u_0
    ATHAD_MF_TEQ,     // t_eq
    ATHAD_MF_QC,      // sources of c, cloud, ice, gr (consecutive)
    ATHAD_MF_QCL,
    ATHAD_MF_QI,
    ATHAD_MF_QG,
    ATHAD_MF_MV,      // moist-convective momentum sources of v and w
    ATHAD_MF_MW,
    ATHAD_MF_COUNT
};
struct RK4MArgs {
    Dims d;
    const GeoF* geo;
    const double* t_ref;
    const double* dlnrho;
    double* Y[11];              // FP64 current level: stage-1 stencil input, stage-4 output
    const double* Yn[11];       // FP64 time level n
    const double* p_dyn; const double* nue; const double* t_eq; const double* p_stat; const double* r_humid;
    const double* S_c; const double* S_r; const double* S_i; const double* S_s; const double* S_g; const double* S_v;
    const double* MC_t; const double* MC_q; const double* MC_v; const double* MC_w;
    const float* Yin[11];       // FP32 stage state read (stages 2-4)
    float* Yout[11];            // FP32 stage state written (stages 1-3)
    float* Ybnd[11];            // stage 1: second stage buffer that receives the boundary
    float* Yn32[11];            // FP32 time level n (written by stage 1, read by 2-3)
    float* K[11];               // FP32 accumulator
    float* F[ATHAD_MF_COUNT];   // packed forcing
    double* Yn_store[11];       // store_n: stage 4 also writes the new time level n here
    double* aux_u; double* aux_v; double* aux_w;
    double* prod; double* tke_source; double* dis_source;
    float inv_2dr, inv_2dthe, inv_2dphi, inv_dr, inv_dthe, inv_dphi, inv_dr2, inv_dthe2, inv_dphi2;
    float half_dt_f, dt_f, diffusion_ramp, tke_max_nd, force_nd, coeff_energy_p;
    float inv_re, inv_pr_turb, nue_max, nue_air_nd, diff_prec_re_inv, diff_co2_re_inv, buoy_pref, drag_pref;
    double half_dt, dt_sixth, coeff_energy, coeff_MC_t, coeff_MC_q, coeff_MC_vel, lv, ls, L_atm_over_u0;
    int turb_model, wall_mode, nontrad, curvature, tracer_diff_flux, write_diag;
    int store_n;                // fuse storeIntermediateData3D into stage 4
};
void launch_rk4m_stage(int stage, const RK4MArgs& a, cudaStream_t st);

// Batched mixed-precision step (k_rk4m.cu): per-member step scalars, the device tables the
// persistent stage kernel reads, and the batched level mean.
struct BatchStep {
    float half_dt_f, dt_f, diffusion_ramp, drag_pref;
    double half_dt, dt_sixth;
    double g, dt, u_0;         // buoyancy prefactor ramp * g * dt / u_0, formed per stage
    int iter;                  // the member's current iteration number (1-based)
    int ramp_iters;            // buoyancy ramp = min(1, iter / ramp_iters)
    int write_diag, active;
};
struct BatchTables {
    const RK4MArgs* args;      // [n] per member; stage buffer A in Yout, B in Ybnd
    const BatchStep* step;     // [n]
    const int* tile_start;     // [n+1] first tile of each member (for the launch's shape)
    int n, total_tiles;
};
struct BatchShape { int bx, by, min_blocks; };
int batch_shape_count();
BatchShape batch_shape_info(int shape);
int batch_shape_grid(int shape);   // persistent grid: SMs x resident CTAs of that shape
void launch_rk4m_batch_stage(int stage, int shape, const BatchTables& T, int grid, cudaStream_t st);
struct LevelMeanMember {
    Dims d;
    const double* t; const double* sin_w; double* out;
    int level0;                // first global level index of this member
};
void launch_batch_level_mean(const LevelMeanMember* M, int n, int total_levels, int max_jm,
                             const BatchStep* step, cudaStream_t st);

// Per-(i,j) coefficients of the 7-point Poisson operator, PressureSolverAtm.h:236-269,
// computed on the host once per context.
struct PoiIJ {
    double denom, inv_denom, num1, num2, num3;
    double exp_rm, exp_2_rm, inv_rm, inv_rmsinthe, sinthe, costhe;
};

struct PoissonArgs {
    Dims d;
    const PoiIJ* poi;           // [im*jm]
    const double* dlnrho;       // [im] (anelastic)
    double* aux_u; double* aux_v; double* aux_w;
    double* src;                // clamped divergence source (scratch field)
    double* p;
    unsigned long long* counters;   // [2] clamped sources: [1] accumulated by the source
                                    // launch, [0] the call's total (folded by the ceiling)
    double inv_2dr, inv_2dthe, inv_2dphi;
    int anelastic, metric_div;
    int aux_lid;                // the boundary passes also write the aux radial boundary
    int first_sweep;            // the ceiling starts the call's count instead of adding
    double ceiling;
};
void launch_poisson_prepare(const PoissonArgs& a, cudaStream_t st);   // aux BC + source field
void launch_poisson_sweep(const PoissonArgs& a, cudaStream_t st);     // colours (with their
                                                                      // sources) + BCs + ceiling
void launch_poisson_bcs(const PoissonArgs& a, cudaStream_t st);       // BCs only
void launch_project_correct(const PoissonArgs& a, double* u, double* v, double* w, cudaStream_t st);

// Column physics
struct ColumnArgs {
    Dims d;
    const double* height;      // [im] layer heights (float-rounded, as the reference)
    const double* step_f;      // [im] SaturationAdjustment step (float difference)
    double* t; double* c; double* cloud; double* ice; double* gr; double* co2;
    double* p_stat; double* r_humid; double* r_dry;
    double* S_c_c; double* P_rain; double* P_snow; double* P_graupel; double* Precipitation;
    double* S_v; double* S_c; double* S_i; double* S_r; double* S_s; double* S_g;
    double* t_top_init; double* p_stat_landscape;   // 2-D, pitched rows [jm][pitch]
    double* rho_base; double* dlnrho;               // [im]
    double* row_sum; double* row_cnt;               // scratch [im*jm]
    const double* coslat;                           // [jm] mirror-symmetric weights
    unsigned long long* counters;
    double t_0, t_00, t_max_phys, cloud_cap, M_bg, R_bg, R_mix, r_air, g, t_skin, c_h2o_dry_top;
    double inv_2dr, inv_dr;
    int set_water_profile;
};
void launch_saturation_adjust(const ColumnArgs& a, cudaStream_t st);
void launch_densities(const ColumnArgs& a, cudaStream_t st);

// Moist convection: every 3-D field by athad_field id, 2-D inputs, column tables, constants.
struct MoistArgs {
    Dims d;
    double* F[ATHAD_NFIELDS];
    const double* evaporation;   // 2-D [jm][pitch]
    const double* q_sensible;    // 2-D [jm][pitch]
    const double* height;        // [im] layer heights (float-rounded)
    const double* step;          // [im] height differences, step[im-1] = step[im-2]
    const double* cose;          // [jm] cos(theta_equator - theta_j), mirror-symmetric
    double t_0, cp_l, s_0, lv, ls, g, u_0, r_Earth, p_0, co2_0, c_0, M_bg, R_bg;
    int convection_perturbation, convection_mode, iter_prec;
};
void launch_moist_convection(const MoistArgs& a, cudaStream_t st);

void launch_fill(const Dims& d, double* dst, double v, cudaStream_t st);

// Per-iteration boundary conditions (k_bc.cu)
struct BcArgs {
    Dims d;
    double* F[ATHAD_NFIELDS];
    const double* t_top_init;   // 2-D, pitched rows [jm][pitch]
    const double* vel_star;     // 2-D, pitched rows [jm][pitch]
    double tke_wall_den;        // sqrt(C_nue) * u_0 * u_0
    double dis_wall;            // omega (or epsilon) at the wall, non-dimensional
    int set_dis_wall;
    int wall_bc;                // 0: no wall values (RunTimeSlice's boundary conditions)
    // bcSolidGround's value limits (BC_Atm.h:470-545), non-dimensional
    double tke_max_nd, nue_max, vel_max_nd;
};
void launch_boundary_conditions(const BcArgs& a, cudaStream_t st);

// Smoothing filters (k_filters.cu)
struct FilterArgs {
    Dims d;
    double* field[3];           // u, v, w for the post-RK4 filters
    const int* polar_passes;    // [jm] zonal passes per row
    const double* src[3];       // the zonal passes read these rows instead of field[] (null:
                                // in place)
};
void launch_post_rk4_filters(const FilterArgs& a, cudaStream_t st);
void launch_damp_wiggles(const Dims& d, double* f, double* scratch, cudaStream_t st);
void launch_repitch(const Dims& d, const double* packed, double* dst, cudaStream_t st);

// TurbulenceAtm::run (k_turb.cu).  Per-level constants built on the host as the reference
// forms them: rad.z, 1/(rm+1), metricRadius(rm), get_layer_height(i), and clamp_nue's
// taper factor of the eddy viscosity above abl_height.
struct TurbLevel {
    double rm, exp_rm, rmet, height, nue_fac;
};
struct TurbArgs {
    Dims d;
    const double* u; const double* v; const double* w;
    double* tke; double* dis; double* prod; double* nue; double* tke_source; double* dis_source;
    double* vel_star;           // 2-D, jm rows of pitch
    const double* sin_w;        // sin(theta), mirror-exact
    const TurbLevel* lev;       // [im]
    double inv_2dr, inv_2dthe, inv_2dphi, dr, dthe, dphi;
    double u_0, L_atm, re_turb, nue_max, y_mount;
    int turb_model;
};
void launch_turbulence_run(const TurbArgs& a, cudaStream_t st);

// TwoCatIceScheme::run (k_ice.cu)
struct IceArgs {
    Dims d;
    double* t; double* c; double* cloud; double* ice; double* gr;
    const double* co2; const double* p_stat; const double* r_humid;
    double* P_rain; double* P_snow; double* P_graupel; double* Precipitation;
    double* P_rainn; double* P_snown;
    double* S_v; double* S_c; double* S_i; double* S_r; double* S_s; double* S_g; double* S_c_c;
    const double* step_f;       // [im] float layer thickness, get_layer_height(i+1) - (i)
    double t_0, t_000, M_bg;
    double t_00, ls;            // OneCat's and ThreeCat's temperature bands; ThreeCat's t_crit
    // ThreeCat's constants, formed on the host as ThreeCatIceScheme.h:147-170 does: A_r, A_s,
    // A_g, B_rad^(-8/9), B_s^(-12/13), B_g^(-12/13) and 100 * saturationPressure(t_0)
    double A_r, A_s, A_g, B_rad_neg89, B_s_neg1213, B_g_neg1213, E_sat_t_0_Pa;
    // OneCat's carry of S_au across columns: per column (serial order n = (k-1)*(jm-2) + j-1)
    // the rate at its last cloudy cell, whether it has one, and the value it enters with
    double* sau_exit; double* sau_has; double* sau_entry;
};
void launch_two_cat_ice(const IceArgs& a, cudaStream_t st);
void launch_zero_cat_ice(const IceArgs& a, cudaStream_t st);
void launch_one_cat_ice(const IceArgs& a, cudaStream_t st);
void launch_three_cat_ice(const IceArgs& a, cudaStream_t st);
// IceSchemeCommon::extrapolateBC of n <= 3 flux fields P[q], the seam averaged where avg[q]
void launch_precip_bc(const Dims& d, double* const* P, const int* avg, int n, cudaStream_t st);

// MultiLayerRadiation::run (k_rad.cu)
struct RadArgs {
    Dims d;
    double* t;
    const double* c; const double* co2; const double* p_stat; const double* cloud; const double* ice;
    double* radiation; double* epsilon;
    double* epsilon_2D; double* albedo;   // 2-D, jm rows of pitch
    double* T; double* dn;                // scratch fields: layer temperature [K], downward flux
    const double* step_f;                 // [im] float layer thickness
    double t_0, g, R_bg, sigma, kappa_H2O, kappa_CO2, kappa_bg, geothermal_flux;
    double albedo_surface, albedo_cloud, rad_equator_short, rad_pole_short;
};
void launch_multilayer_radiation(const RadArgs& a, cudaStream_t st);

// the moist iteration's caps and the vapour ceiling (k_caps.cu)
struct CapsArgs {
    Dims d;
    double* c; double* cloud; double* ice; const double* co2; const double* p_stat;
    const double* P_rain; const double* P_snow; const double* P_graupel; const double* P_conv;
    double* Precipitation;
    double* S[7];                 // S_v, S_c, S_i, S_r, S_s, S_g, S_c_c
    double cloud_cap, g;
    double* row_q; double* row_w; // [im*jm] per-row partial sums
    unsigned long long* count;    // cells clamped to the ceiling
    double* sums;                 // [2]: clipped water, air mass
};
void launch_moist_caps(const CapsArgs& a, cudaStream_t st);
// searchMinMax_3D (k_diag.cu); scratch holds 32 B per (i, j) row
void launch_min_max(const Dims& d, const double* x, double* scratch, double* out_v, long long* out_a,
                    cudaStream_t st);
void launch_vapour_ceiling(const CapsArgs& a, cudaStream_t st);

// findResiduumAtm (k_diag.cu).  scratch: 48 B per (i, j) row of the band; out: [6] words =
// residuum, its linear (i, j, k) position, sum, finite count, non-finite count, first
// non-finite key ((j*km + k)*im + i)
struct ResiduumArgs {
    Dims d;
    const double* u; const double* v; const double* w;
    const double* sinthe;         // [jm] max(0.55, sin theta_j), theta the running sum
    const double* rad;            // [im] rad.z
    double dr, dthe, dphi;
    int i0, i1;                   // the band, inclusive
    double* scratch;
    unsigned long long* out;
};
void launch_find_residuum(const ResiduumArgs& a, cudaStream_t st);

// co2Column / waterBudget (k_diag.cu): per (i, j) row sums, then per level
// levels[6 i ..] = sum_j coslat_j x {air mass, water mass, CO2 mass, water fraction, 1 (km
// times)} and the column CO2 path co2_total
struct BudgetArgs {
    Dims d;
    const double* p_stat; const double* c; const double* cloud; const double* ice;
    const double* gr; const double* co2;
    const double* coslat;         // [jm]
    double g;
    double* rows;                 // [4 im jm]
    double* levels;               // [6 im]
    double* co2_total;            // 2-D [jm][pitch], or nullptr
};
void launch_budgets(const BudgetArgs& a, cudaStream_t st);

// standAtm_DewPoint_HumidRel (k_diag.cu)
struct StandAtmArgs {
    Dims d;
    const double* t; const double* c; const double* co2; const double* p_stat;
    const double* height;         // [im] get_layer_height
    const int* i_trop;            // [jm] tropopause level per row
    double* temp_stand; double* temp_dew; double* humid_rel;
    double t_0, M_bg;
};
void launch_stand_atm(const StandAtmArgs& a, cudaStream_t st);
// waterVapourEvaporation and latentSensibleHeat (k_surface.cu)
struct SurfaceArgs {
    Dims d;
    double* c; const double* t; const double* co2; const double* p_stat;
    const double* u; const double* v; const double* w;
    double* evap; double* evap_dalton; double* evap_meyer; double* evap_rohwer; double* c_fix;  // 2-D
    double* q_latent; double* q_sensible;
    const double* sin_w;          // [jm] mirror-exact sin theta
    const double* rad;            // [im] rad.z
    double t_0, u_0, M_bg, coeff_Dalton, cp_l;
    double w_norm, weight[3];     // the vertical spread: w_norm, e^-i w_norm for i = 1..3
    double dr, dthe, dphi;
};
void launch_water_vapour_evaporation(const SurfaceArgs& a, cudaStream_t st);
void launch_latent_sensible_heat(const SurfaceArgs& a, cudaStream_t st);
// planetaryShortWave's per-row albedo sums, summed over k in order (k_rad.cu)
void launch_albedo_rows(const Dims& d, const double* albedo, double* out, cudaStream_t st);
void launch_rad_blend(const Dims& d, const double* t_before, double* t, double omega, cudaStream_t st);

}  // namespace athad
