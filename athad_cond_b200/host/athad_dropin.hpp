// athad_dropin.hpp - C++ host side of the drop-in: the five hot-path call sites of
// cAtmosphereModel::run_3D_loop (atmosphere/cAtmosphereModel.cpp:1158, 1218, 1247, 1418,
// 1509) routed to the device through the C ABI of include/athad_gpu.h.
//
// Header-only and templated on the model type, so it compiles against the reference's
// cAtmosphereModel without this library depending on the reference's headers.  Each
// member mirrors one reference call, with the same name and the same in-place effect on
// the model's Array members:
//
//     SolveRungeKutta(m)        m.solveRungeKutta_Atmosphere_Turb()          :1509
//     PressureSolverRun(m)      PressureSolverAtm(m).run()                   :1158
//     SaturationAdjustmentRun(m) SaturationAdjustment(m).run()               :1218
//     MoistConvectionRun(m, it) MoistConvection(m).run(it)                   :1247
//     Densities(m, water)       ThermoAtm(m).densities(water)                :567, 634, 1418
//     BoundaryConditions(m)     BC_Atm(m).bcRadius(); TurbulenceAtm(m).apply_wall_bc();
//                               BC_Atm(m).bcTheta(); BC_Atm(m).bcPhi();
//                               bcScalarSurfSur(); bcSolidGround()           :1439-1446
//     PostRK4Filters(m)         the polar zonal and radial Shapiro filters   :1507-1520
//     DampMoistWiggles(m)       AtomUtils::damp_wiggles of t, ice, c, cloud  :1225-1228
//     TurbulenceRun(m)          TurbulenceAtm(m).run()                       :614, 1426
//     TwoCatIceSchemeRun(m)     TwoCatIceScheme(m).run()                     :589, 1238
//     MultiLayerRadiationRun(m) MultiLayerRadiation(m).run()                 :831-1007
//     RadiativeHeating(m, w)    radiation mode 2's apply_radiative_heating   :864-879, 1656
//     StandAtmDewPointHumidRel(m) ThermoAtm(m).standAtm_DewPoint_HumidRel()  :636, 1420
//     FindResiduumAtm(m)        UtilsAtm(m).findResiduumAtm()                :668, 1645
//     WaterVapourEvaporation(m) ThermoAtm(m).waterVapourEvaporation()        :637, 1421
//     LatentSensibleHeat(m)     ThermoAtm(m).latentSensibleHeat()            :638, 1422
//     Co2Column(m)              ThermoAtm(m).co2Column(report)               :632, 1416
//     WaterBudget(m)            ThermoAtm(m).waterBudget(report, stage)      :633, 1216, 1417
//
// The model's fields stay resident on the device.  While the reference's other modules
// (boundary conditions, filters, ice scheme, turbulence, radiation) still run on the host,
// every call uploads the fields it reads and downloads the fields it writes; a caller that
// keeps those modules off the loop can use the Device() handle and the C ABI directly.
// Errors surface as std::runtime_error carrying the library's message, which is what the
// reference's own physics code throws (and cli/cond.cpp:27-29 catches).
#pragma once

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/athad_gpu.h"

namespace athad_dropin {

inline void check(athad_ctx* ctx, athad_status s, const char* what)
{
    if (s != ATHAD_OK)
        throw std::runtime_error(std::string("athad: ") + what + ": " +
                                 (ctx ? athad_last_error(ctx) : "no context") + " (status " +
                                 std::to_string((int)s) + ")");
}

// Fills athad_params from the model's own members (AtmosphereParams.h.inc and m_comp).
template <class Model>
athad_params params_from(const Model& m, athad_wall_mode wall = ATHAD_WALL_MIRROR)
{
    athad_params p;
    athad_default_params(&p);
    const std::string& tm = m.turb_model;
    p.turb_model = (tm == "k_epsilon") ? ATHAD_TURB_K_EPSILON
                 : (tm == "k_omega") ? ATHAD_TURB_K_OMEGA : ATHAD_TURB_K_OMEGA_SST;
    p.wall_mode = wall;   // MIRROR: mirror-symmetric SST wall distance; REFERENCE: as the reference
    p.metric_r0 = m.m_metric_r0;            // as initMetricRadius resolved it
    p.re_turb = m.re_turb;
    p.convection_perturbation = m.convection_perturbation;
    p.convection_mode = m.convection_mode;
    p.iter_prec = m.iter_prec;
    p.category_ice_scheme = m.CategoryIceScheme;
    p.r_air = m.r_air; p.g = m.g; p.u_0 = m.u_0; p.cp_l = m.cp_l; p.t_0 = m.t_0; p.c_0 = m.c_0;
    p.L_atm = m.L_atm; p.zeta = m.zeta; p.omega = m.omega; p.lamda = m.lamda; p.lv = m.lv;
    p.ls = m.ls; p.pr_turb = m.pr_turb; p.sc_WaterVapour = m.sc_WaterVapour; p.sc_CO2 = m.sc_CO2;
    p.r_Earth = m.r_Earth; p.p_0 = m.p_0; p.t_00 = m.t_00; p.t_max_phys = m.t_max_phys;
    p.cloud_cap = m.cloud_cap; p.t_skin = m.t_skin; p.c_h2o_dry_top = m.c_h2o_dry_top;
    p.co2_0 = m.co2_0; p.s_0 = m.s_0; p.R_Air = m.R_Air; p.R_WaterVapour = m.R_WaterVapour;
    p.M_bg = m.m_comp.M_bg; p.R_bg = m.m_comp.R_bg; p.R_mix = m.m_comp.R_mix;
    p.abl_height = m.abl_height; p.t_000 = m.t_000;
    p.sigma = m.sigma; p.kappa_H2O = m.kappa_H2O; p.kappa_CO2 = m.kappa_CO2; p.kappa_bg = m.kappa_bg;
    p.geothermal_flux = m.geothermal_flux; p.albedo_surface = m.albedo_surface;
    p.albedo_cloud = m.albedo_cloud; p.rad_equator_short = m.rad_equator_short;
    p.rad_pole_short = m.rad_pole_short;
    p.coeff_Dalton = m.coeff_Dalton;
    p.r_0_water = m.r_0_water;
    return p;
}

template <class Model>
class Device {
public:
    explicit Device(const Model& m, athad_wall_mode wall = ATHAD_WALL_MIRROR)
        : im_(m.im), jm_(m.jm), km_(m.km), buf_((size_t)m.im * m.jm * m.km)
    {
        const athad_grid g{m.im, m.jm, m.km};
        const athad_params p = params_from(m, wall);
        check(nullptr, athad_create(&g, &p, &ctx_), "create");
    }
    ~Device() { if (ctx_) athad_destroy(ctx_); }
    Device(const Device&) = delete;
    Device& operator=(const Device&) = delete;

    athad_ctx* handle() { return ctx_; }

    // Pack a jagged Array (one new[] row of km doubles per (i, j), lib/Array.cpp:62-71).
    template <class Arr>
    void up(athad_field f, const Arr& a)
    {
        size_t q = 0;
        for (int i = 0; i < im_; i++)
            for (int j = 0; j < jm_; j++)
                for (int k = 0; k < km_; k++) buf_[q++] = a.x[i][j][k];
        check(ctx_, athad_upload(ctx_, f, buf_.data(), buf_.size()), "upload");
        check(ctx_, athad_synchronize(ctx_), "upload sync");
    }
    template <class Arr>
    void down(athad_field f, Arr& a)
    {
        check(ctx_, athad_download(ctx_, f, buf_.data(), buf_.size()), "download");
        size_t q = 0;
        for (int i = 0; i < im_; i++)
            for (int j = 0; j < jm_; j++)
                for (int k = 0; k < km_; k++) a.x[i][j][k] = buf_[q++];
    }
    template <class Arr2>
    void up2(athad_field2d f, const Arr2& a)
    {
        std::vector<double> b((size_t)jm_ * km_);
        for (int j = 0; j < jm_; j++)
            for (int k = 0; k < km_; k++) b[(size_t)j * km_ + k] = a.y[j][k];
        check(ctx_, athad_upload_2d(ctx_, f, b.data(), b.size()), "upload_2d");
        check(ctx_, athad_synchronize(ctx_), "upload sync");
    }
    template <class Arr2>
    void down2(athad_field2d f, Arr2& a)
    {
        std::vector<double> b((size_t)jm_ * km_);
        check(ctx_, athad_download_2d(ctx_, f, b.data(), b.size()), "download_2d");
        for (int j = 0; j < jm_; j++)
            for (int k = 0; k < km_; k++) a.y[j][k] = b[(size_t)j * km_ + k];
    }
    void down_profile(athad_profile f, std::vector<double>& v)
    {
        v.resize(im_);
        check(ctx_, athad_download_profile(ctx_, f, v.data(), v.size()), "download_profile");
    }
    void up_profile(athad_profile f, const std::vector<double>& v)
    {
        if ((int)v.size() != im_) return;
        check(ctx_, athad_upload_profile(ctx_, f, v.data(), v.size()), "upload_profile");
    }

    // cAtmosphereModel::solveRungeKutta_Atmosphere_Turb (RungeKutta_Atm_Turb.cpp:44-273)
    void SolveRungeKutta(Model& m)
    {
        up(ATHAD_T, m.t); up(ATHAD_U, m.u); up(ATHAD_V, m.v); up(ATHAD_W, m.w); up(ATHAD_C, m.c);
        up(ATHAD_CLOUD, m.cloud); up(ATHAD_ICE, m.ice); up(ATHAD_GR, m.gr); up(ATHAD_CO2, m.co2);
        up(ATHAD_TKE, m.tke); up(ATHAD_DIS, m.dis);
        up(ATHAD_TN, m.tn); up(ATHAD_UN, m.un); up(ATHAD_VN, m.vn); up(ATHAD_WN, m.wn);
        up(ATHAD_CN, m.cn); up(ATHAD_CLOUDN, m.cloudn); up(ATHAD_ICEN, m.icen); up(ATHAD_GRN, m.grn);
        up(ATHAD_CO2N, m.co2n); up(ATHAD_TKEN, m.tken); up(ATHAD_DISN, m.disn);
        up(ATHAD_P_DYN, m.p_dyn); up(ATHAD_NUE, m.nue); up(ATHAD_T_EQ, m.t_eq);
        up(ATHAD_P_STAT, m.p_stat); up(ATHAD_R_HUMID, m.r_humid);
        up(ATHAD_S_C, m.S_c); up(ATHAD_S_R, m.S_r); up(ATHAD_S_I, m.S_i); up(ATHAD_S_S, m.S_s);
        up(ATHAD_S_G, m.S_g); up(ATHAD_S_V, m.S_v);
        up(ATHAD_MC_T, m.MC_t); up(ATHAD_MC_Q, m.MC_q); up(ATHAD_MC_V, m.MC_v); up(ATHAD_MC_W, m.MC_w);
        up_profile(ATHAD_PROF_DLNRHO_DR, m.m_dlnrho_dr);
        // the right-hand side's outputs are written in the interior: the boundary cells keep
        // the model's values
        up(ATHAD_CORIOLIS_FORCE, m.CoriolisForce); up(ATHAD_BUOYANCY_FORCE, m.BuoyancyForce);
        up(ATHAD_PRESSURE_GRADIENT_FORCE, m.PressureGradientForce);
        up(ATHAD_Q_LATENT, m.Q_Latent); up(ATHAD_Q_SENSIBLE, m.Q_Sensible);
        const bool budget = m.vbudget_capture || m.wbudget_capture;
        athad_step_scalars s{m.dt, m.diffusion_ramp, m.buoyancy_ramp, budget ? 3 : 1, 0};
        check(ctx_, athad_rk4_step(ctx_, &s), "rk4_step");
        down(ATHAD_CORIOLIS_FORCE, m.CoriolisForce); down(ATHAD_BUOYANCY_FORCE, m.BuoyancyForce);
        down(ATHAD_PRESSURE_GRADIENT_FORCE, m.PressureGradientForce);
        down(ATHAD_Q_LATENT, m.Q_Latent); down(ATHAD_Q_SENSIBLE, m.Q_Sensible);
        if (budget) {
            down(ATHAD_VBUD_PGF, m.vbud_pgf); down(ATHAD_VBUD_COR, m.vbud_cor); down(ATHAD_VBUD_ADVV, m.vbud_advv);
            down(ATHAD_VBUD_ADVH, m.vbud_advh); down(ATHAD_VBUD_DIFF, m.vbud_diff); down(ATHAD_VBUD_OTHER, m.vbud_other);
            down(ATHAD_WBUD_PGF, m.wbud_pgf); down(ATHAD_WBUD_COR, m.wbud_cor); down(ATHAD_WBUD_ADVV, m.wbud_advv);
            down(ATHAD_WBUD_ADVH, m.wbud_advh); down(ATHAD_WBUD_DIFF, m.wbud_diff); down(ATHAD_WBUD_OTHER, m.wbud_other);
        }
        down(ATHAD_T, m.t); down(ATHAD_U, m.u); down(ATHAD_V, m.v); down(ATHAD_W, m.w);
        down(ATHAD_C, m.c); down(ATHAD_CLOUD, m.cloud); down(ATHAD_ICE, m.ice); down(ATHAD_GR, m.gr);
        down(ATHAD_CO2, m.co2); down(ATHAD_TKE, m.tke); down(ATHAD_DIS, m.dis);
        down(ATHAD_AUX_U, m.aux_u); down(ATHAD_AUX_V, m.aux_v); down(ATHAD_AUX_W, m.aux_w);
        down(ATHAD_PROD, m.prod); down(ATHAD_TKE_SOURCE, m.tke_source); down(ATHAD_DIS_SOURCE, m.dis_source);
        down_profile(ATHAD_PROF_T_REF_LEVEL, m.t_ref_level);
    }

    // PressureSolverAtm::run (PressureSolverAtm.h:27-669)
    void PressureSolverRun(Model& m, int n_sweeps = 1)
    {
        up(ATHAD_AUX_U, m.aux_u); up(ATHAD_AUX_V, m.aux_v); up(ATHAD_AUX_W, m.aux_w);
        up(ATHAD_P_DYN, m.p_dyn);
        up_profile(ATHAD_PROF_DLNRHO_DR, m.m_dlnrho_dr);
        check(ctx_, athad_pressure_sweep(ctx_, n_sweeps, m.total_iter_count), "pressure_sweep");
        down(ATHAD_P_DYN, m.p_dyn);
        down(ATHAD_AUX_U, m.aux_u); down(ATHAD_AUX_V, m.aux_v); down(ATHAD_AUX_W, m.aux_w);
    }

    // SaturationAdjustment::run (SaturationAdjustment.h:25-45)
    void SaturationAdjustmentRun(Model& m)
    {
        up(ATHAD_T, m.t); up(ATHAD_C, m.c); up(ATHAD_CLOUD, m.cloud); up(ATHAD_ICE, m.ice);
        up(ATHAD_GR, m.gr); up(ATHAD_CO2, m.co2); up(ATHAD_P_STAT, m.p_stat); up(ATHAD_R_HUMID, m.r_humid);
        up(ATHAD_S_C_C, m.S_c_c); up(ATHAD_P_RAIN, m.P_rain); up(ATHAD_P_SNOW, m.P_snow);
        up(ATHAD_P_GRAUPEL, m.P_graupel); up(ATHAD_PRECIPITATION, m.Precipitation);
        up(ATHAD_S_V, m.S_v); up(ATHAD_S_C, m.S_c); up(ATHAD_S_I, m.S_i); up(ATHAD_S_R, m.S_r);
        up(ATHAD_S_S, m.S_s); up(ATHAD_S_G, m.S_g);
        check(ctx_, athad_saturation_adjust(ctx_), "saturation_adjust");
        down(ATHAD_T, m.t); down(ATHAD_C, m.c); down(ATHAD_CLOUD, m.cloud); down(ATHAD_ICE, m.ice);
        down(ATHAD_GR, m.gr); down(ATHAD_S_C_C, m.S_c_c); down(ATHAD_P_RAIN, m.P_rain);
        down(ATHAD_P_SNOW, m.P_snow); down(ATHAD_P_GRAUPEL, m.P_graupel);
        down(ATHAD_PRECIPITATION, m.Precipitation); down(ATHAD_S_V, m.S_v); down(ATHAD_S_C, m.S_c);
        down(ATHAD_S_I, m.S_i); down(ATHAD_S_R, m.S_r); down(ATHAD_S_S, m.S_s); down(ATHAD_S_G, m.S_g);
    }

    // MoistConvection::run (MoistConvection.h:106-140)
    void MoistConvectionRun(Model& m, int iter_n)
    {
        up(ATHAD_T, m.t); up(ATHAD_U, m.u); up(ATHAD_V, m.v); up(ATHAD_W, m.w); up(ATHAD_C, m.c);
        up(ATHAD_CLOUD, m.cloud); up(ATHAD_CO2, m.co2); up(ATHAD_P_STAT, m.p_stat);
        up(ATHAD_R_HUMID, m.r_humid);
        up2(ATHAD_2D_EVAPORATION, m.Evaporation); up2(ATHAD_2D_Q_SENSIBLE, m.Q_sensible_2D);
        // fields the scheme carries from one call to the next (not reset by precompute)
        up(ATHAD_E_U, m.E_u); up(ATHAD_D_U, m.D_u); up(ATHAD_E_D, m.E_d); up(ATHAD_D_D, m.D_d);
        up(ATHAD_U_U, m.u_u); up(ATHAD_V_U, m.v_u); up(ATHAD_W_U, m.w_u);
        up(ATHAD_U_D, m.u_d); up(ATHAD_V_D, m.v_d); up(ATHAD_W_D, m.w_d);
        up(ATHAD_CLOUD_BASE, m.CloudBase); up(ATHAD_LEVEL_FREE_SINKING, m.LevelFreeSinking);
        up(ATHAD_DEEP_BEG, m.Deep_beg); up(ATHAD_DEEP_END, m.Deep_end);
        up(ATHAD_MC_T, m.MC_t); up(ATHAD_MC_Q, m.MC_q); up(ATHAD_MC_V, m.MC_v); up(ATHAD_MC_W, m.MC_w);
        check(ctx_, athad_moist_convection(ctx_, iter_n), "moist_convection");
        down(ATHAD_MC_S, m.s); down(ATHAD_MC_S_U, m.s_u); down(ATHAD_MC_S_D, m.s_d);
        down(ATHAD_M_U, m.M_u); down(ATHAD_M_D, m.M_d); down(ATHAD_Q_V_U, m.q_v_u);
        down(ATHAD_Q_C_U, m.q_c_u); down(ATHAD_Q_V_D, m.q_v_d);
        down(ATHAD_U_U, m.u_u); down(ATHAD_V_U, m.v_u); down(ATHAD_W_U, m.w_u);
        down(ATHAD_U_D, m.u_d); down(ATHAD_V_D, m.v_d); down(ATHAD_W_D, m.w_d);
        down(ATHAD_E_U, m.E_u); down(ATHAD_D_U, m.D_u); down(ATHAD_E_D, m.E_d); down(ATHAD_D_D, m.D_d);
        down(ATHAD_C_U, m.c_u); down(ATHAD_E_L, m.e_l); down(ATHAD_E_DD, m.e_d); down(ATHAD_E_P, m.e_p);
        down(ATHAD_G_P, m.g_p); down(ATHAD_P_CONV, m.P_conv);
        down(ATHAD_CLOUD_BASE, m.CloudBase); down(ATHAD_LEVEL_FREE_SINKING, m.LevelFreeSinking);
        down(ATHAD_DEEP_BEG, m.Deep_beg); down(ATHAD_DEEP_END, m.Deep_end);
        down(ATHAD_MC_T, m.MC_t); down(ATHAD_MC_Q, m.MC_q); down(ATHAD_MC_V, m.MC_v); down(ATHAD_MC_W, m.MC_w);
    }

    // ThermoAtm::densities (ThermoAtm.h:1436-1666)
    void Densities(Model& m, bool set_water_profile = false)
    {
        up(ATHAD_T, m.t); up(ATHAD_C, m.c); up(ATHAD_CO2, m.co2); up(ATHAD_CLOUD, m.cloud);
        up(ATHAD_ICE, m.ice);
        check(ctx_, athad_densities(ctx_, set_water_profile ? 1 : 0), "densities");
        down(ATHAD_T, m.t); down(ATHAD_P_STAT, m.p_stat); down(ATHAD_R_HUMID, m.r_humid);
        down(ATHAD_R_DRY, m.r_dry);
        if (set_water_profile) down(ATHAD_C, m.c);
        std::vector<double> tt((size_t)jm_ * km_), ps((size_t)jm_ * km_);
        check(ctx_, athad_download_2d(ctx_, ATHAD_2D_T_TOP_INIT, tt.data(), tt.size()), "t_top_init");
        check(ctx_, athad_download_2d(ctx_, ATHAD_2D_P_STAT_LANDSCAPE, ps.data(), ps.size()), "p_stat_landscape");
        if ((int)m.t_top_init.size() == jm_)
            for (int j = 0; j < jm_; j++)
                for (int k = 0; k < km_; k++) m.t_top_init[j][k] = tt[(size_t)j * km_ + k];
        for (int j = 0; j < jm_; j++)
            for (int k = 0; k < km_; k++) m.p_stat_landscape.y[j][k] = ps[(size_t)j * km_ + k];
        down_profile(ATHAD_PROF_RHO_BASE, m.m_rho_base);
        down_profile(ATHAD_PROF_DLNRHO_DR, m.m_dlnrho_dr);
    }

    // the per-iteration boundary conditions (cAtmosphereModel.cpp:1439-1446), flat terrain
    void BoundaryConditions(Model& m)
    {
#define ATHAD_BC_FIELDS(X) X(ATHAD_T, t) X(ATHAD_U, u) X(ATHAD_V, v) X(ATHAD_W, w) X(ATHAD_C, c) \
        X(ATHAD_CLOUD, cloud) X(ATHAD_ICE, ice) X(ATHAD_GR, gr) X(ATHAD_CO2, co2) X(ATHAD_TKE, tke) \
        X(ATHAD_DIS, dis) X(ATHAD_NUE, nue) X(ATHAD_PROD, prod) X(ATHAD_TKE_SOURCE, tke_source) \
        X(ATHAD_DIS_SOURCE, dis_source) X(ATHAD_UN, un) X(ATHAD_VN, vn) X(ATHAD_WN, wn) \
        X(ATHAD_TKEN, tken) X(ATHAD_DISN, disn) \
        X(ATHAD_P_STAT, p_stat) X(ATHAD_R_HUMID, r_humid) X(ATHAD_R_DRY, r_dry) X(ATHAD_S_C_C, S_c_c) \
        X(ATHAD_S_V, S_v) X(ATHAD_S_C, S_c) X(ATHAD_S_I, S_i) X(ATHAD_S_R, S_r) X(ATHAD_S_S, S_s) \
        X(ATHAD_S_G, S_g) X(ATHAD_Q_V_U, q_v_u) X(ATHAD_Q_C_U, q_c_u) X(ATHAD_U_U, u_u) \
        X(ATHAD_V_U, v_u) X(ATHAD_W_U, w_u) X(ATHAD_MC_S, s) X(ATHAD_MC_S_U, s_u) X(ATHAD_MC_S_D, s_d) \
        X(ATHAD_M_U, M_u) X(ATHAD_M_D, M_d) X(ATHAD_C_U, c_u) X(ATHAD_E_DD, e_d) X(ATHAD_E_L, e_l) \
        X(ATHAD_E_P, e_p) X(ATHAD_G_P, g_p) X(ATHAD_P_CONV, P_conv) X(ATHAD_Q_LATENT, Q_Latent) \
        X(ATHAD_Q_SENSIBLE, Q_Sensible) X(ATHAD_CORIOLIS_FORCE, CoriolisForce) \
        X(ATHAD_BUOYANCY_FORCE, BuoyancyForce) X(ATHAD_RADIATION, radiation)
#define ATHAD_BC_UP(F, N) up(F, m.N);
#define ATHAD_BC_DOWN(F, N) down(F, m.N);
        ATHAD_BC_FIELDS(ATHAD_BC_UP)
        std::vector<double> tt((size_t)jm_ * km_, 0.0);
        if ((int)m.t_top_init.size() == jm_) {
            for (int j = 0; j < jm_; j++)
                for (int k = 0; k < km_; k++) tt[(size_t)j * km_ + k] = m.t_top_init[j][k];
        } else {   // BC_Atm.h:613-614: without the snapshot the lid is a zero-gradient copy
            for (int j = 0; j < jm_; j++)
                for (int k = 0; k < km_; k++) tt[(size_t)j * km_ + k] = m.t.x[im_ - 2][j][k];
        }
        check(ctx_, athad_upload_2d(ctx_, ATHAD_2D_T_TOP_INIT, tt.data(), tt.size()), "t_top_init");
        up2(ATHAD_2D_VEL_STAR, m.vel_star);
        check(ctx_, athad_boundary_conditions(ctx_), "boundary_conditions");
        ATHAD_BC_FIELDS(ATHAD_BC_DOWN)
#undef ATHAD_BC_UP
#undef ATHAD_BC_DOWN
#undef ATHAD_BC_FIELDS
    }

    // the filters after the RK4 step (cAtmosphereModel.cpp:1507-1520), flat terrain
    void PostRK4Filters(Model& m)
    {
        up(ATHAD_U, m.u); up(ATHAD_V, m.v); up(ATHAD_W, m.w);
        check(ctx_, athad_post_rk4_filters(ctx_), "post_rk4_filters");
        down(ATHAD_U, m.u); down(ATHAD_V, m.v); down(ATHAD_W, m.w);
    }

    // AtomUtils::damp_wiggles of t, ice, c, cloud (cAtmosphereModel.cpp:1225-1228)
    void DampMoistWiggles(Model& m)
    {
        up(ATHAD_T, m.t); up(ATHAD_ICE, m.ice); up(ATHAD_C, m.c); up(ATHAD_CLOUD, m.cloud);
        const athad_field f[4] = {ATHAD_T, ATHAD_ICE, ATHAD_C, ATHAD_CLOUD};
        for (int q = 0; q < 4; q++) check(ctx_, athad_damp_wiggles(ctx_, f[q]), "damp_wiggles");
        down(ATHAD_T, m.t); down(ATHAD_ICE, m.ice); down(ATHAD_C, m.c); down(ATHAD_CLOUD, m.cloud);
    }

    // TwoCatIceScheme(m).run() (cAtmosphereModel.cpp:589, 1238), flat terrain
    void TwoCatIceSchemeRun(Model& m) { IceSchemeCall(m, athad_two_cat_ice_scheme, "two_cat_ice_scheme"); }
    // the whole CategoryIceScheme switch (cAtmosphereModel.cpp:581-596, 1230-1245) on the
    // model's CategoryIceScheme, flat terrain
    void IceSchemeRun(Model& m) { IceSchemeCall(m, athad_ice_scheme, "ice_scheme"); }

private:
    void IceSchemeCall(Model& m, athad_status (*fn)(athad_ctx*), const char* what)
    {
#define ATHAD_ICE_FIELDS(X) X(ATHAD_T, t) X(ATHAD_C, c) X(ATHAD_CLOUD, cloud) X(ATHAD_ICE, ice) \
        X(ATHAD_GR, gr) X(ATHAD_P_RAIN, P_rain) X(ATHAD_P_SNOW, P_snow) X(ATHAD_P_GRAUPEL, P_graupel) \
        X(ATHAD_PRECIPITATION, Precipitation) X(ATHAD_P_RAINN, P_rainn) X(ATHAD_P_SNOWN, P_snown) \
        X(ATHAD_S_V, S_v) X(ATHAD_S_C, S_c) X(ATHAD_S_I, S_i) X(ATHAD_S_R, S_r) X(ATHAD_S_S, S_s) \
        X(ATHAD_S_G, S_g) X(ATHAD_S_C_C, S_c_c)
#define ATHAD_ICE_UP(F, N) up(F, m.N);
#define ATHAD_ICE_DOWN(F, N) down(F, m.N);
        ATHAD_ICE_FIELDS(ATHAD_ICE_UP)
        up(ATHAD_CO2, m.co2); up(ATHAD_P_STAT, m.p_stat); up(ATHAD_R_HUMID, m.r_humid);
        check(ctx_, fn(ctx_), what);
        ATHAD_ICE_FIELDS(ATHAD_ICE_DOWN)
#undef ATHAD_ICE_UP
#undef ATHAD_ICE_DOWN
#undef ATHAD_ICE_FIELDS
    }

public:

    // MultiLayerRadiation(m).run() (cAtmosphereModel.cpp:831-1007), and radiation mode 2's
    // heating t := t (1 - omega) + MLR(t) omega (:864-879; omega_rad = 0.05, :801)
    void MultiLayerRadiationRun(Model& m) { radiation(m, false, 0.0); }
    void RadiativeHeating(Model& m, double omega_rad) { radiation(m, true, omega_rad); }

    // TurbulenceAtm(m).run() (cAtmosphereModel.cpp:614, 1426), flat terrain.  The closure is
    // the one the context was created with (athad_params.turb_model from m.turb_model).
    void TurbulenceRun(Model& m)
    {
        up(ATHAD_U, m.u); up(ATHAD_V, m.v); up(ATHAD_W, m.w);
        up(ATHAD_TKE, m.tke); up(ATHAD_DIS, m.dis); up(ATHAD_NUE, m.nue);
        // the sources are written in the interior only; the rest keeps the model's values
        up(ATHAD_PROD, m.prod); up(ATHAD_TKE_SOURCE, m.tke_source); up(ATHAD_DIS_SOURCE, m.dis_source);
        check(ctx_, athad_turbulence_run(ctx_), "turbulence_run");
        down(ATHAD_TKE, m.tke); down(ATHAD_DIS, m.dis); down(ATHAD_NUE, m.nue);
        down(ATHAD_PROD, m.prod); down(ATHAD_TKE_SOURCE, m.tke_source);
        down(ATHAD_DIS_SOURCE, m.dis_source);
        down2(ATHAD_2D_VEL_STAR, m.vel_star);
    }

    // ThermoAtm(m).forces() (cAtmosphereModel.cpp:635, 1419): its Coriolis and buoyancy
    // arrays (the centrifugal and pressure-gradient ones are output only and stay the
    // host's); the buoyancy reference is the model's level mean once it has one
    void Forces(Model& m)
    {
        up(ATHAD_U, m.u); up(ATHAD_V, m.v); up(ATHAD_W, m.w); up(ATHAD_T, m.t); up(ATHAD_R_HUMID, m.r_humid);
        up(ATHAD_CORIOLIS_FORCE, m.CoriolisForce); up(ATHAD_BUOYANCY_FORCE, m.BuoyancyForce);
        up_profile(ATHAD_PROF_T_REF_LEVEL, m.t_ref_level);
        check(ctx_, athad_forces(ctx_), "forces");
        down(ATHAD_CORIOLIS_FORCE, m.CoriolisForce); down(ATHAD_BUOYANCY_FORCE, m.BuoyancyForce);
    }

    // ThermoAtm(m).standAtm_DewPoint_HumidRel() (cAtmosphereModel.cpp:636, 1420), flat
    // terrain: TempStand, TempDewPoint, HumidityRel from t, c, co2, p_stat and the model's
    // tropopause levels
    void StandAtmDewPointHumidRel(Model& m)
    {
        check(ctx_, athad_set_tropopause_layers(ctx_, m.tropopause_layers.data(),
                                                (int32_t)m.tropopause_layers.size()), "set_tropopause_layers");
        up(ATHAD_T, m.t); up(ATHAD_C, m.c); up(ATHAD_CO2, m.co2); up(ATHAD_P_STAT, m.p_stat);
        check(ctx_, athad_stand_atm_dew_point(ctx_), "stand_atm_dew_point");
        down(ATHAD_TEMP_STAND, m.TempStand); down(ATHAD_TEMP_DEW_POINT, m.TempDewPoint);
        down(ATHAD_HUMIDITY_REL, m.HumidityRel);
    }

    // UtilsAtm(m).findResiduumAtm() (cAtmosphereModel.cpp:668, 1645): the figures the
    // reference prints, returned instead; m.residuum_old is set as the reference sets it
    athad_residuum_report FindResiduumAtm(Model& m)
    {
        up(ATHAD_U, m.u); up(ATHAD_V, m.v); up(ATHAD_W, m.w);
        athad_residuum_report r;
        check(ctx_, athad_find_residuum(ctx_, &r), "find_residuum");
        r.residuum_prev = m.residuum_old;
        m.residuum_old = r.residuum;
        return r;
    }

    // ThermoAtm(m).waterVapourEvaporation() (cAtmosphereModel.cpp:637, 1421), flat terrain
    void WaterVapourEvaporation(Model& m)
    {
        up(ATHAD_T, m.t); up(ATHAD_C, m.c); up(ATHAD_CO2, m.co2); up(ATHAD_P_STAT, m.p_stat);
        up(ATHAD_U, m.u); up(ATHAD_V, m.v); up(ATHAD_W, m.w);
        // a supercritical column leaves c_fix as it was
        up2(ATHAD_2D_C_FIX, m.c_fix);
        check(ctx_, athad_water_vapour_evaporation(ctx_), "water_vapour_evaporation");
        down(ATHAD_C, m.c);
        down2(ATHAD_2D_EVAPORATION, m.Evaporation);
        down2(ATHAD_2D_EVAPORATION_DALTON, m.Evaporation_Dalton);
        down2(ATHAD_2D_EVAPORATION_MEYER, m.Evaporation_Meyer);
        down2(ATHAD_2D_EVAPORATION_ROHWER, m.Evaporation_Rohwer);
        down2(ATHAD_2D_C_FIX, m.c_fix);
    }

    // ThermoAtm(m).latentSensibleHeat() (cAtmosphereModel.cpp:638, 1422), flat terrain
    void LatentSensibleHeat(Model& m)
    {
        up(ATHAD_T, m.t);
        up(ATHAD_Q_LATENT, m.Q_Latent); up(ATHAD_Q_SENSIBLE, m.Q_Sensible);   // the boundary cells keep theirs
        check(ctx_, athad_latent_sensible_heat(ctx_), "latent_sensible_heat");
        down(ATHAD_Q_LATENT, m.Q_Latent); down(ATHAD_Q_SENSIBLE, m.Q_Sensible);
    }

    // ThermoAtm(m).co2Column(report) (cAtmosphereModel.cpp:632, 1416): m.co2_total and the
    // CO2 budget, returned for the caller to print; m.m_q_co2_ref set on the first call as
    // the reference sets it
    athad_budget_report Co2Column(Model& m)
    {
        up(ATHAD_P_STAT, m.p_stat); up(ATHAD_CO2, m.co2);
        athad_budget_report r;
        check(ctx_, athad_co2_column(ctx_, &r), "co2_column");
        down2(ATHAD_2D_CO2_TOTAL, m.co2_total);
        if (m.m_q_co2_ref <= 0.0) m.m_q_co2_ref = r.q_mean;
        return r;
    }

    // ThermoAtm(m).waterBudget(report, stage) (cAtmosphereModel.cpp:633, 1216, 1417): the
    // water budget, returned for the caller to print; the model's first-call references
    // (m_q_h2o_ref, m_air_levels, m_q_h2o_fixed_ref, m_q_h2o_levels) set as the reference
    // sets them.  The context keeps its own references from its first call.
    athad_budget_report WaterBudget(Model& m, std::vector<double>* level_drift = nullptr)
    {
        up(ATHAD_P_STAT, m.p_stat); up(ATHAD_C, m.c); up(ATHAD_CLOUD, m.cloud);
        up(ATHAD_ICE, m.ice); up(ATHAD_GR, m.gr);
        athad_budget_report r;
        std::vector<double> lev(im_);
        check(ctx_, athad_water_budget(ctx_, &r, lev.data()), "water_budget");
        if (m.m_q_h2o_ref <= 0.0) m.m_q_h2o_ref = r.q_ref;
        if (m.m_q_h2o_fixed_ref <= 0.0) m.m_q_h2o_fixed_ref = r.q_fixed_ref;
        if (level_drift) *level_drift = lev;
        return r;
    }

private:
    void radiation(Model& m, bool heating, double omega_rad)
    {
        up(ATHAD_T, m.t); up(ATHAD_C, m.c); up(ATHAD_CO2, m.co2); up(ATHAD_P_STAT, m.p_stat);
        up(ATHAD_CLOUD, m.cloud); up(ATHAD_ICE, m.ice);
        if (heating) check(ctx_, athad_radiative_heating(ctx_, omega_rad), "radiative_heating");
        else check(ctx_, athad_multilayer_radiation(ctx_), "multilayer_radiation");
        down(ATHAD_T, m.t); down(ATHAD_RADIATION, m.radiation); down(ATHAD_EPSILON, m.epsilon);
        down2(ATHAD_2D_EPSILON, m.epsilon_2D); down2(ATHAD_2D_ALBEDO, m.albedo);
    }

    int im_, jm_, km_;
    std::vector<double> buf_;
    athad_ctx* ctx_ = nullptr;
};

// Every 3-D field a context holds and the model member it mirrors (athad_field order).
#define ATHAD_ALL_FIELDS(X) \
    X(ATHAD_T, t) X(ATHAD_U, u) X(ATHAD_V, v) X(ATHAD_W, w) X(ATHAD_C, c) X(ATHAD_CLOUD, cloud) \
    X(ATHAD_ICE, ice) X(ATHAD_GR, gr) X(ATHAD_CO2, co2) X(ATHAD_TKE, tke) X(ATHAD_DIS, dis) \
    X(ATHAD_TN, tn) X(ATHAD_UN, un) X(ATHAD_VN, vn) X(ATHAD_WN, wn) X(ATHAD_CN, cn) \
    X(ATHAD_CLOUDN, cloudn) X(ATHAD_ICEN, icen) X(ATHAD_GRN, grn) X(ATHAD_CO2N, co2n) \
    X(ATHAD_TKEN, tken) X(ATHAD_DISN, disn) X(ATHAD_P_DYN, p_dyn) X(ATHAD_NUE, nue) \
    X(ATHAD_T_EQ, t_eq) X(ATHAD_P_STAT, p_stat) X(ATHAD_R_HUMID, r_humid) X(ATHAD_S_C, S_c) \
    X(ATHAD_S_R, S_r) X(ATHAD_S_I, S_i) X(ATHAD_S_S, S_s) X(ATHAD_S_G, S_g) X(ATHAD_S_V, S_v) \
    X(ATHAD_MC_T, MC_t) X(ATHAD_MC_Q, MC_q) X(ATHAD_MC_V, MC_v) X(ATHAD_MC_W, MC_w) \
    X(ATHAD_AUX_U, aux_u) X(ATHAD_AUX_V, aux_v) X(ATHAD_AUX_W, aux_w) X(ATHAD_PROD, prod) \
    X(ATHAD_TKE_SOURCE, tke_source) X(ATHAD_DIS_SOURCE, dis_source) X(ATHAD_S_C_C, S_c_c) \
    X(ATHAD_P_RAIN, P_rain) X(ATHAD_P_SNOW, P_snow) X(ATHAD_P_GRAUPEL, P_graupel) \
    X(ATHAD_PRECIPITATION, Precipitation) X(ATHAD_R_DRY, r_dry) X(ATHAD_MC_S, s) \
    X(ATHAD_MC_S_U, s_u) X(ATHAD_MC_S_D, s_d) X(ATHAD_M_U, M_u) X(ATHAD_M_D, M_d) \
    X(ATHAD_Q_V_U, q_v_u) X(ATHAD_Q_C_U, q_c_u) X(ATHAD_Q_V_D, q_v_d) X(ATHAD_U_U, u_u) \
    X(ATHAD_V_U, v_u) X(ATHAD_W_U, w_u) X(ATHAD_U_D, u_d) X(ATHAD_V_D, v_d) X(ATHAD_W_D, w_d) \
    X(ATHAD_E_U, E_u) X(ATHAD_D_U, D_u) X(ATHAD_E_D, E_d) X(ATHAD_D_D, D_d) X(ATHAD_C_U, c_u) \
    X(ATHAD_E_L, e_l) X(ATHAD_E_DD, e_d) X(ATHAD_E_P, e_p) X(ATHAD_G_P, g_p) X(ATHAD_P_CONV, P_conv) \
    X(ATHAD_CLOUD_BASE, CloudBase) X(ATHAD_LEVEL_FREE_SINKING, LevelFreeSinking) \
    X(ATHAD_DEEP_BEG, Deep_beg) X(ATHAD_DEEP_END, Deep_end) X(ATHAD_P_RAINN, P_rainn) \
    X(ATHAD_P_SNOWN, P_snown) X(ATHAD_RADIATION, radiation) X(ATHAD_EPSILON, epsilon) \
    X(ATHAD_TEMP_STAND, TempStand) X(ATHAD_TEMP_DEW_POINT, TempDewPoint) \
    X(ATHAD_HUMIDITY_REL, HumidityRel) X(ATHAD_Q_LATENT, Q_Latent) X(ATHAD_Q_SENSIBLE, Q_Sensible) \
    X(ATHAD_CORIOLIS_FORCE, CoriolisForce) X(ATHAD_BUOYANCY_FORCE, BuoyancyForce) \
    X(ATHAD_PRESSURE_GRADIENT_FORCE, PressureGradientForce) \
    X(ATHAD_VBUD_PGF, vbud_pgf) X(ATHAD_VBUD_COR, vbud_cor) X(ATHAD_VBUD_ADVV, vbud_advv) \
    X(ATHAD_VBUD_ADVH, vbud_advh) X(ATHAD_VBUD_DIFF, vbud_diff) X(ATHAD_VBUD_OTHER, vbud_other) \
    X(ATHAD_WBUD_PGF, wbud_pgf) X(ATHAD_WBUD_COR, wbud_cor) X(ATHAD_WBUD_ADVV, wbud_advv) \
    X(ATHAD_WBUD_ADVH, wbud_advh) X(ATHAD_WBUD_DIFF, wbud_diff) X(ATHAD_WBUD_OTHER, wbud_other)
#define ATHAD_ALL_FIELDS2D(X) \
    X(ATHAD_2D_P_STAT_LANDSCAPE, p_stat_landscape) X(ATHAD_2D_EVAPORATION, Evaporation) \
    X(ATHAD_2D_Q_SENSIBLE, Q_sensible_2D) X(ATHAD_2D_VEL_STAR, vel_star) X(ATHAD_2D_EPSILON, epsilon_2D) \
    X(ATHAD_2D_ALBEDO, albedo) X(ATHAD_2D_EVAPORATION_DALTON, Evaporation_Dalton) \
    X(ATHAD_2D_EVAPORATION_MEYER, Evaporation_Meyer) X(ATHAD_2D_EVAPORATION_ROHWER, Evaporation_Rohwer) \
    X(ATHAD_2D_C_FIX, c_fix) X(ATHAD_2D_CO2_TOTAL, co2_total)

// What one iteration of the resident loop reads back: the figures the reference prints.
struct IterationReport {
    athad_residuum_report residuum;
    bool moist = false;                  // the moist block ran (iter_n % 2 == 0)
    athad_budget_report h2o_post_rk4{}, co2{}, h2o{};
    double t_skin = 0.0;
};

// The device-resident drop-in of cAtmosphereModel::run_3D_loop's body
// (cAtmosphereModel.cpp:1156-1661): the model's state is uploaded once (Attach), every module
// of an iteration then runs on the device in the reference's order and cadence with nothing
// crossing PCIe but the few figures the reference prints, and Sync downloads the state into
// the model on the iterations whose output the reference writes (its `checkpoint`, the restart
// dumps).  The patched loop keeps the reference's own loop header (iteration counters, the
// diffusion and buoyancy ramps, dt) and its output code:
//
//     athad_dropin::Device<cAtmosphereModel> dev(*this);
//     athad_dropin::ResidentLoop<cAtmosphereModel> loop(dev, *this);
//     for (iter_n = iter_start; iter_n <= nm; iter_n++) {
//         total_iter_count++; ... diffusion_ramp, dt, buoyancy_ramp as the reference ...
//         auto report = loop.Iteration(*this);
//         if (iter_n % checkpoint == 0) loop.Sync(*this);   // before the file output
//         ... the reference's printing and output ...
//     }
//
// Configuration of cli/config_cond.xml: flat terrain, radiation mode 2 (omega_rad 0.05), no
// inviscid spin-up (moist block every 2nd iteration).  The zonal-mean momentum-budget
// differencing of checkpoint iterations (:1471-1520) is the caller's, from synced fields;
// the right-hand side's budget terms are captured on those iterations.
template <class Model>
class ResidentLoop {
public:
    ResidentLoop(Device<Model>& dev, Model& m, double omega_rad = 0.05) : dev_(dev), omega_rad_(omega_rad)
    {
        Attach(m);
    }

    // Uploads the model's whole state: every field the context holds, the 2-D fields, the
    // lid snapshot, the profiles and the tropopause levels.
    void Attach(Model& m)
    {
#define ATHAD_UP3(F, N) dev_.up(F, m.N);
#define ATHAD_UP2(F, N) dev_.up2(F, m.N);
        ATHAD_ALL_FIELDS(ATHAD_UP3)
        ATHAD_ALL_FIELDS2D(ATHAD_UP2)
#undef ATHAD_UP3
#undef ATHAD_UP2
        athad_ctx* ctx = dev_.handle();
        const int jm = m.jm, km = m.km;
        std::vector<double> tt((size_t)jm * km, 0.0);
        if ((int)m.t_top_init.size() == jm)
            for (int j = 0; j < jm; j++)
                for (int k = 0; k < km; k++) tt[(size_t)j * km + k] = m.t_top_init[j][k];
        check(ctx, athad_upload_2d(ctx, ATHAD_2D_T_TOP_INIT, tt.data(), tt.size()), "t_top_init");
        dev_.up_profile(ATHAD_PROF_T_REF_LEVEL, m.t_ref_level);
        dev_.up_profile(ATHAD_PROF_RHO_BASE, m.m_rho_base);
        dev_.up_profile(ATHAD_PROF_DLNRHO_DR, m.m_dlnrho_dr);
        check(ctx, athad_set_tropopause_layers(ctx, m.tropopause_layers.data(),
                                               (int32_t)m.tropopause_layers.size()), "set_tropopause_layers");
        check(ctx, athad_synchronize(ctx), "attach");
    }

    // One iteration for m.iter_n with the model's m.dt, m.diffusion_ramp, m.buoyancy_ramp and
    // m.total_iter_count; sets m.residuum_old and m.t_skin as the reference does.
    IterationReport Iteration(Model& m)
    {
        athad_ctx* ctx = dev_.handle();
        IterationReport r;
        const int it = m.iter_n;
        if (it % 4 == 0)                                                  // :1156-1159
            check(ctx, athad_pressure_sweep(ctx, 1, m.total_iter_count), "pressure_sweep");
        if (it % 2 == 0) {                                                // :1182-1434
            r.moist = true;
            check(ctx, athad_water_budget(ctx, &r.h2o_post_rk4, nullptr), "water_budget");
            check(ctx, athad_saturation_adjust(ctx), "saturation_adjust");
            for (athad_field f : {ATHAD_T, ATHAD_ICE, ATHAD_C, ATHAD_CLOUD}) damp(ctx, f);
            check(ctx, athad_ice_scheme(ctx), "ice_scheme");
            for (athad_field f : {ATHAD_P_RAIN, ATHAD_P_SNOW}) damp(ctx, f);
            check(ctx, athad_moist_convection(ctx, it), "moist_convection");
            for (athad_field f : {ATHAD_P_CONV, ATHAD_E_U, ATHAD_M_U, ATHAD_Q_V_U, ATHAD_Q_C_U, ATHAD_E_D,
                                  ATHAD_M_D, ATHAD_Q_V_D, ATHAD_MC_T, ATHAD_MC_V, ATHAD_MC_W})
                damp(ctx, f);
            check(ctx, athad_moist_caps(ctx), "moist_caps");
            check(ctx, athad_vapour_ceiling(ctx, nullptr), "vapour_ceiling");
            check(ctx, athad_co2_column(ctx, &r.co2), "co2_column");
            check(ctx, athad_water_budget(ctx, &r.h2o, nullptr), "water_budget");
            check(ctx, athad_densities(ctx, 0), "densities");
            check(ctx, athad_forces(ctx), "forces");
            check(ctx, athad_stand_atm_dew_point(ctx), "stand_atm_dew_point");
            check(ctx, athad_water_vapour_evaporation(ctx), "water_vapour_evaporation");
            check(ctx, athad_latent_sensible_heat(ctx), "latent_sensible_heat");
            check(ctx, athad_turbulence_run(ctx), "turbulence_run");
            for (athad_field f : {ATHAD_TKE, ATHAD_DIS, ATHAD_NUE, ATHAD_PROD, ATHAD_TKE_SOURCE, ATHAD_DIS_SOURCE})
                damp(ctx, f);
        }
        check(ctx, athad_boundary_conditions(ctx), "boundary_conditions");   // :1439-1446
        const int budget = (m.checkpoint > 0 && it % m.checkpoint == 0) ? 2 : 0;   // :1471, 1502
        athad_step_scalars s{m.dt, m.diffusion_ramp, m.buoyancy_ramp, 1 | budget, 0};
        check(ctx, athad_rk4_step(ctx, &s), "rk4_step");                  // :1509
        check(ctx, athad_post_rk4_filters(ctx), "post_rk4_filters");      // :1524-1575
        check(ctx, athad_find_residuum(ctx, &r.residuum), "find_residuum");   // :1645
        r.residuum.residuum_prev = m.residuum_old;
        m.residuum_old = r.residuum.residuum;
        check(ctx, athad_store_n_level(ctx), "store_n_level");           // :1647
        check(ctx, athad_radiative_heating(ctx, omega_rad_), "radiative_heating");   // :1656
        check(ctx, athad_update_skin_temperature(ctx, m.t_skin_relax, &r.t_skin), "skin");   // :1661
        m.t_skin = r.t_skin;
        return r;
    }

    // Downloads the whole device state into the model (for the reference's output code).
    void Sync(Model& m)
    {
#define ATHAD_DOWN3(F, N) dev_.down(F, m.N);
#define ATHAD_DOWN2(F, N) dev_.down2(F, m.N);
        ATHAD_ALL_FIELDS(ATHAD_DOWN3)
        ATHAD_ALL_FIELDS2D(ATHAD_DOWN2)
#undef ATHAD_DOWN3
#undef ATHAD_DOWN2
        dev_.down_profile(ATHAD_PROF_T_REF_LEVEL, m.t_ref_level);
        dev_.down_profile(ATHAD_PROF_RHO_BASE, m.m_rho_base);
        dev_.down_profile(ATHAD_PROF_DLNRHO_DR, m.m_dlnrho_dr);
    }

private:
    static void damp(athad_ctx* ctx, athad_field f) { check(ctx, athad_damp_wiggles(ctx, f), "damp_wiggles"); }
    Device<Model>& dev_;
    double omega_rad_;
};

}  // namespace athad_dropin
