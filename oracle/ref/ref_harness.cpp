// ref_harness.cpp - a C entry layer around the unmodified reference, so the tests can run
// the reference's own hot-path functions on a state they choose and read the results.
// TEST INFRASTRUCTURE ONLY (the oracle's pin); built into oracle/_ref/ by
// oracle/ref/Makefile from the reference sources where they lie.
//
// The reference keeps its model state in private members of cAtmosphereModel and runs its
// physics through friend classes.  To reach them without editing the reference, the
// standard headers are included first and the access specifiers are then widened for the
// reference headers only.  Object layout does not depend on access, so this TU and the
// reference's own objects agree on every member's address.
#include <algorithm>
#include <cassert>
#include <chrono>
#include <climits>
#include <cmath>
#include <csignal>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fenv.h>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <sys/types.h>
#include <tuple>
#include <vector>
#include <omp.h>
#include "tinyxml2.h"

#define private public
#define protected public
#include "cAtmosphereModel.h"
// MoistConvection.h defines two non-inline globals that cAtmosphereModel.cpp defines too;
// give this TU's copies their own names (same initialisers).
#define eps_u harness_eps_u
#define del_u harness_del_u
#include "MoistConvection.h"
#undef eps_u
#undef del_u
#include "ZeroCatIceScheme.h"
#include "OneCatIceScheme.h"
#include "TwoCatIceScheme.h"
#include "ThreeCatIceScheme.h"
#include "SaturationAdjustment.h"
#include "VelocityInitializer.h"
#include "PressureSolverAtm.h"
#include "ThermoAtm.h"
#include "UtilsAtm.h"
#include "BC_Atm.h"
#include "TurbulenceAtm.h"
#include "MultiLayerRadiation.h"
#undef private
#undef protected

namespace {

struct NullBuf : std::streambuf {
    int overflow(int c) override { return c; }
};
NullBuf g_null;
std::streambuf* g_saved = nullptr;
std::streambuf* g_null_buf() { return &g_null; }

Array* field3(cAtmosphereModel* m, const std::string& n)
{
#define F(name) if (n == #name) return &m->name;
    F(t) F(u) F(v) F(w) F(c) F(cloud) F(ice) F(gr) F(co2) F(tke) F(dis)
    F(tn) F(un) F(vn) F(wn) F(cn) F(cloudn) F(icen) F(grn) F(co2n) F(tken) F(disn)
    F(p_dyn) F(nue) F(t_eq) F(p_stat) F(r_humid)
    F(S_c) F(S_r) F(S_i) F(S_s) F(S_g) F(S_v)
    F(MC_t) F(MC_q) F(MC_v) F(MC_w)
    F(aux_u) F(aux_v) F(aux_w)
    F(prod) F(tke_source) F(dis_source)
    F(S_c_c) F(P_rain) F(P_snow) F(P_graupel) F(Precipitation)
    F(r_dry)
    F(s) F(s_u) F(s_d) F(M_u) F(M_d) F(q_v_u) F(q_c_u) F(q_v_d)
    F(u_u) F(v_u) F(w_u) F(u_d) F(v_d) F(w_d)
    F(E_u) F(D_u) F(E_d) F(D_d)
    F(c_u) F(e_l) F(e_d) F(e_p) F(g_p)
    F(P_conv) F(CloudBase) F(LevelFreeSinking) F(Deep_beg) F(Deep_end)
    F(P_rainn) F(P_snown) F(radiation) F(epsilon)
    F(TempStand) F(TempDewPoint) F(HumidityRel) F(Q_Latent) F(Q_Sensible)
    F(rhs_t) F(rhs_u) F(rhs_v) F(rhs_w) F(rhs_c) F(rhs_cloud) F(rhs_ice) F(rhs_g) F(rhs_co2)
    F(rhs_tke) F(rhs_dis) F(h) F(p_hydro)
    F(CoriolisForce) F(BuoyancyForce) F(PressureGradientForce)
    F(vbud_pgf) F(vbud_cor) F(vbud_advv) F(vbud_advh) F(vbud_diff) F(vbud_other)
    F(wbud_pgf) F(wbud_cor) F(wbud_advv) F(wbud_advh) F(wbud_diff) F(wbud_other)
#undef F
    return nullptr;
}

Array_2D* field2(cAtmosphereModel* m, const std::string& n)
{
    if (n == "p_stat_landscape") return &m->p_stat_landscape;
    if (n == "Evaporation") return &m->Evaporation;
    if (n == "Q_sensible_2D") return &m->Q_sensible_2D;
    if (n == "vel_star") return &m->vel_star;
    if (n == "epsilon_2D") return &m->epsilon_2D;
    if (n == "albedo") return &m->albedo;
    if (n == "Evaporation_Dalton") return &m->Evaporation_Dalton;
    if (n == "Evaporation_Meyer") return &m->Evaporation_Meyer;
    if (n == "Evaporation_Rohwer") return &m->Evaporation_Rohwer;
    if (n == "c_fix") return &m->c_fix;
    if (n == "co2_total") return &m->co2_total;
    return nullptr;
}

std::vector<double>* profile(cAtmosphereModel* m, const std::string& n)
{
    if (n == "t_ref_level") return &m->t_ref_level;
    if (n == "rho_base") return &m->m_rho_base;
    if (n == "dlnrho_dr") return &m->m_dlnrho_dr;
    return nullptr;
}

}  // namespace

extern "C" {

void ref_dims(int* im, int* jm, int* km)
{
    *im = cAtmosphereModel::im; *jm = cAtmosphereModel::jm; *km = cAtmosphereModel::km;
}

void ref_set_threads(int n) { omp_set_num_threads(n); }

void ref_quiet(int q)
{
    if (q && !g_saved) g_saved = std::cout.rdbuf(&g_null);
    if (!q && g_saved) { std::cout.rdbuf(g_saved); g_saved = nullptr; }
}

// xml == NULL: the compiled-in defaults (SetDefaultConfig, cAtmosphereDefaults.cpp.inc),
// which are the values of cli/config_cond.xml, then the composition LoadConfig would resolve.
void* ref_new(const char* xml)
{
    cAtmosphereModel* m = new cAtmosphereModel();
    if (xml) m->LoadConfig(xml);
    else m->initComposition();
    return m;
}

void ref_delete(void* p) { delete (cAtmosphereModel*)p; }

// The reference's initial state: RunTimeSlice (cAtmosphereModel.cpp:468-668) for Ma = 0
// without its file output, the printed diagnostics and the standard-atmosphere dew-point
// diagnostic (standAtm_DewPoint_HumidRel, a 60-step bisection per cell that no hot-path
// function reads), then the Held-Suarez target snapshot of run_3D_loop (:750-753).
// ref_init_state_upto stops after stage `upto` (1 velocities, 2 temperature, 3 water and
// the co2/densities fixed point, 4 cloud and ice, 5 saturation adjustment, 6 ice scheme,
// 7 moist convection, 8 turbulence, 9 the diagnosis block from precipitationSum to
// vegetationLand, 10 boundary conditions, 11 projection, 12 everything).
int ref_init_state_upto(void* p, int upto)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    m->m_current_time = m->m_time_list.insert(0).first;
    UtilsAtm(*m).resetArrays();
    m->dt = m->dt_visc;
    m->iter_n = 0;
    m->total_iter_count = 0;
    if (m->turb_model.empty() || m->turb_model == "none") m->turb_model = "laminar";
    m->use_turbulence_model = (m->turb_model != "laminar");
    m->use_k_epsilon_turbulence_model = (m->turb_model == "k_epsilon");
    m->use_k_omega_turbulence_model = (m->turb_model == "k_omega");
    m->use_k_omega_SST_turbulence_model = (m->turb_model == "k_omega_SST");
    m->initGridCoordinates();
    m->initMetricRadius();
    m->init_layer_heights();
    m->init_tropopause_layers();
    m->read_Atmosphere_Surface_Data(0);
    m->LandOceanFraction();
    if (!m->use_NASA_velocity) VelocityInitializer(*m).compute();
    BC_Atm(*m).bcVelSurfSur();
    AtomUtils::damp_wiggles(m->u, &m->i_topography, true, true, true);
    AtomUtils::damp_wiggles(m->v, &m->i_topography, true, true, true);
    AtomUtils::damp_wiggles(m->w, &m->i_topography, true, true, true);
    if (upto <= 1) return 0;
    m->initTemperatureData(0);
    AtomUtils::damp_wiggles(m->t, &m->i_topography, true, true, true);
    m->t_top_init.assign(m->jm, std::vector<double>(m->km, 0.0));
    for (int j = 0; j < m->jm; j++)
        for (int k = 0; k < m->km; k++) m->t_top_init[j][k] = m->t.x[m->im - 1][j][k];
    if (upto <= 2) return 0;
    m->initWaterWapour();
    for (int pass = 0; pass < 2; pass++) {
        ThermoAtm(*m).co2Atmosphere();
        ThermoAtm(*m).densities(true);
    }
    if (upto <= 3) return 0;
    m->initCloudIce();
    if (upto <= 4) return 0;
    SaturationAdjustment(*m).run();
    AtomUtils::damp_wiggles(m->ice, &m->i_topography, true, true, true);
    AtomUtils::damp_wiggles(m->c, &m->i_topography, true, true, true);
    AtomUtils::damp_wiggles(m->cloud, &m->i_topography, true, true, true);
    ThermoAtm(*m).precipitableWater();
    if (upto <= 5) return 0;
    switch (m->CategoryIceScheme) {
        case 0: ZeroCatIceScheme(*m).run(); break;
        case 1: OneCatIceScheme(*m).run(); break;
        case 2: TwoCatIceScheme(*m).run(); break;
        case 3: ThreeCatIceScheme(*m).run(); break;
        default: break;
    }
    AtomUtils::damp_wiggles(m->P_rain, &m->i_topography, true, true, true);
    AtomUtils::damp_wiggles(m->P_snow, &m->i_topography, true, true, true);
    if (upto <= 6) return 0;
    MoistConvection(*m).run(m->iter_n);
    for (Array* a : {&m->P_conv, &m->E_u, &m->M_u, &m->q_v_u, &m->q_c_u, &m->E_d, &m->M_d, &m->q_v_d})
        AtomUtils::damp_wiggles(*a, &m->i_topography, true, true, true);
    if (upto <= 7) return 0;
    if (m->turb_model != "laminar") {
        TurbulenceAtm(*m).init();
        TurbulenceAtm(*m).run();
        for (Array* a : {&m->tke, &m->dis, &m->nue, &m->prod, &m->tke_source, &m->dis_source})
            AtomUtils::damp_wiggles(*a, &m->i_topography, true, true, true);
    }
    if (upto <= 8) return 0;
    UtilsAtm(*m).precipitationSum();
    ThermoAtm(*m).co2Atmosphere();
    ThermoAtm(*m).co2Column(true);
    ThermoAtm(*m).waterBudget(true);
    ThermoAtm(*m).densities();
    ThermoAtm(*m).forces();
    ThermoAtm(*m).waterVapourEvaporation();
    ThermoAtm(*m).latentSensibleHeat();
    ThermoAtm(*m).vegetationLand();
    if (upto <= 9) return 0;
    BC_Atm(*m).bcRadius();
    BC_Atm(*m).bcTheta();
    BC_Atm(*m).bcPhi();
    BC_Atm(*m).bcScalarSurfSur();
    BC_Atm(*m).bcSolidGround();
    if (upto <= 10) return 0;
    PressureSolverAtm(*m).project_initial_velocity(200);
    if (upto <= 11) return 0;
    UtilsAtm(*m).storeIntermediateData3D(1.0);
    for (int i = 0; i < m->im; i++)
        for (int j = 0; j < m->jm; j++)
            for (int k = 0; k < m->km; k++) m->t_eq.x[i][j][k] = m->t.x[i][j][k];
    return 0;
}

int ref_init_state(void* p) { return ref_init_state_upto(p, 99); }

int ref_get3(void* p, const char* name, double* out)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    Array* a = field3(m, name);
    if (!a || !a->x) return -1;
    size_t q = 0;
    for (int i = 0; i < m->im; i++)
        for (int j = 0; j < m->jm; j++) {
            std::memcpy(out + q, a->x[i][j], sizeof(double) * m->km);
            q += m->km;
        }
    return 0;
}

int ref_set3(void* p, const char* name, const double* in)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    Array* a = field3(m, name);
    if (!a || !a->x) return -1;
    size_t q = 0;
    for (int i = 0; i < m->im; i++)
        for (int j = 0; j < m->jm; j++) {
            std::memcpy(a->x[i][j], in + q, sizeof(double) * m->km);
            q += m->km;
        }
    return 0;
}

int ref_get2(void* p, const char* name, double* out)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    if (std::string(name) == "t_top_init") {
        if ((int)m->t_top_init.size() != m->jm) return -1;
        for (int j = 0; j < m->jm; j++)
            for (int k = 0; k < m->km; k++) out[(size_t)j * m->km + k] = m->t_top_init[j][k];
        return 0;
    }
    Array_2D* a = field2(m, name);
    if (!a || !a->y) return -1;
    for (int j = 0; j < m->jm; j++)
        for (int k = 0; k < m->km; k++) out[(size_t)j * m->km + k] = a->y[j][k];
    return 0;
}

int ref_set2(void* p, const char* name, const double* in)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    if (std::string(name) == "t_top_init") {
        m->t_top_init.assign(m->jm, std::vector<double>(m->km, 0.0));
        for (int j = 0; j < m->jm; j++)
            for (int k = 0; k < m->km; k++) m->t_top_init[j][k] = in[(size_t)j * m->km + k];
        return 0;
    }
    Array_2D* a = field2(m, name);
    if (!a || !a->y) return -1;
    for (int j = 0; j < m->jm; j++)
        for (int k = 0; k < m->km; k++) a->y[j][k] = in[(size_t)j * m->km + k];
    return 0;
}

int ref_getp(void* p, const char* name, double* out)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    std::vector<double>* v = profile(m, name);
    if (!v || (int)v->size() != m->im) return -1;
    std::memcpy(out, v->data(), sizeof(double) * m->im);
    return 0;
}

int ref_setp(void* p, const char* name, const double* in)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    std::vector<double>* v = profile(m, name);
    if (!v) return -1;
    v->assign(in, in + m->im);
    return 0;
}

// scalars the run loop sets before the hot-path calls (cAtmosphereModel.cpp:1109-1131)
void ref_set_scalars(void* p, double dt, double diffusion_ramp, double buoyancy_ramp,
                     int total_iter_count, int iter_n)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    m->dt = dt;
    m->diffusion_ramp = diffusion_ramp;
    m->buoyancy_ramp = buoyancy_ramp;
    m->total_iter_count = total_iter_count;
    m->iter_n = iter_n;
}

// the momentum-budget capture of the right-hand side (vbudget_capture / wbudget_capture)
void ref_set_budget_capture(void* p, int on)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    m->vbudget_capture = (on != 0);
    m->wbudget_capture = (on != 0);
}

// a few derived constants, for the tests to compare with their own derivation
void ref_constants(void* p, double* out)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    out[0] = m->re_turb;
    out[1] = m->m_metric_r0;
    out[2] = m->metricShellLength();
    out[3] = m->m_comp.M_bg;
    out[4] = m->m_comp.R_bg;
    out[5] = m->m_comp.R_mix;
    out[6] = m->dt_visc;
}

void ref_rk4(void* p) { ((cAtmosphereModel*)p)->solveRungeKutta_Atmosphere_Turb(); }
void ref_pressure(void* p) { PressureSolverAtm(*(cAtmosphereModel*)p).run(false); }
void ref_project(void* p, int n) { PressureSolverAtm(*(cAtmosphereModel*)p).project_initial_velocity(n); }
void ref_satadj(void* p) { SaturationAdjustment(*(cAtmosphereModel*)p).run(); }
void ref_densities(void* p, int set_water) { ThermoAtm(*(cAtmosphereModel*)p).densities(set_water != 0); }
void ref_moist(void* p, int iter_n)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    m->iter_n = iter_n;
    MoistConvection(*m).run(iter_n);
}
void ref_store(void* p) { UtilsAtm(*(cAtmosphereModel*)p).storeIntermediateData3D(1.0); }
// the filters after the RK4 step, cAtmosphereModel.cpp:1507-1520, in their order
void ref_post_rk4_filters(void* p)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    AtomUtils::polar_zonal_filter(m->u, m->the.z, &m->i_topography, 30.0, 12, 3.0);
    AtomUtils::polar_zonal_filter(m->v, m->the.z, &m->i_topography, 30.0, 12, 3.0);
    AtomUtils::polar_zonal_filter(m->w, m->the.z, &m->i_topography, 30.0, 12, 3.0);
    AtomUtils::orographic_shapiro_filter(m->u, m->i_topography, 2, 3, 3);
    AtomUtils::orographic_shapiro_filter(m->v, m->i_topography, 2, 3, 3);
    AtomUtils::orographic_shapiro_filter(m->w, m->i_topography, 2, 3, 3);
    AtomUtils::radial_shapiro_filter(m->u, m->i_topography, 2, 1.0);
    AtomUtils::radial_shapiro_filter_ho(m->v, m->i_topography, 2, 1.0);
    AtomUtils::radial_shapiro_filter_ho(m->w, m->i_topography, 2, 1.0);
    AtomUtils::orographic_radial_shapiro_filter(m->t, m->i_topography, 2, 10, 2);
    AtomUtils::orographic_radial_shapiro_filter(m->c, m->i_topography, 2, 10, 2);
    AtomUtils::orographic_radial_shapiro_filter(m->cloud, m->i_topography, 2, 10, 2);
    AtomUtils::orographic_radial_shapiro_filter(m->ice, m->i_topography, 2, 10, 2);
    AtomUtils::steep_massif_field_smoothing(m->u, m->i_topography, 6, 3, 30, 1);
    AtomUtils::steep_massif_field_smoothing(m->v, m->i_topography, 6, 3, 30, 1);
    AtomUtils::steep_massif_field_smoothing(m->w, m->i_topography, 6, 3, 30, 1);
    AtomUtils::steep_massif_field_smoothing(m->p_dyn, m->i_topography, 6, 3, 30, 1);
    AtomUtils::coastal_velocity_sponge(m->u, m->i_topography, 3.0, 1.0, 12);
    AtomUtils::coastal_velocity_sponge(m->v, m->i_topography, 3.0, 1.0, 12);
    AtomUtils::coastal_velocity_sponge(m->w, m->i_topography, 3.0, 1.0, 12);
}
// the moist iteration's damp_wiggles of one field (cAtmosphereModel.cpp:1225-1228)
int ref_damp_wiggles(void* p, const char* name)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    Array* a = field3(m, name);
    if (!a) return -1;
    AtomUtils::damp_wiggles(*a, &m->i_topography, true, true, true);
    return 0;
}
// the per-iteration boundary conditions of cAtmosphereModel.cpp:1439-1446
void ref_bc(void* p)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    BC_Atm(*m).bcRadius();
    if (m->turb_model != "laminar") TurbulenceAtm(*m).apply_wall_bc();
    BC_Atm(*m).bcTheta();
    BC_Atm(*m).bcPhi();
    BC_Atm(*m).bcScalarSurfSur();
    BC_Atm(*m).bcSolidGround();
}
// TurbulenceAtm::run, the moist iteration's call (cAtmosphereModel.cpp:1426); the closure
// is the model's turb_model string, which TurbulenceAtm parses on construction
void ref_turbulence_run(void* p) { TurbulenceAtm(*(cAtmosphereModel*)p).run(); }
void ref_set_turb_model(void* p, const char* s) { ((cAtmosphereModel*)p)->turb_model = s; }
// the moist iteration's ice scheme of the configuration (CategoryIceScheme = 2,
// cAtmosphereModel.cpp:1238)
void ref_two_cat_ice(void* p) { TwoCatIceScheme(*(cAtmosphereModel*)p).run(); }
// the other CategoryIceScheme values' schemes, run on the model as they are
void ref_zero_cat_ice(void* p) { ZeroCatIceScheme(*(cAtmosphereModel*)p).run(); }
void ref_one_cat_ice(void* p) { OneCatIceScheme(*(cAtmosphereModel*)p).run(); }
void ref_three_cat_ice(void* p) { ThreeCatIceScheme(*(cAtmosphereModel*)p).run(); }
// MultiLayerRadiation::run, and radiation mode 2's apply_radiative_heating (the lambda of
// cAtmosphereModel.cpp:864-879, which saves t, runs the radiation and blends t toward the
// radiative equilibrium by omega_rad; restated here around the reference's own run())
// UtilsAtm::precipitationSum (the only callable part of the moist iteration's caps)
void ref_precipitation_sum(void* p) { UtilsAtm(*(cAtmosphereModel*)p).precipitationSum(); }
void ref_mlr(void* p) { MultiLayerRadiation(*(cAtmosphereModel*)p).run(); }
void ref_radiative_heating(void* p, double omega_rad)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    std::vector<double> t_backup((size_t)m->im * m->jm * m->km);
    size_t idx = 0;
    for (int i = 0; i < m->im; i++)
        for (int j = 0; j < m->jm; j++)
            for (int k = 0; k < m->km; k++) t_backup[idx++] = m->t.x[i][j][k];
    MultiLayerRadiation(*m).run();
    idx = 0;
    for (int i = 0; i < m->im; i++)
        for (int j = 0; j < m->jm; j++)
            for (int k = 0; k < m->km; k++) {
                const double re = m->t.x[i][j][k];
                m->t.x[i][j][k] = t_backup[idx++] * (1.0 - omega_rad) + re * omega_rad;
            }
}
void ref_level_mean(void* p) { ((cAtmosphereModel*)p)->computeLevelMeanTemperature(); }

// ThermoAtm::co2Column and ::waterBudget as first calls (the references they keep cleared
// first): out = m_q_co2_ref, m_q_h2o_ref, m_q_h2o_fixed_ref, m_air_levels [im],
// m_q_h2o_levels [im]
void ref_budgets(void* p, double* out)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    m->m_q_co2_ref = -1.0;
    m->m_q_h2o_ref = -1.0;
    m->m_q_h2o_fixed_ref = -1.0;
    m->m_air_levels.clear();
    m->m_q_h2o_levels.clear();
    ThermoAtm(*m).co2Column(false);
    ThermoAtm(*m).waterBudget(false);
    out[0] = m->m_q_co2_ref;
    out[1] = m->m_q_h2o_ref;
    out[2] = m->m_q_h2o_fixed_ref;
    for (int i = 0; i < m->im; i++) {
        out[3 + i] = m->m_air_levels[i];
        out[3 + m->im + i] = m->m_q_h2o_levels[i];
    }
}

// cAtmosphereModel::updateSkinTemperature with the given relaxation: the new t_skin
double ref_skin(void* p, double relax)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    m->t_skin_relax = relax;
    std::streambuf* prev = std::cout.rdbuf(g_null_buf());
    m->updateSkinTemperature(false);
    std::cout.rdbuf(prev);
    return m->t_skin;
}

// ThermoAtm::waterVapourEvaporation and ::latentSensibleHeat
void ref_evaporation(void* p) { ThermoAtm(*(cAtmosphereModel*)p).waterVapourEvaporation(); }
void ref_latent_sensible(void* p) { ThermoAtm(*(cAtmosphereModel*)p).latentSensibleHeat(); }

// ThermoAtm::standAtm_DewPoint_HumidRel, and the tropopause levels it reads (jm doubles)
void ref_stand_atm(void* p) { ThermoAtm(*(cAtmosphereModel*)p).standAtm_DewPoint_HumidRel(); }
void ref_tropopause(void* p, double* out)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    for (int j = 0; j < m->jm; j++) out[j] = m->tropopause_layers[j];
}

// UtilsAtm::findResiduumAtm.  It reports through its printout (and keeps the residuum in
// residuum_old), so the printout is captured and read back: out = residuum (exact),
// residuum_old before the call, grid average (8 significant digits); idx = i, j, k of the
// residuum, the finite cell count, the non-finite count (0 when the warning is absent).
void ref_residuum(void* p, double* out, long long* idx)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    out[1] = m->residuum_old;
    std::ostringstream cap;
    std::streambuf* prev = std::cout.rdbuf(cap.rdbuf());
    UtilsAtm(*m).findResiduumAtm();
    std::cout.rdbuf(prev);
    const std::string txt = cap.str();
    out[0] = m->residuum_old;
    auto after = [&](const char* key) -> std::string {
        const size_t at = txt.find(key);
        return (at == std::string::npos) ? std::string() : txt.substr(at + std::strlen(key));
    };
    std::string t = after("i_error = ");
    idx[0] = t.empty() ? -1 : std::atoll(t.c_str());
    t = after("j_error = ");
    idx[1] = t.empty() ? -1 : std::atoll(t.c_str());
    t = after("k_error = ");
    idx[2] = t.empty() ? -1 : std::atoll(t.c_str());
    t = after("grid average absolute error = ");
    out[2] = t.empty() ? -1.0 : std::atof(t.c_str());
    const size_t lp = t.find('(');
    idx[3] = (lp == std::string::npos) ? -1 : std::atoll(t.c_str() + lp + 1);
    t = after("WARNING \xe2\x80\x94 ");
    idx[4] = t.empty() ? 0 : std::atoll(t.c_str());
}

// RHS_Atmosphere_Turb at one cell on the current state, with the CellGeometry the RK4
// driver builds (RungeKutta_Atm_Turb.cpp:92-135).  out = rhs_t..rhs_dis (11), aux_u/v/w,
// prod, tke_source, dis_source.
void ref_rhs_cell(void* p, int i, int j, int k, double* out)
{
    cAtmosphereModel* m = (cAtmosphereModel*)p;
    cAtmosphereModel::CellGeometry geo;
    geo.rm = m->rad.z[i];
    geo.rm2 = geo.rm * geo.rm;
    geo.exp_rm = 1.0 / (geo.rm + 1.0);
    geo.exp_2_rm = geo.exp_rm * geo.exp_rm;
    double st = sin(m->the.z[j]);
    if (st < 0.55) st = 0.55;
    geo.sinthe = st;
    geo.sinthe2 = geo.sinthe * geo.sinthe;
    geo.costhe = cos(m->the.z[j]);
    const double rmet = m->metricRadius(geo.rm);
    const double rmet2 = rmet * rmet;
    geo.inv_rm = 1.0 / rmet;
    geo.inv_rm2 = 1.0 / rmet2;
    geo.inv_rmsinthe = 1.0 / (rmet * geo.sinthe);
    geo.inv_rm2sinthe = geo.inv_rm2 / geo.sinthe;
    geo.inv_rm2sinthe2 = geo.inv_rm2 / geo.sinthe2;
    geo.costhe_inv_rm2sinthe = geo.costhe * geo.inv_rm2sinthe;
    geo.inv_2dr = 1.0 / (2.0 * m->dr);
    geo.inv_2dthe = 1.0 / (2.0 * m->dthe);
    geo.inv_2dphi = 1.0 / (2.0 * m->dphi);
    geo.inv_dr2 = 1.0 / (m->dr * m->dr);
    geo.inv_dthe2 = 1.0 / (m->dthe * m->dthe);
    geo.inv_dphi2 = 1.0 / (m->dphi * m->dphi);
    if ((int)m->t_ref_level.size() != m->im) m->computeLevelMeanTemperature();
    m->RHS_Atmosphere_Turb(i, j, k, geo);
    const Array* r[11] = {&m->rhs_t, &m->rhs_u, &m->rhs_v, &m->rhs_w, &m->rhs_c, &m->rhs_cloud,
                          &m->rhs_ice, &m->rhs_g, &m->rhs_co2, &m->rhs_tke, &m->rhs_dis};
    for (int q = 0; q < 11; q++) out[q] = r[q]->x[i][j][k];
    out[11] = m->aux_u.x[i][j][k];
    out[12] = m->aux_v.x[i][j][k];
    out[13] = m->aux_w.x[i][j][k];
    out[14] = m->prod.x[i][j][k];
    out[15] = m->tke_source.x[i][j][k];
    out[16] = m->dis_source.x[i][j][k];
}

}  // extern "C"
