/*
 * or_ice.c - the ice / precipitation schemes (TEST INFRASTRUCTURE ONLY), flat terrain.
 *
 * TwoCatIceScheme::run (the configuration's CategoryIceScheme 2):
 *   initArrays               TwoCatIceScheme.h:126-158
 *   computeColumns           :162-484  (per (j, k) column, top-down, up to iter_prec_end
 *                                        passes until the rain flux at i_check settles)
 *   applyBoundaryConditions  :489-492 -> IceSchemeCommon::extrapolateBC (IceSchemeCommon.h:27-52)
 *   applyTopography          :497-501  (no land: nothing)
 * Within a column the reference keeps N_i, m_i, S_nuc and S_i_dep from one cell to the
 * next where a branch does not assign them; the restatement carries them the same way.
 *
 * ZeroCatIceScheme::run (ZeroCatIceScheme.h:37-230), OneCatIceScheme::run
 * (OneCatIceScheme.h:50-378) and ThreeCatIceScheme::run (ThreeCatIceScheme.h:70-470), with
 * IceSchemeCommon::depositionThrottle (IceSchemeCommon.h:203-237).  Each loops its columns
 * in the reference's order; OneCat's serial loop keeps S_au across cells and columns where a
 * cell has no cloud water, and the restatement carries it the same way (0 before the first
 * assignment, where the reference reads an uninitialised value).  All three read the rain
 * flux at level 23 for their convergence test, so they need im >= 24.
 */
#include "or_internal.h"

/* TwoCatIce constants, TwoCatIceScheme.h:17-71 */
#define TC_N_I_0    1.0e2
#define TC_M_I_0    1.0e-12
#define TC_M_I_MAX  1.0e-9
#define TC_M_S_0    3.0e-9
#define TC_C_I_DEP  1.3e-5
#define TC_C_C_AU   1.0e-3
#define TC_Q_C_CRIT 5.0e-4
#define TC_C_I_AU   1.0e-3
#define TC_C_AC     0.24
#define TC_C_RIM    18.6
#define TC_C_RIM_SNOW (18.6 / 5.0)
#define TC_C_AGG    10.3
#define TC_C_I_CRI  0.24
#define TC_C_R_CRI  3.2e-5
#define TC_A_EV     1.0e-3
#define TC_B_EV     5.9
#define TC_C_S_DEP  1.8e-2
#define TC_B_S_DEP  12.3
#define TC_C_S_MELT 8.43e-5
#define TC_B_S_MELT 12.05
#define TC_C_R_FRZ  3.75e-2
#define TC_T_NUC    267.15
#define TC_T_D      248.15
#define TC_T_HN     236.15
#define TC_T_R_FRZ  271.15
#define TC_ITER_PREC_END 3
#define TC_I_CHECK  1

static double q_sat_of(const or_params* p, double* const* f, size_t c, double E)
{
    const double M_other = or_M_nonwater(f[OF_C][c], f[OF_CO2][c], p->M_bg);
    return or_saturation_mass_fraction(E, f[OF_P_STAT][c], M_other);
}

/* IceSchemeCommon::extrapolateBC, c43 = 1 and c13 = 0 (const int members,
 * cAtmosphereModel.h:158); the phi-seam average where seam_avg is set */
static void extrapolate_bc_avg(int im, int jm, int km, double* P, int seam_avg)
{
    const double c43 = 1.0, c13 = 0.0;
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++)
            P[OR_IDX(im - 1, j, k)] = c43 * P[OR_IDX(im - 2, j, k)] - c13 * P[OR_IDX(im - 3, j, k)];
    for (int k = 0; k < km; k++)
        for (int i = 0; i < im; i++) {
            P[OR_IDX(i, 0, k)] = c43 * P[OR_IDX(i, 1, k)] - c13 * P[OR_IDX(i, 2, k)];
            P[OR_IDX(i, jm - 1, k)] = c43 * P[OR_IDX(i, jm - 2, k)] - c13 * P[OR_IDX(i, jm - 3, k)];
        }
    for (int i = 0; i < im; i++)
        for (int j = 0; j < jm; j++) {
            P[OR_IDX(i, j, 0)] = c43 * P[OR_IDX(i, j, 1)] - c13 * P[OR_IDX(i, j, 2)];
            P[OR_IDX(i, j, km - 1)] = c43 * P[OR_IDX(i, j, km - 2)] - c13 * P[OR_IDX(i, j, km - 3)];
            if (!seam_avg) continue;
            const double a = (P[OR_IDX(i, j, 0)] + P[OR_IDX(i, j, km - 1)]) * 0.5;
            P[OR_IDX(i, j, 0)] = a;
            P[OR_IDX(i, j, km - 1)] = a;
        }
}

static void extrapolate_bc(int im, int jm, int km, double* P) { extrapolate_bc_avg(im, jm, km, P, 1); }

void or_two_cat_ice_scheme(int im, int jm, int km, const or_params* p, double* const* f)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, 0);
    const size_t n = (size_t)im * jm * km;
    double* c_ = f[OF_C];
    double* cloud = f[OF_CLOUD];
    double* ice = f[OF_ICE];
    double* P_rain = f[OF_P_RAIN];
    double* P_snow = f[OF_P_SNOW];
    /* initArrays */
    for (size_t q = 0; q < n; q++) {
        c_[q] = or_max(0.0, c_[q]);
        cloud[q] = or_max(0.0, cloud[q]);
        ice[q] = or_max(0.0, ice[q]);
        f[OF_P_RAINN][q] = or_max(0.0, f[OF_P_RAINN][q]);
        f[OF_P_SNOWN][q] = or_max(0.0, f[OF_P_SNOWN][q]);
        P_rain[q] = f[OF_P_RAINN][q];
        P_snow[q] = f[OF_P_SNOWN][q];
    }
    const double t_0 = p->t_0;
    const double exp_1_6 = 1.0 / 6.0, exp_1_3 = 1.0 / 3.0, exp_2_3 = 2.0 / 3.0;
    const double exp_8_13 = 8.0 / 13.0, exp_5_26 = 5.0 / 26.0, exp_3_2 = 3.0 / 2.0;
    const double P_max = 50.0 / 86400.0;
    for (int k = 1; k < km - 1; k++)
        for (int j = 1; j < jm - 1; j++) {
            const double Rain_check = P_rain[OR_IDX(TC_I_CHECK, j, k)];
            double m_i = TC_M_I_MAX, N_i = 0.0, S_nuc = 0.0, S_i_dep = 0.0;
            for (int iter_prec = 1; iter_prec <= TC_ITER_PREC_END; iter_prec++) {
                P_rain[OR_IDX(im - 1, j, k)] = 0.0;
                P_snow[OR_IDX(im - 1, j, k)] = 0.0;
                for (int i = im - 2; i >= 0; i--) {
                    const size_t c = OR_IDX(i, j, k);
                    const double t_guard = f[OF_T][c] * t_0;
                    /* IceSchemeCommon::canCondense, :108-111 */
                    if (t_guard >= OR_T_CRIT || !(q_sat_of(p, f, c, or_saturation_pressure(t_guard)) < 1.0)) {
                        or_evaporate_where_impossible(p, f, c, t_guard);
                        continue;
                    }
                    const double Rain = P_rain[c];
                    const double Snow = P_snow[c];
                    double R49 = 0.0, R79 = 0.0, R139 = 0.0;
                    if (Rain > 1e-12) {
                        const double rb = pow(Rain, 1.0 / 9.0);
                        const double r2 = rb * rb;
                        const double r4 = r2 * r2;
                        R49 = r4;
                        R79 = Rain / r2;
                        R139 = Rain * r4;
                    }
                    const double t_u = f[OF_T][c] * t_0;
                    const double q_sat = q_sat_of(p, f, c, or_saturation_pressure(t_u));
                    const double q_Ice = q_sat_of(p, f, c, or_sublimation_pressure(t_u));
                    const double step = (double)((float)g.height[i + 1] - (float)g.height[i]);
                    const double rh = f[OF_R_HUMID][c];
                    const double mass_layer = rh * step;
                    const double dt_snow_dim = step / 0.96;
                    const double cv = c_[c], cl = cloud[c], ic = ice[c];
                    if (!(t_u > t_0) && !(t_u <= TC_T_HN)) {
                        N_i = TC_N_I_0 * exp(0.2 * (t_0 - t_u));
                        m_i = or_min((rh * ic) / N_i, TC_M_I_MAX);
                        if (m_i > TC_M_I_MAX) m_i = TC_M_I_MAX;
                        if (m_i < TC_M_I_0) m_i = TC_M_I_0;
                    }
                    if (ic == 0.0) {
                        if ((t_u < TC_T_D && cv >= q_Ice) || ((TC_T_D <= t_u && t_u <= TC_T_NUC) && cv >= q_sat))
                            S_nuc = TC_M_I_0 / (rh * dt_snow_dim) * N_i;
                    } else {
                        S_nuc = 0.0;
                    }
                    double S_c_frz = (t_u < TC_T_HN) ? cl / dt_snow_dim : 0.0;
                    if (cv > q_Ice) S_i_dep = TC_C_I_DEP * N_i * pow(m_i, exp_1_3) * (cv - q_Ice);
                    if (cv < q_Ice) S_i_dep = or_max(-ic / dt_snow_dim, (cv - q_Ice) / dt_snow_dim);
                    double S_c_au = (cl > TC_Q_C_CRIT) ? TC_C_C_AU * (cl - TC_Q_C_CRIT) : 0.0;
                    double S_i_au = (ic > 0.0) ? or_max(TC_C_I_AU * ic, 0.0) : 0.0;
                    double S_d_au = (S_i_dep > 0.0) ? S_i_dep / (1.5 * (pow(TC_M_S_0 / m_i, exp_2_3) - 1.0)) : 0.0;
                    double S_ac = (t_u >= t_0 && cl > TC_Q_C_CRIT) ? TC_C_AC * (cl - TC_Q_C_CRIT) * R79 : 0.0;
                    double S_rim = (t_u < t_0) ? TC_C_RIM_SNOW * cl * Snow : 0.0;
                    double S_shed = (t_u >= t_0) ? TC_C_RIM * cl * Snow : 0.0;
                    double S_s_melt = 0.0, S_i_melt = 0.0;
                    if (t_u > t_0) {
                        if (Snow > 1e-12) {
                            S_s_melt = TC_C_S_MELT * (1.0 + TC_B_S_MELT * pow(Snow, exp_5_26))
                                     * (t_u - t_0) * pow(Snow, exp_1_3);
                            S_s_melt = or_min(S_s_melt, Snow / mass_layer);
                        }
                        S_i_melt = ic / dt_snow_dim;
                    }
                    double S_agg = 0.0, S_i_cri = 0.0, S_r_cri = 0.0;
                    if (t_u <= t_0) {
                        S_agg = TC_C_AGG * ic * Snow;
                        S_i_cri = TC_C_I_CRI * ic * R79;
                        S_r_cri = TC_C_R_CRI * ic / m_i * R139;
                    }
                    double S_ev = 0.0;
                    if (t_u > t_0 && Rain > 1e-12 && cv < q_sat) {
                        S_ev = TC_A_EV * (1.0 + TC_B_EV * pow(Rain, exp_1_6)) * (q_sat - cv) * R49;
                        S_ev = or_min(S_ev, Rain / mass_layer);
                    }
                    double S_s_dep = 0.0;
                    if (t_u < t_0 && Snow > 1e-12) {
                        S_s_dep = TC_C_S_DEP * (1.0 + TC_B_S_DEP * pow(Snow, exp_5_26)) * (cv - q_Ice)
                                * pow(Snow, exp_8_13);
                        if (S_s_dep < 0.0) S_s_dep = or_max(S_s_dep, -Snow / mass_layer);
                    }
                    double S_r_frz = 0.0;
                    if (t_u <= t_0) {
                        const double t_frz = or_max(TC_T_R_FRZ - t_u, 0.0);
                        S_r_frz = TC_C_R_FRZ * pow(t_frz, exp_3_2) * pow(Rain, exp_3_2);
                    }
                    /* limiters, :413-434 */
                    const double S_cloud_total = S_c_au + S_ac + S_rim + S_c_frz + S_shed;
                    const double max_cloud_loss = cl / dt_snow_dim;
                    if (S_cloud_total > max_cloud_loss && S_cloud_total > 0) {
                        const double fac = max_cloud_loss / S_cloud_total;
                        S_c_au *= fac; S_ac *= fac; S_rim *= fac; S_c_frz *= fac; S_shed *= fac;
                    }
                    const double S_ice_total = S_i_au + S_d_au + S_agg + S_i_cri + S_i_melt;
                    const double max_ice_loss = ic / dt_snow_dim;
                    if (S_ice_total > max_ice_loss && S_ice_total > 0) {
                        const double fac = max_ice_loss / S_ice_total;
                        S_i_au *= fac; S_d_au *= fac; S_agg *= fac; S_i_cri *= fac; S_i_melt *= fac;
                    }
                    /* sources and sinks, :438-465 */
                    const double S_c_c = f[OF_S_C_C][c];
                    f[OF_S_V][c] = -S_c_c + S_ev - S_i_dep - S_s_dep - S_nuc;
                    f[OF_S_C][c] = S_c_c - S_c_au - S_ac - S_c_frz + S_i_melt - S_rim - S_shed;
                    f[OF_S_I][c] = S_nuc + S_c_frz + S_i_dep - S_i_melt - S_i_au - S_d_au - S_agg - S_i_cri;
                    f[OF_S_R][c] = S_c_au + S_ac - S_ev + S_shed - S_r_cri - S_r_frz + S_s_melt;
                    f[OF_S_S][c] = S_i_au + S_d_au + S_agg + S_rim + S_s_dep + S_i_cri + S_r_cri + S_r_frz
                                 - S_s_melt;
                    /* the fluxes, integrated top-down and capped at 50 mm/d, :478-509 */
                    const double dP_rain = (S_c_au + S_ac + S_shed + S_s_melt - S_ev - S_r_frz) * mass_layer;
                    P_rain[c] = or_min(P_max, or_max(0.0, P_rain[c + (size_t)jm * km] + dP_rain));
                    const double dP_snow = (S_i_au + S_d_au + S_rim + S_agg + S_r_frz - S_s_melt) * mass_layer;
                    P_snow[c] = (t_u < t_0 && t_u >= p->t_000)
                              ? or_min(P_max, or_max(0.0, P_snow[c + (size_t)jm * km] + dP_snow)) : 0.0;
                    f[OF_PRECIPITATION][c] = or_min(P_max, P_rain[c] + P_snow[c]);
                }
                const double P_rain_diff = fabs(P_rain[OR_IDX(TC_I_CHECK, j, k)] - Rain_check) * 8.64e4;
                if (P_rain_diff <= 1.0e-3) break;
            }
        }
    extrapolate_bc(im, jm, km, P_rain);
    extrapolate_bc(im, jm, km, P_snow);
    or_geom_free(&g);
}

/* ---------------------------------------------------------------------------------------
 * shared by ZeroCat, OneCat and ThreeCat
 * ------------------------------------------------------------------------------------- */

#define IC_CHECK_LEVEL 23      /* the convergence level of ZeroCat/OneCat/ThreeCat */

/* IceSchemeCommon::canCondense (IceSchemeCommon.h:108-111) */
static int can_condense(const or_params* p, double* const* f, size_t c, double t_u)
{
    if (t_u >= OR_T_CRIT) return 0;
    return q_sat_of(p, f, c, or_saturation_pressure(t_u)) < 1.0;
}

/* the layer thickness table, float heights subtracted in float (get_layer_height) */
static void step_table(const or_geom* g, int im, double* step)
{
    for (int i = 0; i < im; i++)
        step[i] = (i < im - 1) ? (double)((float)g->height[i + 1] - (float)g->height[i]) : 0.0;
}

/* IceSchemeCommon::depositionThrottle (IceSchemeCommon.h:203-237) */
typedef struct ice_snow_rates { double S_i_dep, S_i_au, S_d_au, N_i, m_i; } ice_snow_rates;

static ice_snow_rates deposition_throttle(const or_params* p, double* const* f, size_t c,
                                          double t_u, double q_Ice, double dt_snow_dim)
{
    const double N_i_0 = 1.0e2, m_i_0 = 1.0e-12, m_i_max = 1.0e-9, m_s_0 = 3.0e-9;
    const double c_i_dep = 1.3e-5, c_i_au = 1.0e-3, t_hn = 236.15;
    ice_snow_rates r = { 0.0, 0.0, 0.0, 0.0, 1.0e-9 };
    const double cv = f[OF_C][c], ice = f[OF_ICE][c];
    double N_i = 0.0, m_i = m_i_max;
    if (t_u <= p->t_0 && t_u > t_hn) {
        N_i = N_i_0 * exp(0.2 * (p->t_0 - t_u));
        m_i = or_min(f[OF_R_HUMID][c] * ice / N_i, m_i_max);
        m_i = or_max(m_i_0, or_min(m_i, m_i_max));
    }
    if (cv > q_Ice)      r.S_i_dep = c_i_dep * N_i * pow(m_i, 1.0 / 3.0) * (cv - q_Ice);
    else if (cv < q_Ice) r.S_i_dep = or_max(-ice / dt_snow_dim, (cv - q_Ice) / dt_snow_dim);
    if (ice > 0.0)       r.S_i_au = or_max(c_i_au * ice, 0.0);
    if (r.S_i_dep > 0.0) r.S_d_au = r.S_i_dep / (1.5 * (pow(m_s_0 / m_i, 2.0 / 3.0) - 1.0));
    r.N_i = N_i; r.m_i = m_i;
    return r;
}

/* ---------------------------------------------------------------------------------------
 * ZeroCatIceScheme::run (ZeroCatIceScheme.h:37-230)
 * ------------------------------------------------------------------------------------- */
void or_zero_cat_ice_scheme(int im, int jm, int km, const or_params* p, double* const* f)
{
    const double tau_r_inv = 1.0 / 3.3e3, q_c_crit = 5.0e-4, b_ev = 8.05, c_ac = 0.24;
    const int iter_prec_end = 2;
    or_geom g;
    or_geom_init(&g, im, jm, km, p, 0);
    double* step = (double*)malloc((size_t)im * sizeof(double));
    step_table(&g, im, step);
    const size_t n = (size_t)im * jm * km, up = (size_t)jm * km;
    double* c_ = f[OF_C];
    double* cloud = f[OF_CLOUD];
    double* P_rain = f[OF_P_RAIN];
    double* P_snow = f[OF_P_SNOW];
    const double t_0 = p->t_0;
    /* initArrays, :69-94 */
    for (size_t q = 0; q < n; q++) {
        c_[q] = or_max(0.0, c_[q]);
        cloud[q] = or_max(0.0, cloud[q]);
        P_rain[q] = or_max(0.0, f[OF_P_RAINN][q]);
        P_snow[q] = or_max(0.0, f[OF_P_SNOWN][q]);
    }
    /* computeColumns, :98-181 */
    for (int j = 1; j < jm - 1; j++)
        for (int k = 1; k < km - 1; k++)
            for (int iter_prec = 1; iter_prec <= iter_prec_end; iter_prec++) {
                const double Rain_check = P_rain[OR_IDX(IC_CHECK_LEVEL, j, k)];
                P_rain[OR_IDX(im - 1, j, k)] = 0.0;
                P_snow[OR_IDX(im - 1, j, k)] = 0.0;
                for (int i = im - 2; i >= 0; i--) {
                    const size_t c = OR_IDX(i, j, k);
                    const double t_guard = f[OF_T][c] * t_0;
                    if (!can_condense(p, f, c, t_guard)) {
                        or_evaporate_where_impossible(p, f, c, t_guard);
                        continue;
                    }
                    const double Rain = P_rain[c];
                    const double t_u = f[OF_T][c] * t_0;
                    const double cl_i = cloud[c];
                    const double q_sat = q_sat_of(p, f, c, or_saturation_pressure(t_u));
                    const double S_ac = (t_u >= t_0 && Rain > 0.0) ? c_ac * cl_i * pow(Rain, 7.0 / 9.0) : 0.0;
                    const double S_au = (cl_i > q_c_crit) ? (cl_i - q_c_crit) * tau_r_inv : 0.0;
                    double S_ev = 0.0;
                    if (t_u >= t_0 && Rain > 0.0) {
                        const double a_ev = 2.76e-3 * exp(0.055 * (t_0 - t_u));
                        const double Rain_1_6 = pow(Rain, 1.0 / 6.0);
                        const double Rain_4_9 = pow(Rain, 4.0 / 9.0);
                        S_ev = a_ev * (1.0 + b_ev * Rain_1_6) * (q_sat - c_[c]) * Rain_4_9;
                    }
                    const double S_c_c = f[OF_S_C_C][c];
                    f[OF_S_V][c] = -S_c_c + S_ev;
                    f[OF_S_C][c] = S_c_c - S_au - S_ac;
                    f[OF_S_R][c] = S_au + S_ac - S_ev;
                    if (t_u >= t_0)
                        P_rain[c] = or_max(0.0, P_rain[c + up] + f[OF_R_HUMID][c + up] * f[OF_S_R][c + up] * step[i]);
                    else
                        P_rain[c] = 0.0;
                    f[OF_PRECIPITATION][c] = P_rain[c];
                }
                const double P_rain_diff = fabs(P_rain[OR_IDX(IC_CHECK_LEVEL, j, k)] - Rain_check) * 8.64e4;
                if (P_rain_diff <= 1.0e-3) break;
            }
    /* applyBoundaryConditions, :206-209; applyTopography (no land: nothing) */
    extrapolate_bc_avg(im, jm, km, P_rain, 1);
    extrapolate_bc_avg(im, jm, km, P_snow, 0);
    free(step);
    or_geom_free(&g);
}

/* ---------------------------------------------------------------------------------------
 * OneCatIceScheme::run (OneCatIceScheme.h:50-378)
 * ------------------------------------------------------------------------------------- */
void or_one_cat_ice_scheme(int im, int jm, int km, const or_params* p, double* const* f)
{
    const double c_ac = 0.24, c_rim = 0.69, b_ev = 5.98, a_melt = 3.90e-6, b_melt = 10.50;
    const double a_if = 1.92e-6, a_cf = 3.97e-5, E_cf = 5.0e-3;
    const double N_cf_0_surf = 2.0e5, N_cf_0_top = 1.0e4, tau_r = 3.3e3;
    const double q_c_crit = 5.0e-4, a_mc = 0.08, a_mv = 0.02, P_max_flux = 3.0e-3;
    const int iter_prec_end = 2;
    or_geom g;
    or_geom_init(&g, im, jm, km, p, 0);
    double* step = (double*)malloc((size_t)im * sizeof(double));
    step_table(&g, im, step);
    const size_t n = (size_t)im * jm * km, up = (size_t)jm * km;
    double* c_ = f[OF_C];
    double* cloud = f[OF_CLOUD];
    double* P_rain = f[OF_P_RAIN];
    double* P_snow = f[OF_P_SNOW];
    const double t_0 = p->t_0, t_00 = p->t_00, t_000 = p->t_000;
    const double t_m1 = 0.5 * (t_0 + t_000), t_m2 = 0.5 * (t_0 + t_00);
    /* initArrays, :89-104: the restart copies are not clamped */
    for (size_t q = 0; q < n; q++) {
        if (c_[q] < 0.0) c_[q] = 0.0;
        if (cloud[q] < 0.0) cloud[q] = 0.0;
        if (f[OF_ICE][q] < 0.0) f[OF_ICE][q] = 0.0;
        P_rain[q] = f[OF_P_RAINN][q];
        P_snow[q] = f[OF_P_SNOWN][q];
    }
    /* computeColumns, :108-349; S_au lives across cells and columns */
    double S_au = 0.0;
    for (int k = 1; k < km - 1; k++)
        for (int j = 1; j < jm - 1; j++)
            for (int iter_prec = 1; iter_prec <= iter_prec_end; iter_prec++) {
                const double Rain_check = P_rain[OR_IDX(IC_CHECK_LEVEL, j, k)];
                P_rain[OR_IDX(im - 1, j, k)] = 0.0;
                P_snow[OR_IDX(im - 1, j, k)] = 0.0;
                for (int i = im - 2; i >= 0; i--) {
                    const size_t c = OR_IDX(i, j, k);
                    const double t_guard = f[OF_T][c] * t_0;
                    if (!can_condense(p, f, c, t_guard)) {
                        or_evaporate_where_impossible(p, f, c, t_guard);
                        continue;
                    }
                    const double Rain = P_rain[c];
                    const double Snow = P_snow[c];
                    const double t_u = f[OF_T][c] * t_0;
                    const double q_sat = q_sat_of(p, f, c, or_saturation_pressure(t_u));
                    const double q_Ice = q_sat_of(p, f, c, or_sublimation_pressure(t_u));
                    const double dt_snow_dim = step[i] / 0.96;
                    const ice_snow_rates thr = deposition_throttle(p, f, c, t_u, q_Ice, dt_snow_dim);
                    double a_m;
                    if (t_u < t_0 && t_u >= t_m1)
                        a_m = a_mc - a_mv * (1.0 + cos(2.0 * M_PI * (t_u - t_m1) / (t_0 - t_000)));
                    else
                        a_m = a_mc;
                    double eps_t;
                    if (t_u > t_00 && t_u <= t_0)
                        eps_t = 0.5 * (1.0 + sin(M_PI * (t_m2 - t_u) / (t_0 - t_00)));
                    else
                        eps_t = 0.0;
                    const double cl = cloud[c];
                    if (cl > 0.0) S_au = (1.0 - eps_t) / tau_r * or_max(0.0, cl - q_c_crit);
                    const double S_ac = (1.0 - eps_t) * c_ac * cl * pow(Rain, 7.0 / 9.0);
                    double S_rim = 0.0, S_shed = 0.0;
                    if (t_u < t_0)
                        S_rim = (cl > q_c_crit) ? (c_rim / 5.0) / a_m * (cl - q_c_crit) * Snow : 0.0;
                    if (t_u >= t_0)
                        S_shed = (cl > q_c_crit) ? (c_rim / 5.0) / a_m * (cl - q_c_crit) * Snow : 0.0;
                    const double a_ev = 2.76e-3 * exp(0.055 * (t_0 - t_u));
                    const double S_ev = a_ev * (1.0 + b_ev * pow(Rain, 1.0 / 6.0)) * (q_sat - c_[c])
                                      * pow(Rain, 4.0 / 9.0);
                    const double S_melt = a_melt / pow(a_mc, -0.5)
                                        * (1.0 + b_melt * pow(a_mc, -0.25) * pow(Snow, 0.9 / 4.3))
                                        * ((t_u - t_0) * pow(Snow, 5.0 / 8.6));
                    const double p0 = f[OF_P_STAT][OR_IDX(0, j, k)];
                    double N_cf_0 = N_cf_0_surf + (N_cf_0_surf - N_cf_0_top) / (p0 - 500.0)
                                  * (f[OF_P_STAT][c] - p0);
                    if (f[OF_P_STAT][c] <= 500.0) N_cf_0 = N_cf_0_top;
                    const double N_cf = (t_u < 270.16) ? N_cf_0 * pow(270.16 - t_u, 1.3) : 0.0;
                    double S_frz = 0.0;
                    if (t_u <= t_0 && t_u >= t_00) {
                        const double S_if_frz = a_if * (exp(a_if * (t_u - t_0)) - 1.0) * pow(Rain, 14.0 / 9.0);
                        const double S_cf_frz = a_cf * E_cf * N_cf * pow(Rain, 13.0 / 9.0);
                        S_frz = S_if_frz + S_cf_frz;
                    }
                    f[OF_S_V][c] = -f[OF_S_C_C][c] + S_ev;
                    f[OF_S_C][c] = f[OF_S_C_C][c] - S_au - S_ac - S_rim - S_shed;
                    f[OF_S_R][c] = S_au + S_ac - S_ev + S_shed - S_frz + S_melt;
                    f[OF_S_S][c] = thr.S_i_au + thr.S_d_au + S_rim + S_frz - S_melt;
                    double pr = (t_u >= t_0) ? P_rain[c + up] + f[OF_R_HUMID][c + up] * f[OF_S_R][c + up] * step[i] : 0.0;
                    if (pr < 0.0) pr = 0.0;
                    if (pr > P_max_flux) pr = P_max_flux;
                    P_rain[c] = pr;
                    double ps = (t_u < t_0 && t_u >= t_00)
                              ? P_snow[c + up] + f[OF_R_HUMID][c + up] * f[OF_S_S][c + up] * step[i] : 0.0;
                    if (ps < 0.0) ps = 0.0;
                    if (ps > P_max_flux) ps = P_max_flux;
                    P_snow[c] = ps;
                    f[OF_PRECIPITATION][c] = pr + ps;
                }
                const double P_rain_diff = fabs(P_rain[OR_IDX(IC_CHECK_LEVEL, j, k)] - Rain_check) * 8.64e4;
                if (P_rain_diff <= 1.0e-3) break;
            }
    /* applyBoundaryConditions, :354-357; applyTopography (no land: nothing) */
    extrapolate_bc_avg(im, jm, km, P_rain, 1);
    extrapolate_bc_avg(im, jm, km, P_snow, 1);
    free(step);
    or_geom_free(&g);
}

/* ---------------------------------------------------------------------------------------
 * ThreeCatIceScheme::run (ThreeCatIceScheme.h:70-470)
 * ------------------------------------------------------------------------------------- */
void or_three_cat_ice_scheme(int im, int jm, int km, const or_params* p, double* const* f)
{
    /* ThreeCatIce constants, :17-66 */
    const double N_g_0 = 4.0e6, m_i_0 = 1.0e-12, N_r_0 = 8.0e+6, N_s_0 = 8.0e+5;
    const double v_s_0 = 130.0, v_r_0 = 4.9, v_g_0 = 442.0;
    const double c_c_au = 4.0e-4, c_ac = 0.24, c_rim = 18.6, c_agg = 10.3, c_i_cri = 0.24;
    const double c_r_cri = 3.2e-5, b_ev = 5.9, c_r_frz = 3.75e-2;
    const double z_csg = 0.5, c_g_rim = 4.43, c_g_agg = 2.46, a_s_m = 0.038, a_g_m = 169.6;
    const double t_nuc = 267.15, t_d = 248.15, t_hn = 236.15, t_r_frz = 271.15;
    const double P_norm_floor = 1.0e-6, P_max_flux = 3.0e-3;
    const int iter_prec_end = 2;
    or_geom g;
    or_geom_init(&g, im, jm, km, p, 0);
    double* step = (double*)malloc((size_t)im * sizeof(double));
    step_table(&g, im, step);
    const size_t n = (size_t)im * jm * km, up = (size_t)jm * km;
    double* c_ = f[OF_C];
    double* cloud = f[OF_CLOUD];
    double* ice = f[OF_ICE];
    double* P_rain = f[OF_P_RAIN];
    double* P_snow = f[OF_P_SNOW];
    double* P_graupel = f[OF_P_GRAUPEL];
    const double t_0 = p->t_0;
    /* initArrays, :119-144: the restart copies are not clamped */
    for (size_t q = 0; q < n; q++) {
        c_[q] = or_max(0.0, c_[q]);
        cloud[q] = or_max(0.0, cloud[q]);
        ice[q] = or_max(0.0, ice[q]);
        f[OF_GR][q] = or_max(0.0, f[OF_GR][q]);
        P_rain[q] = f[OF_P_RAINN][q];
        P_snow[q] = f[OF_P_SNOWN][q];
    }
    /* computeColumns' constants, :147-170 */
    const double gamma_4_5 = tgamma(4.5), gamma_4_0 = tgamma(4.0), gamma_3_25 = tgamma(3.25);
    const double A_r = p->r_0_water * M_PI * N_r_0;
    const double A_s = 2.0 * a_s_m * N_s_0;
    const double A_g = 2.0 * a_g_m * N_g_0;
    const double B_rad = p->r_0_water * M_PI * N_r_0 * v_r_0 * gamma_4_5 / gamma_4_0;
    const double B_s = N_s_0 * v_s_0 * a_s_m * gamma_3_25;
    const double B_g = N_g_0 * v_g_0 * a_g_m * gamma_3_25;
    const double B_rad_neg89 = pow(B_rad, -8.0 / 9.0);
    const double B_s_neg1213 = pow(B_s, -12.0 / 13.0);
    const double B_g_neg1213 = pow(B_g, -12.0 / 13.0);
    const double E_sat_t_0_Pa = 1e2 * or_saturation_pressure(t_0);
    /* :175-420 */
    for (int j = 1; j < jm - 1; j++)
        for (int k = 1; k < km - 1; k++) {
            P_rain[OR_IDX(IC_CHECK_LEVEL, j, k)] = 0.0;
            for (int iter_prec = 1; iter_prec <= iter_prec_end; iter_prec++) {
                const double Rain_check = P_rain[OR_IDX(IC_CHECK_LEVEL, j, k)];
                P_rain[OR_IDX(im - 1, j, k)] = 0.0;
                P_snow[OR_IDX(im - 1, j, k)] = 0.0;
                P_graupel[OR_IDX(im - 1, j, k)] = 0.0;
                for (int i = im - 2; i >= 0; i--) {
                    const size_t c = OR_IDX(i, j, k);
                    const double t_guard = f[OF_T][c] * t_0;
                    if (!can_condense(p, f, c, t_guard)) {
                        or_evaporate_where_impossible(p, f, c, t_guard);
                        continue;
                    }
                    const size_t c0 = OR_IDX(0, j, k);
                    const double P_rain_0 = or_max(P_rain[c0], P_norm_floor);
                    const double P_snow_0 = or_max(P_snow[c0], P_norm_floor);
                    const double P_graupel_0 = or_max(P_graupel[c0], P_norm_floor);
                    const double Rain = P_rain[c] / P_rain_0;
                    const double Snow = P_snow[c] / P_snow_0;
                    const double Graupel = P_graupel[c] / P_graupel_0;
                    const double Rain_79 = (Rain > 0.0) ? pow(Rain, 7.0 / 9.0) : 0.0;
                    const double Rain_89 = (Rain > 0.0) ? pow(Rain, 8.0 / 9.0) : 0.0;
                    const double Rain_139 = (Rain > 0.0) ? pow(Rain, 13.0 / 9.0) : 0.0;
                    const double Rain_16 = (Rain > 0.0) ? pow(Rain, 1.0 / 6.0) : 0.0;
                    const double Rain_49 = (Rain > 0.0) ? pow(Rain, 4.0 / 9.0) : 0.0;
                    const double r_q_r = A_r * B_rad_neg89 * Rain_89;
                    const double r_q_s = A_s * B_s_neg1213 * ((Snow > 0.0) ? pow(Snow, 12.0 / 13.0) : 0.0);
                    const double r_q_g = A_g * B_g_neg1213 * ((Graupel > 0.0) ? pow(Graupel, 12.0 / 13.0) : 0.0);
                    const double t_u = f[OF_T][c] * t_0;
                    const double p_u_0 = 1e2 * f[OF_P_STAT][c];
                    const double r_h_i = f[OF_R_HUMID][c];
                    const double c_ijk = c_[c], cl_i = cloud[c], ice_i = ice[c];
                    const double step_i = step[i];
                    const double q_sat = q_sat_of(p, f, c, or_saturation_pressure(t_u));
                    const double q_Ice = q_sat_of(p, f, c, or_sublimation_pressure(t_u));
                    const double dt_rain_dim = step_i / 1.6;
                    const double dt_snow_dim = step_i / 0.96;
                    const double rh_rqs_08 = (r_q_s > 0.0) ? pow(r_h_i * r_q_s, 0.8) : 0.0;
                    const double rh_rqg_06 = (r_q_g > 0.0) ? pow(r_h_i * r_q_g, 0.6) : 0.0;
                    const double rh_rqg_95 = (r_q_g > 0.0) ? pow(r_h_i * r_q_g, 0.94878) : 0.0;
                    const ice_snow_rates thr = deposition_throttle(p, f, c, t_u, q_Ice, dt_snow_dim);
                    const double m_i = thr.m_i, N_i = thr.N_i;
                    double S_nuc = 0.0;
                    if (ice_i == 0.0) {
                        if ((t_u < t_d && c_ijk >= q_Ice) || (t_d <= t_u && t_u <= t_nuc && c_ijk >= q_sat))
                            S_nuc = m_i_0 / (r_h_i * dt_snow_dim) * N_i;
                    }
                    const double S_c_frz = (t_u < t_hn && cl_i > 0.0) ? cl_i / dt_rain_dim : 0.0;
                    const double S_i_dep = thr.S_i_dep;
                    const double S_c_au = (t_u >= t_0 && cl_i > 0.0) ? or_max(c_c_au * (cl_i - 0.0002), 0.0) : 0.0;
                    const double S_i_au = thr.S_i_au, S_d_au = thr.S_d_au;
                    const double S_ac = (t_u >= t_0) ? c_ac * cl_i * Rain_79 : 0.0;
                    double S_s_rim, S_g_rim, S_s_shed, S_g_shed;
                    if (t_u < t_0) {
                        S_s_rim = c_rim * cl_i * Snow;
                        S_g_rim = c_rim * cl_i * rh_rqg_95;
                        S_s_shed = 0.0;
                        S_g_shed = 0.0;
                    } else {
                        S_s_rim = 0.0;
                        S_g_rim = 0.0;
                        S_s_shed = c_rim * cl_i * Snow;
                        S_g_shed = c_g_rim * cl_i * rh_rqg_95;
                    }
                    double S_s_agg = 0.0, S_g_agg = 0.0, S_i_cri = 0.0, S_r_cri = 0.0;
                    if (t_u <= t_0) {
                        S_s_agg = c_agg * ice_i * Snow;
                        S_g_agg = c_g_agg * ice_i * rh_rqg_95;
                        S_i_cri = c_i_cri * ice_i * Rain_79;
                        S_r_cri = c_r_cri * ice_i / m_i * Rain_139;
                    }
                    double S_ev = 0.0;
                    if (t_u >= t_0 && Rain > 0.0) {
                        const double a_ev = 2.76e-3 * exp(0.055 * (t_0 - t_u));
                        S_ev = a_ev * (1.0 + b_ev * Rain_16) * (q_sat - c_ijk) * Rain_49;
                    }
                    double S_s_dep, S_g_dep;
                    const double inv_p_u_0 = 1.0 / p_u_0;
                    const double c_minus_qIce = c_ijk - q_Ice;
                    const double d_v = (t_u >= t_0)
                        ? 101325.0 * inv_p_u_0 * (2.22e-5 + 1.46e-7 * (t_u - t_0))
                        : 101325.0 * inv_p_u_0 * (2.22e-5 + 1.25e-7 * (t_u - t_0));
                    const double l_h = 0.024 + 8.0e-5 * (t_u - t_0);
                    const double q_sat_t_0 = or_saturation_mass_fraction(
                        E_sat_t_0_Pa, p_u_0, or_M_nonwater(c_ijk, f[OF_CO2][c], p->M_bg));
                    const double t_crit = (c_ijk >= q_sat_t_0)
                        ? t_0 - (1.0 / l_h) * p->ls * d_v * r_h_i * (c_ijk - q_sat_t_0) : t_0;
                    if (t_u < t_0) {
                        S_s_dep = (2.91955 - 0.0109928 * t_u + 15871.3 * inv_p_u_0 + 1.74744e-6 * p_u_0)
                                * c_minus_qIce * rh_rqs_08;
                        S_g_dep = 0.0;
                    } else if (t_u < t_crit) {
                        S_s_dep = (0.28003 - 0.146293e-6 * p_u_0) * c_minus_qIce * rh_rqs_08;
                        S_g_dep = (0.0418521 - 4.7524e-8 * p_u_0) * c_minus_qIce * rh_rqg_06;
                    } else {
                        S_s_dep = (2.41897 + 31282.3 * inv_p_u_0) * c_minus_qIce * rh_rqs_08;
                        S_g_dep = (0.153907 - 7.86703e-7 * p_u_0) * c_minus_qIce * rh_rqg_06;
                    }
                    double S_s_melt = 0.0, S_g_melt = 0.0;
                    if (t_u >= t_0) {
                        const double a_melt = 2.95e+3;
                        const double melt_driver = (t_u - t_0) + a_melt * (c_ijk - q_sat_t_0);
                        S_s_melt = melt_driver * (0.612654e-3 + 79.6863 * inv_p_u_0) * rh_rqs_08;
                        S_g_melt = melt_driver * (7.39441e-5 + 12.31698 * inv_p_u_0) * rh_rqg_06;
                    }
                    const double S_i_melt = (t_u > t_0 && ice_i > 0.0) ? ice_i / dt_snow_dim : 0.0;
                    double S_r_frz;
                    if (t_u > t_hn) {
                        const double t_frz = or_max(t_r_frz - t_u, 0.0);
                        S_r_frz = c_r_frz * pow(t_frz, 1.5) * pow(r_h_i * r_q_r, 27.0 / 16.0);
                    } else {
                        S_r_frz = Rain / dt_rain_dim;
                    }
                    const double S_csg = (t_u <= t_0 && cl_i > 0.0002)
                        ? z_csg * cl_i * ((r_q_s > 0.0) ? pow(r_h_i * r_q_s, 0.75) : 0.0) : 0.0;
                    const double S_c_c = f[OF_S_C_C][c];
                    f[OF_S_V][c] = -S_c_c + S_ev - S_i_dep - S_s_dep - S_g_dep - S_nuc;
                    f[OF_S_C][c] = S_c_c - S_c_au - S_ac - S_c_frz + S_i_melt
                                 - S_s_rim - S_g_rim - S_s_shed - S_g_shed;
                    f[OF_S_I][c] = S_nuc + S_c_frz + S_i_dep - S_i_melt
                                 - S_i_au - S_d_au - S_s_agg - S_g_agg - S_i_cri;
                    f[OF_S_R][c] = S_c_au + S_ac - S_ev + S_s_shed + S_g_shed
                                 - S_r_cri - S_r_frz + S_s_melt + S_g_melt;
                    f[OF_S_S][c] = S_i_au + S_d_au + S_s_agg + S_s_rim + S_s_dep
                                 + S_i_cri + S_r_cri - S_s_melt - S_csg;
                    f[OF_S_G][c] = S_g_agg + S_g_rim + S_g_dep + S_i_cri + S_r_cri
                                 + S_r_frz - S_g_melt + S_csg;
                    /* the capped top-down fluxes, :395-412 */
                    const double rh_up = f[OF_R_HUMID][c + up];
                    P_rain[c] = (t_u >= t_0)
                        ? or_min(P_max_flux, or_max(0.0, P_rain[c + up] + rh_up * f[OF_S_R][c + up] * step_i)) : 0.0;
                    P_snow[c] = (t_u < t_0 && t_u >= p->t_000)
                        ? or_min(P_max_flux, or_max(0.0, P_snow[c + up] + rh_up * f[OF_S_S][c + up] * step_i)) : 0.0;
                    P_graupel[c] = (t_u < t_0 && t_u >= p->t_00)
                        ? or_min(P_max_flux, or_max(0.0, P_graupel[c + up] + rh_up * f[OF_S_G][c + up] * step_i)) : 0.0;
                    f[OF_PRECIPITATION][c] = P_rain[c] + P_snow[c] + P_graupel[c];
                }
                const double P_rain_diff = fabs(P_rain[OR_IDX(IC_CHECK_LEVEL, j, k)] - Rain_check) * 8.64e4;
                if (P_rain_diff <= 1.0e-3) break;
            }
        }
    /* applyBoundaryConditions, :447-451; applyTopography (no land: nothing) */
    extrapolate_bc_avg(im, jm, km, P_rain, 1);
    extrapolate_bc_avg(im, jm, km, P_snow, 1);
    extrapolate_bc_avg(im, jm, km, P_graupel, 1);
    free(step);
    or_geom_free(&g);
}

/* the CategoryIceScheme switch, cAtmosphereModel.cpp:581-596 and 1230-1245 */
void or_ice_scheme(int im, int jm, int km, const or_params* p, double* const* f)
{
    switch (p->category_ice_scheme) {
    case 0: or_zero_cat_ice_scheme(im, jm, km, p, f); break;
    case 1: or_one_cat_ice_scheme(im, jm, km, p, f); break;
    case 2: or_two_cat_ice_scheme(im, jm, km, p, f); break;
    case 3: or_three_cat_ice_scheme(im, jm, km, p, f); break;
    default: break;
    }
}
