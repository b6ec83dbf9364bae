/*
 * or_ice.c - TwoCatIceScheme::run (TEST INFRASTRUCTURE ONLY), flat terrain:
 *
 *   initArrays               TwoCatIceScheme.h:126-158
 *   computeColumns           :162-484  (per (j, k) column, top-down, up to iter_prec_end
 *                                        passes until the rain flux at i_check settles)
 *   applyBoundaryConditions  :489-492 -> IceSchemeCommon::extrapolateBC (IceSchemeCommon.h:27-52)
 *   applyTopography          :497-501  (no land: nothing)
 *
 * Within a column the reference keeps N_i, m_i, S_nuc and S_i_dep from one cell to the
 * next where a branch does not assign them; the restatement carries them the same way.
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

/* IceSchemeCommon::extrapolateBC with the phi-seam average, c43 = 1 and c13 = 0 (const
 * int members, cAtmosphereModel.h:158) */
static void extrapolate_bc(int im, int jm, int km, double* P)
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
            const double a = (P[OR_IDX(i, j, 0)] + P[OR_IDX(i, j, km - 1)]) * 0.5;
            P[OR_IDX(i, j, 0)] = a;
            P[OR_IDX(i, j, km - 1)] = a;
        }
}

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
