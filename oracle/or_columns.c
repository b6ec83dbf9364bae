/*
 * or_columns.c - oracle restatement of the per-cell and per-column moist physics:
 * saturation adjustment and the column thermodynamics (densities).
 * TEST INFRASTRUCTURE ONLY, see athad_oracle.h.
 */
#include "or_internal.h"

/* IceSchemeCommon::evaporateWhereImpossible, IceSchemeCommon.h:121-190 */
void or_evaporate_where_impossible(const or_params* p, double* const* f, size_t c, double t_u)
{
    const double q_cond = or_max(0.0, f[OF_CLOUD][c]) + or_max(0.0, f[OF_ICE][c])
                        + or_max(0.0, f[OF_GR][c]);
    if (q_cond > 0.0) {
        const double c_max = or_max(0.0, 1.0 - f[OF_CO2][c]);
        const double c_new = or_min(c_max, f[OF_C][c] + q_cond);
        const double q_used = or_max(0.0, c_new - f[OF_C][c]);
        f[OF_C][c] = c_new;
        f[OF_CLOUD][c] = 0.0;
        f[OF_ICE][c] = 0.0;
        f[OF_GR][c] = 0.0;
        if (t_u < OR_T_CRIT) {
            const double cp_loc = or_cp_of(f[OF_C][c], f[OF_CO2][c], t_u, p->M_bg);
            if (cp_loc > 0.0) {
                double T_new = t_u - or_latent_heat(t_u) * q_used / cp_loc;
                if (T_new < 1.0) T_new = 1.0;
                f[OF_T][c] = T_new / p->t_0;
            }
        }
    }
    {
        const double v_rain = 1.6, v_snow = 0.96, v_graupel = 2.0;
        const double rho = or_max(1.0e-6, f[OF_R_HUMID][c]);
        const double q_p = or_max(0.0, f[OF_P_RAIN][c]) / (v_rain * rho)
                         + or_max(0.0, f[OF_P_SNOW][c]) / (v_snow * rho)
                         + or_max(0.0, f[OF_P_GRAUPEL][c]) / (v_graupel * rho);
        if (q_p > 0.0) {
            const double c_max = or_max(0.0, 1.0 - f[OF_CO2][c]);
            f[OF_C][c] = or_min(c_max, f[OF_C][c] + q_p);
        }
    }
    f[OF_P_RAIN][c] = 0.0; f[OF_P_SNOW][c] = 0.0; f[OF_P_GRAUPEL][c] = 0.0;
    f[OF_PRECIPITATION][c] = 0.0;
    f[OF_S_V][c] = 0.0; f[OF_S_C][c] = 0.0; f[OF_S_I][c] = 0.0; f[OF_S_R][c] = 0.0;
    f[OF_S_S][c] = 0.0; f[OF_S_G][c] = 0.0; f[OF_S_C_C][c] = 0.0;
}

/* SaturationAdjustment::run = computeSteps, adjustSaturation, applyTopography (identity
 * with flat terrain), clampAndFade: SaturationAdjustment.h:25-459. */
int or_column_geometry(int im, int jm, int km, const or_params* p, int compat, double* height,
                       double* step_f)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, compat);
    for (int i = 0; i < im; i++) {
        height[i] = g.height[i];
        /* computeSteps (SaturationAdjustment.h:56-60), as or_saturation_adjust forms it */
        const float h1 = (i + 1 <= im - 1) ? (float)g.height[i + 1] : -1.0f;
        const float h0 = (float)g.height[i];
        step_f[i] = (double)(float)(h1 - h0);
    }
    or_geom_free(&g);
    return 0;
}

void or_saturation_adjust(int im, int jm, int km, const or_params* p, int compat,
                          double* const* f, int64_t* counters)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, compat);
    const double fade_K = 5.0;
    const int iter_prec_end = 20;
    /* computeSteps (:56-60): a float difference of float layer heights */
    double* step = (double*)malloc(sizeof(double) * im);
    for (int i = 0; i < im; i++) {
        const float h1 = (i + 1 <= im - 1) ? (float)g.height[i + 1] : -1.0f;
        const float h0 = (float)g.height[i];
        step[i] = (double)(float)(h1 - h0);
    }
    const double inv_t_0 = 1.0 / p->t_0;
    const double t_range_inv = 1.0 / (p->t_0 - p->t_00);
    for (int j = 0; j < jm; j++)              /* :75-78 */
        for (int k = 0; k < km; k++) f[OF_S_C_C][OR_IDX(0, j, k)] = 0.0;

    for (int i = 1; i < im - 1; i++)          /* adjustSaturation, :90-286 */
        for (int j = 0; j < jm; j++) {
            const double dt_dim = step[i] / 1.6;
            for (int k = 0; k < km; k++) {
                const size_t c = OR_IDX(i, j, k);
                f[OF_S_C_C][c] = 0.0;
                const double q_v_old = or_max(0.0, f[OF_C][c]);
                const double q_c_old = or_max(0.0, f[OF_CLOUD][c]);
                const double q_i_old = or_max(0.0, f[OF_ICE][c]);
                double T = f[OF_T][c] * p->t_0;
                if (T >= OR_T_CRIT) continue;
                const double p_local = f[OF_P_STAT][c];
                const double co2 = f[OF_CO2][c];
                const double M_other = or_M_nonwater(f[OF_C][c], co2, p->M_bg);
                const double E_sat0 = or_saturation_pressure_auto(T);
                const double q_sat0 = or_saturation_mass_fraction(E_sat0, p_local, M_other);
                const double alpha_entry = 1.0 / (1.0 + exp(-(T - p->t_00) / fade_K));
                if ((q_v_old > q_sat0 && alpha_entry > 0.01) ||
                    (q_v_old < q_sat0 && (q_c_old > 1e-12 || q_i_old > 1e-12))) {
                    double q_v_b = q_v_old, q_c_b = q_c_old, q_i_b = q_i_old;
                    double q_v_hyp = q_v_b;
                    const double T_original = f[OF_T][c] * p->t_0;
                    for (int iter = 1; iter <= iter_prec_end; iter++) {
                        const double CND = or_max(0.0, or_min(1.0, (T - p->t_00) * t_range_inv));
                        const double DEP = 1.0 - CND;
                        double d_q_v = q_v_hyp - q_v_b;
                        if (d_q_v > 0) {
                            const double max_evap = q_c_b + q_i_b;
                            if (d_q_v > max_evap) d_q_v = max_evap;
                        }
                        const double d_cnd = d_q_v * CND;
                        const double d_dep = d_q_v * DEP;
                        q_v_b += d_q_v;
                        q_c_b = or_max(0.0, q_c_b - d_cnd);
                        q_i_b = or_max(0.0, q_i_b - d_dep);
                        const double cp_loc = or_cp_of(q_v_b, co2, T, p->M_bg);
                        T -= (or_latent_heat(T) * d_cnd
                              + or_latent_heat_sublimation(T) * d_dep) / cp_loc;
                        const double E_sat = or_saturation_pressure(T);
                        const double E_Ice = or_sublimation_pressure(T);
                        const double q_sat = or_saturation_mass_fraction(E_sat, p_local, M_other);
                        const double q_Ice = or_saturation_mass_fraction(E_Ice, p_local, M_other);
                        const double q_sum = q_c_b + q_i_b;
                        const double q_v_target = (q_sum > 1e-12)
                            ? (q_c_b * q_sat + q_i_b * q_Ice) / q_sum
                            : ((T >= p->t_0) ? q_sat : q_Ice);
                        const double cp_g = or_cp_of(q_v_b, co2, T, p->M_bg);
                        const double L_cnd = or_latent_heat(T);
                        const double L_dep = or_latent_heat_sublimation(T);
                        const double Gain = CND * (L_cnd / cp_g)
                                          * or_dqsat_dT_from(E_sat, L_cnd, T, p_local, M_other)
                                          + DEP * (L_dep / cp_g)
                                          * or_dqsat_dT_from(E_Ice, L_dep, T, p_local, M_other);
                        const double omega = 1.0 / (1.0 + Gain);
                        q_v_hyp = q_v_b + omega * (q_v_target - q_v_b);
                        if (fabs(q_v_b / q_v_hyp - 1.0) <= 1.0e-6) break;
                    }
                    q_c_b = or_max(0.0, q_c_b);
                    q_i_b = or_max(0.0, q_i_b);
                    if (T > OR_T_CRIT) T = OR_T_CRIT;
                    if (!isnan(T) && !isnan(q_v_b)) {
                        f[OF_S_C_C][c] = alpha_entry * (q_c_b - q_c_old) / dt_dim;
                        f[OF_C][c] = q_v_old + alpha_entry * (q_v_b - q_v_old);
                        f[OF_CLOUD][c] = q_c_old + alpha_entry * (q_c_b - q_c_old);
                        f[OF_ICE][c] = q_i_old + alpha_entry * (q_i_b - q_i_old);
                        f[OF_T][c] = (T_original + alpha_entry * (T - T_original)) * inv_t_0;
                    }
                    if (T < p->t_00) {
                        f[OF_CLOUD][c] = 0.0;
                        f[OF_ICE][c] = 0.0;
                    }
                }
            }
        }

    /* clampAndFade, :303-459 */
    int64_t n_ceiling = 0;
    const double T_max = p->t_max_phys, cloud_cap = p->cloud_cap;
    const size_t n = (size_t)im * jm * km;
    for (size_t c = 0; c < n; c++) {
        if (f[OF_C][c] < 0.0) f[OF_C][c] = 0.0;
        if (f[OF_CLOUD][c] < 0.0) f[OF_CLOUD][c] = 0.0;
        if (f[OF_ICE][c] < 0.0) f[OF_ICE][c] = 0.0;
        const double c_max = or_max(0.0, 1.0 - f[OF_CO2][c]);
        if (f[OF_C][c] > c_max) { f[OF_C][c] = c_max; n_ceiling++; }
        double T_dim = f[OF_T][c] * p->t_0;
        if (T_dim > T_max) { T_dim = T_max; f[OF_T][c] = T_max * inv_t_0; }
        {
            const double M_o = or_M_nonwater(f[OF_C][c], f[OF_CO2][c], p->M_bg);
            const double q_s = or_saturation_mass_fraction_at(T_dim, f[OF_P_STAT][c], M_o);
            if (T_dim >= OR_T_CRIT || q_s >= 1.0) {
                or_evaporate_where_impossible(p, f, c, T_dim);
                continue;
            }
        }
        const double p_local = f[OF_P_STAT][c];
        const double M_other = or_M_nonwater(f[OF_C][c], f[OF_CO2][c], p->M_bg);
        const double E_sat = or_saturation_pressure_auto(T_dim);
        const double q_sat = or_saturation_mass_fraction(E_sat, p_local, M_other);
        if (f[OF_C][c] > q_sat) {
            const double excess = f[OF_C][c] - q_sat;
            f[OF_C][c] = q_sat;
            if (T_dim >= p->t_00) {
                f[OF_CLOUD][c] += excess;
                T_dim += or_latent_heat(T_dim) * excess
                       / or_cp_of(f[OF_C][c], f[OF_CO2][c], T_dim, p->M_bg);
            } else {
                f[OF_ICE][c] += excess;
                T_dim += or_latent_heat_sublimation(T_dim) * excess
                       / or_cp_of(f[OF_C][c], f[OF_CO2][c], T_dim, p->M_bg);
            }
            if (T_dim > T_max) T_dim = T_max;
            f[OF_T][c] = T_dim * inv_t_0;
        }
        if (f[OF_CLOUD][c] > cloud_cap) f[OF_CLOUD][c] = cloud_cap;
        if (f[OF_ICE][c] > cloud_cap) f[OF_ICE][c] = cloud_cap;
        const double alpha = 1.0 / (1.0 + exp(-(T_dim - p->t_00) / fade_K));
        f[OF_C][c] *= alpha;
        f[OF_CLOUD][c] *= alpha;
        f[OF_ICE][c] *= alpha;
    }
    if (counters) counters[0] = n_ceiling;
    free(step);
    or_geom_free(&g);
}

/* Row sum in the fixed order of a 32-lane strided partial sum reduced by xor butterfly
 * (the order the device reduction uses), over the positive entries of a row. */
static void row_pos_sum_32(const double* row, int km, double* sum, double* cnt)
{
    double ps[32], pc[32];
    for (int l = 0; l < 32; l++) {
        double s = 0.0, q = 0.0;
        for (int k = l; k < km; k += 32) {
            const double r = row[k];
            if (r > 0.0) { s += r; q += 1.0; }
        }
        ps[l] = s; pc[l] = q;
    }
    for (int off = 16; off >= 1; off >>= 1) {
        double ns[32], nc[32];
        for (int l = 0; l < 32; l++) { ns[l] = ps[l] + ps[l ^ off]; nc[l] = pc[l] + pc[l ^ off]; }
        memcpy(ps, ns, sizeof ps); memcpy(pc, nc, sizeof pc);
    }
    *sum = ps[0]; *cnt = pc[0];
}

/* ThermoAtm::densities, ThermoAtm.h:1436-1666 (flat terrain: i_topography == 0). */
void or_densities(int im, int jm, int km, const or_params* p, int compat,
                  int set_water_profile, double* const* f, double* const* f2,
                  double* const* prof)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, compat);
    const double R_mix = p->R_mix;
    const double p_sl_factor = 1e-2 * p->r_air * R_mix;
    const double M_bg = p->M_bg, R_bg = p->R_bg;
    const double* h = g.height;
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            double T_prev = or_max(180.0, f[OF_T][OR_IDX(0, j, k)] * p->t_0);
            double p_prev = p_sl_factor * T_prev;
            double q_sat_min = 1.0;
            for (int i = 0; i < im; i++) {
                const size_t c = OR_IDX(i, j, k);
                const double q_v = f[OF_C][c];
                const double q_c = f[OF_CO2][c];
                const double R_loc = or_R_of(q_v, q_c, R_bg);
                double T_i, p_i;
                if (i == 0) {
                    T_i = T_prev;
                    p_i = p_prev;
                } else {
                    const double dz = h[i] - h[i - 1];
                    const size_t cm = OR_IDX(i - 1, j, k);
                    const double q_v_p = f[OF_C][cm];
                    const double q_c_p = f[OF_CO2][cm];
                    const double cp_loc = or_cp_of(q_v_p, q_c_p, T_prev, M_bg);
                    const double M_nw = or_M_nonwater(q_v_p, q_c_p, M_bg);
                    const double q_s = or_saturation_mass_fraction_at(T_prev, p_prev, M_nw);
                    const double gamma = (q_v_p >= 0.99 * q_s)
                        ? or_moist_lapse(T_prev, p_prev, M_nw, cp_loc, R_loc, p->g)
                        : p->g / cp_loc;
                    const double T_ad = T_prev - gamma * dz;
                    T_i = or_max(p->t_skin, T_ad);
                    const double T_mean = 0.5 * (T_prev + T_i);
                    p_i = p_prev * exp(-p->g * dz / (R_loc * T_mean));
                }
                f[OF_T][c] = T_i / p->t_0;
                f[OF_P_STAT][c] = p_i;
                if (set_water_profile && i > 0) {
                    const double M_nw_i = or_M_nonwater(q_v, q_c, M_bg);
                    const double q_s_i = or_saturation_mass_fraction_at(T_i, p_i, M_nw_i);
                    if (q_s_i < q_sat_min) q_sat_min = q_s_i;
                    f[OF_C][c] = or_max(q_sat_min, p->c_h2o_dry_top);
                }
                const double water_factor = or_max(0.5, 1.0 - f[OF_CLOUD][c] - f[OF_ICE][c]);
                f[OF_R_HUMID][c] = 1e2 * p_i / (R_loc * T_i * water_factor);
                const double R_dry_loc = or_R_of(0.0, q_c, R_bg);
                f[OF_R_DRY][c] = 1e2 * p_i / (R_dry_loc * T_i);
                T_prev = T_i;
                p_prev = p_i;
            }
            const size_t cj = (size_t)j * km + k;
            if (f2 && f2[OF2_T_TOP_INIT]) f2[OF2_T_TOP_INIT][cj] = f[OF_T][OR_IDX(im - 1, j, k)];
            if (f2 && f2[OF2_P_STAT_LANDSCAPE]) f2[OF2_P_STAT_LANDSCAPE][cj] = f[OF_P_STAT][OR_IDX(0, j, k)];
        }

    /* rho_bar and d ln rho_bar / d rad.z, ThermoAtm.h:1629-1660 */
    double* rho_base = prof[OFP_RHO_BASE];
    double* dlnrho = prof[OFP_DLNRHO_DR];
    double* lnrho = (double*)calloc(im, sizeof(double));
    for (int i = 0; i < im; i++) {
        double num = 0.0, den = 0.0;
        if (compat) {
            for (int j = 0; j < jm; j++) {
                const double coslat = cos((j / (double)(jm - 1) - 0.5) * M_PI);
                for (int k = 0; k < km; k++) {
                    const double rho = f[OF_R_HUMID][OR_IDX(i, j, k)];
                    if (!(rho > 0.0)) continue;
                    num += coslat * rho;
                    den += coslat;
                }
            }
        } else {
            const int half = jm / 2;
            for (int j = 0; j <= half; j++) {
                const int jr = jm - 1 - j;
                if (jr < j) break;
                const double coslat = cos((j / (double)(jm - 1) - 0.5) * M_PI);
                double s0, c0, s1, c1;
                row_pos_sum_32(&f[OF_R_HUMID][OR_IDX(i, j, 0)], km, &s0, &c0);
                if (jr != j) {
                    row_pos_sum_32(&f[OF_R_HUMID][OR_IDX(i, jr, 0)], km, &s1, &c1);
                    num += coslat * (s0 + s1);
                    den += coslat * (c0 + c1);
                } else {
                    num += coslat * s0;
                    den += coslat * c0;
                }
            }
        }
        rho_base[i] = (den > 0.0) ? num / den : 0.0;
        lnrho[i] = (rho_base[i] > 0.0) ? log(rho_base[i]) : 0.0;
    }
    const double inv_2dr = 1.0 / (2.0 * g.dr), inv_dr = 1.0 / g.dr;
    for (int i = 0; i < im; i++) dlnrho[i] = 0.0;
    for (int i = 1; i < im - 1; i++) dlnrho[i] = (lnrho[i + 1] - lnrho[i - 1]) * inv_2dr;
    if (im > 1) {
        dlnrho[0] = (lnrho[1] - lnrho[0]) * inv_dr;
        dlnrho[im - 1] = (lnrho[im - 1] - lnrho[im - 2]) * inv_dr;
    }
    free(lnrho);
    or_geom_free(&g);
}
