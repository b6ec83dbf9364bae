/*
 * or_radiation.c - MultiLayerRadiation::run (TEST INFRASTRUCTURE ONLY) and the radiative
 * heating of radiation mode 2 (cAtmosphereModel.cpp:864-879), flat terrain:
 *
 *   surface albedo and the pole-to-equator short-wave parabola   MultiLayerRadiation.h:62-114
 *   per (j, k) column: layer optical depth from the column mass with pressure broadening,
 *   cloud liquid/ice paths, emissivity, the cloud short-wave albedo bump, four upward /
 *   downward grey sweeps that relax each air layer to its radiative equilibrium, a final
 *   sweep, and the linearised surface energy balance                :116-384
 */
#include "or_internal.h"

/* AtomUtils::parabola, lib/Utils.h:158-160 */
static double parabola(double x) { return x * x - 2.0 * x; }

void or_multilayer_radiation(int im, int jm, int km, const or_params* p, double* const* f,
                             double* const* f2)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, 0);
    const int j_max = jm - 1, j_half = j_max / 2;
    double* sw = (double*)malloc(sizeof(double) * jm);
    for (int j = 0; j < jm; j++) sw[j] = p->rad_pole_short;
    const double rad_short_eff = p->rad_pole_short - p->rad_equator_short;
    for (int j = j_half; j >= 0; j--) sw[j] = rad_short_eff * parabola((double)j / (double)j_half) + p->rad_pole_short;
    for (int j = j_max; j > j_half; j--) sw[j] = sw[j_max - j];
    double* up = (double*)malloc(sizeof(double) * im);
    double* dn = (double*)malloc(sizeof(double) * (im + 1));
    double* T = (double*)malloc(sizeof(double) * im);
    const int i_trop = im - 1, i_mount = 0;
    const double t_0 = p->t_0, sigma = p->sigma;
    double* eps3 = f[OF_EPSILON];
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            const size_t q2 = (size_t)j * km + k;
            f2[OF2_ALBEDO][q2] = p->albedo_surface;
            for (int i = i_mount; i <= i_trop; i++) T[i] = f[OF_T][OR_IDX(i, j, k)] * t_0;
            const double p_ref = 1.0e5, inv_g = 1.0 / p->g;
            double lwp_col = 0.0, iwp_col = 0.0;
            for (int i = i_mount; i <= i_trop; i++) {
                const size_t c = OR_IDX(i, j, k);
                double dp_Pa = (i < i_trop) ? (f[OF_P_STAT][c] - f[OF_P_STAT][c + (size_t)jm * km]) * 100.0
                                            : f[OF_P_STAT][c] * 100.0;
                if (dp_Pa < 0.0) dp_Pa = 0.0;
                const double q_v = or_max(0.0, f[OF_C][c]);
                const double q_c = or_max(0.0, f[OF_CO2][c]);
                const double q_b = or_max(0.0, 1.0 - q_v - q_c);
                const double u_col = dp_Pa * inv_g;
                const double broad = f[OF_P_STAT][c] * 100.0 / p_ref;
                const double tau_gas = (p->kappa_H2O * q_v + p->kappa_CO2 * q_c + p->kappa_bg * q_b) * u_col * broad;
                const double k_liq = 0.12, k_ice = 0.055;
                const double dz = (i < i_trop) ? (double)((float)g.height[i + 1] - (float)g.height[i])
                                               : (double)((float)g.height[i] - (float)g.height[i - 1]);
                const double T_i = f[OF_T][c] * t_0;
                const double R_i = or_R_of(q_v, q_c, p->R_bg);
                const double rho_i = (T_i > 0.0) ? (f[OF_P_STAT][c] * 100.0) / (R_i * T_i) : 0.0;
                const double cw_l = or_max(0.0, f[OF_CLOUD][c]);
                const double cw_i = or_max(0.0, f[OF_ICE][c]);
                const double LWP_i = cw_l * rho_i * dz * 1000.0;
                const double IWP_i = cw_i * rho_i * dz * 1000.0;
                lwp_col += LWP_i;
                iwp_col += IWP_i;
                const double tau = tau_gas + k_liq * LWP_i + k_ice * IWP_i;
                eps3[c] = (tau > 700.0) ? 1.0 : (1.0 - exp(-tau));
            }
            f2[OF2_EPSILON][q2] = eps3[OR_IDX(i_mount, j, k)];
            {
                const double alpha_cloud = p->albedo_cloud, f_ice_sw = 0.50, cwp_tau = 100.0;
                const double cwp_sw = lwp_col + f_ice_sw * iwp_col;
                const double tau = cwp_sw / cwp_tau;
                const double refl = tau / (tau + 2.0);
                const double a0 = f2[OF2_ALBEDO][q2];
                if (alpha_cloud > a0) f2[OF2_ALBEDO][q2] = a0 + (alpha_cloud - a0) * refl;
            }
            for (int it = 0; it <= 4; it++) {   /* four relaxation sweeps, then the final one */
                up[i_mount] = sigma * pow(T[i_mount], 4.0);
                for (int i = i_mount + 1; i <= i_trop; i++) {
                    const double e = eps3[OR_IDX(i, j, k)];
                    up[i] = up[i - 1] * (1.0 - e) + e * sigma * pow(T[i], 4.0);
                }
                dn[i_trop + 1] = 0.0;
                for (int i = i_trop; i >= i_mount + 1; i--) {
                    const double e = eps3[OR_IDX(i, j, k)];
                    dn[i] = dn[i + 1] * (1.0 - e) + e * sigma * pow(T[i], 4.0);
                }
                if (it == 4) break;
                for (int i = i_mount + 1; i <= i_trop; i++) {
                    const double emit = 0.5 * (up[i - 1] + dn[i + 1]);
                    T[i] = (emit > 0.0 && or_is_finite(emit)) ? pow(emit / sigma, 0.25) : T[i];
                }
            }
            for (int i = i_mount + 1; i <= i_trop; i++) f[OF_T][OR_IDX(i, j, k)] = T[i] / t_0;
            const double L_down = dn[i_mount + 1];
            const double SW_abs = (1.0 - f2[OF2_ALBEDO][q2]) * sw[j];
            const double T_air1 = T[i_mount + 1];
            const double T_s0 = T[i_mount];
            const double c_H = 15.0;
            const double dsigT4 = 4.0 * sigma * T_s0 * T_s0 * T_s0;
            const double T_s = (SW_abs + p->geothermal_flux + L_down - sigma * pow(T_s0, 4.0)
                               + dsigT4 * T_s0 + c_H * T_air1) / (dsigT4 + c_H);
            f[OF_T][OR_IDX(i_mount, j, k)] = T_s / t_0;
            f[OF_RADIATION][OR_IDX(i_mount, j, k)] = sigma * pow(T_s, 4.0);
            for (int i = i_mount + 1; i <= i_trop; i++) f[OF_RADIATION][OR_IDX(i, j, k)] = up[i];
        }
    free(up); free(dn); free(T); free(sw);
    or_geom_free(&g);
}

void or_radiative_heating(int im, int jm, int km, const or_params* p, double omega_rad,
                          double* const* f, double* const* f2)
{
    const size_t n = (size_t)im * jm * km;
    double* t_backup = (double*)malloc(sizeof(double) * n);
    memcpy(t_backup, f[OF_T], sizeof(double) * n);
    or_multilayer_radiation(im, jm, km, p, f, f2);
    for (size_t q = 0; q < n; q++) f[OF_T][q] = t_backup[q] * (1.0 - omega_rad) + f[OF_T][q] * omega_rad;
    free(t_backup);
}

/* cAtmosphereModel::updateSkinTemperature (cAtmosphereModel.cpp:291-327) with
 * planetaryShortWave (:236-265) and the insolation profile of MultiLayerRadiation.h:102-108 */
double or_update_skin_temperature(int jm, int km, const or_params* p, const double* albedo,
                                  double t_skin, double t_skin_relax)
{
    if (t_skin_relax <= 0.0) return t_skin;
    const int j_max = jm - 1, j_half = j_max / 2;
    double* sw = (double*)malloc(sizeof(double) * jm);
    for (int j = 0; j < jm; j++) sw[j] = p->rad_pole_short;
    const double rad_short_eff = p->rad_pole_short - p->rad_equator_short;
    for (int j = j_half; j >= 0; j--) sw[j] = rad_short_eff * parabola((double)j / (double)j_half) + p->rad_pole_short;
    for (int j = j_max; j > j_half; j--) sw[j] = sw[j_max - j];
    double w_sum = 0.0, abs_w = 0.0, alb_max = 0.0;
    for (int j = 0; j < jm; j++) {
        const double w = cos((j / (double)(jm - 1) - 0.5) * M_PI);
        double alb_k = 0.0;
        for (int k = 0; k < km; k++) alb_k += albedo[(size_t)j * km + k];
        alb_k /= (double)km;
        alb_max = or_max(alb_max, alb_k);
        w_sum += w;
        abs_w += w * (1.0 - alb_k) * sw[j];
    }
    free(sw);
    if (!(w_sum > 0.0) || !(alb_max > 0.0)) return t_skin;
    const double in_mean = abs_w / w_sum + p->geothermal_flux;
    if (!(in_mean > 0.0)) return t_skin;
    const double target = pow(in_mean / p->sigma, 0.25);
    return t_skin + or_min(1.0, t_skin_relax) * (target - t_skin);
}
