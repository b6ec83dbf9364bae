/*
 * or_surface.c - the surface-flux modules of the moist iteration (TEST INFRASTRUCTURE ONLY):
 *
 *   or_water_vapour_evaporation   ThermoAtm::waterVapourEvaporation (ThermoAtm.h:115-398)
 *   or_latent_sensible_heat       ThermoAtm::latentSensibleHeat (ThermoAtm.h:36-112)
 *
 * Flat terrain (no land cells).
 */
#include "or_internal.h"

/* AtomUtils::C_Dalton (lib/Utils.cpp:157-172) at the surface cell c */
static double c_dalton(const or_params* p, double* const* f, size_t c)
{
    const double v_max = 10.0, c_Dalton_max = 0.053;
    const double u = f[OF_U][c], v = f[OF_V][c], w = f[OF_W][c];
    const double vel_magnitude = sqrt((u * u + v * v + w * w) / 3.0) * p->u_0;
    return p->coeff_Dalton * sqrt(c_Dalton_max * c_Dalton_max * vel_magnitude / v_max);
}

/* The sea surface is a saturation boundary (ThermoAtm.h:186-262): the block runs for every
 * column below the critical temperature and ends with `continue`, so the Dalton / Meyer /
 * Rohwer branch after it (:264-362) is never reached. */
void or_water_vapour_evaporation(int im, int jm, int km, const or_params* p, double* const* f,
                                 double* const* f2)
{
    const double hPa_to_mmHg = 0.750062, K_Meyer = 11.0;
    const int n_spread = 3;
    const double r = exp(-1.0);
    const double w_norm = (1.0 - r) / (1.0 - pow(r, n_spread + 1));
    double* c = f[OF_C];
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            const size_t c0 = OR_IDX(0, j, k);
            const size_t q2 = (size_t)j * km + k;
            if (f[OF_T][c0] * p->t_0 >= OR_T_CRIT) {
                f2[OF2_EVAPORATION_DALTON][q2] = 0.0;
                f2[OF2_EVAPORATION_MEYER][q2] = 0.0;
                f2[OF2_EVAPORATION_ROHWER][q2] = 0.0;
                f2[OF2_EVAPORATION][q2] = 0.0;
                continue;
            }
            const double T_s = or_max(180.0, f[OF_T][c0] * p->t_0);
            const double p_s = f[OF_P_STAT][c0];
            const double M_nw = or_M_nonwater(c[c0], f[OF_CO2][c0], p->M_bg);
            const double E_s = or_saturation_pressure_auto(T_s);
            const double q_sea = or_saturation_mass_fraction(E_s, p_s, M_nw);
            const double u = f[OF_U][c0], v = f[OF_V][c0], w = f[OF_W][c0];
            const double vel = sqrt((u * u + v * v + w * w) / 3.0) * p->u_0;
            const double u_kmh_d = vel * 3.6;
            const double e_air = (q_sea > 0.0 && q_sea < 1.0)
                ? c[c0] * p_s * M_nw / (c[c0] * M_nw + (1.0 - c[c0]) * OR_M_H2O)
                : 0.0;
            const double sd_d = or_max(0.0, E_s - e_air);
            f2[OF2_EVAPORATION_DALTON][q2] = c_dalton(p, f, c0) * 24.0 * sd_d;
            f2[OF2_EVAPORATION_MEYER][q2] = K_Meyer * hPa_to_mmHg * (1.0 + u_kmh_d / 16.0) / 30.0 * sd_d;
            f2[OF2_EVAPORATION_ROHWER][q2] = 0.771 * (1.465 - 0.000732 * p_s * hPa_to_mmHg)
                                          * (0.44 + 0.0733 * u_kmh_d) * hPa_to_mmHg * sd_d;
            f2[OF2_EVAPORATION][q2] = f2[OF2_EVAPORATION_DALTON][q2];
            const double c_fix = c[c0];
            f2[OF2_C_FIX][q2] = c_fix;
            c[c0] = c_fix + (q_sea - c_fix) * w_norm;
            for (int i = 1; i <= n_spread && i < im; i++) {
                const size_t ci = OR_IDX(i, j, k);
                const double weight = pow(r, i) * w_norm;
                const double T_i = or_max(180.0, f[OF_T][ci] * p->t_0);
                const double p_i = f[OF_P_STAT][ci];
                const double M_nw_i = or_M_nonwater(c[ci], f[OF_CO2][ci], p->M_bg);
                const double q_s_i = or_saturation_mass_fraction_at(T_i, p_i, M_nw_i);
                c[ci] = or_min(c[ci] + (q_sea - c_fix) * weight, q_s_i);
            }
        }
}

/* compat = 1: sin(theta_j) of the running-sum theta, as the reference forms it; 0: the
 * mirror-exact table (sin theta_j == sin theta_{jm-1-j}), which makes Q_Sensible exactly
 * north-south symmetric. */
void or_latent_sensible_heat(int im, int jm, int km, const or_params* p, int compat, double* const* f)
{
    or_geom g;
    or_geom_init(&g, im, jm, km, p, compat);
    const double inv_2dr = 1.0 / (2.0 * g.dr);
    const double inv_2dthe = 1.0 / (2.0 * g.dthe);
    const double inv_2dphi = 1.0 / (2.0 * g.dphi);
    const double inv_sqrt3 = 1.0 / sqrt(3.0);
    const double* t = f[OF_T];
    for (int j = 0; j < jm; j++)
        for (int k = 0; k < km; k++) {
            f[OF_Q_LATENT][OR_IDX(0, j, k)] = 0.0;
            f[OF_Q_SENSIBLE][OR_IDX(0, j, k)] = 0.0;
        }
    const size_t sI = (size_t)jm * km, sJ = (size_t)km;
    for (int j = 1; j < jm - 1; j++) {
        double sinthe = g.sin_w[j];
        if (fabs(sinthe) < 1e-10) sinthe = 1e-10;
        for (int k = 1; k < km - 1; k++)
            for (int i = 1; i < im - 1; i++) {
                const size_t c = OR_IDX(i, j, k);
                const double rm = g.rad[i];
                const double exp_rm = 1.0 / (rm + 1.0);
                const double inv_rm = 1.0 / rm;
                const double inv_rmsinthe = 1.0 / (rm * sinthe);
                const double dtdr = (t[c + sI] - t[c - sI]) * inv_2dr * exp_rm;
                const double dtdthe = (t[c + sJ] - t[c - sJ]) * inv_2dthe * inv_rm;
                const double dtdphi = (t[c + 1] - t[c - 1]) * inv_2dphi * inv_rmsinthe;
                f[OF_Q_SENSIBLE][c] = p->cp_l * p->t_0 * inv_sqrt3
                                    * sqrt(dtdr * dtdr + dtdthe * dtdthe + dtdphi * dtdphi);
            }
    }
    or_geom_free(&g);
}
