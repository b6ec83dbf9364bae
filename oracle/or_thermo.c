/*
 * or_thermo.c - oracle restatement of the water saturation physics and the mixture
 * properties (TEST INFRASTRUCTURE ONLY, see athad_oracle.h).
 *
 * Follows atmosphere/SaturationH2O.h:46-303 and atmosphere/MixtureAtm.h:33-227: the
 * IAPWS-95 saturation line (Wagner & Pruss), the IAPWS-2011 sublimation curve, the
 * Watson latent heat, the exact (non-dilute) saturation mass fraction, the exact
 * derivative factor and the full moist-lapse expression; Shomate heat capacities.
 */
#include "or_internal.h"

/* SaturationH2O.h:68-93 */
double or_saturation_pressure(double T)
{
    if (T >= OR_T_CRIT) return OR_NO_SATURATION;
    if (T <= 0.0) return 0.0;
    const double Tc = OR_T_CRIT;
    const double theta = 1.0 - T / Tc;
    const double a1 = -7.85951783, a2 = 1.84408259, a3 = -11.7866497;
    const double a4 = 22.6807411, a5 = -15.9618719, a6 = 1.80122502;
    const double t15 = theta * sqrt(theta);
    const double t3 = theta * theta * theta;
    const double t35 = t3 * sqrt(theta);
    const double t4 = t3 * theta;
    const double t75 = t4 * t3 * sqrt(theta);
    const double sum = a1 * theta + a2 * t15 + a3 * t3 + a4 * t35 + a5 * t4 + a6 * t75;
    return 220640.0 * exp((Tc / T) * sum);
}

/* SaturationH2O.h:105-120 */
double or_sublimation_pressure(double T)
{
    if (T <= 0.0) return 0.0;
    const double theta = T / 273.16;
    const double a1 = -0.212144006e2, b1 = 0.333333333e-2;
    const double a2 = 0.273203819e2, b2 = 0.120666667e1;
    const double a3 = -0.610598130e1, b3 = 0.170333333e1;
    const double sum = a1 * pow(theta, b1) + a2 * pow(theta, b2) + a3 * pow(theta, b3);
    return 6.11657 * exp(sum / theta);
}

/* SaturationH2O.h:123-127 */
double or_saturation_pressure_auto(double T)
{
    if (T >= OR_T_CRIT) return OR_NO_SATURATION;
    return (T >= 273.16) ? or_saturation_pressure(T) : or_sublimation_pressure(T);
}

/* SaturationH2O.h:138-147 */
double or_latent_heat(double T)
{
    const double Tc = OR_T_CRIT;
    if (T >= Tc) return 0.0;
    return 2.501e6 * pow((Tc - T) / (Tc - 273.15), 0.38);
}

/* SaturationH2O.h:150-154 */
double or_latent_heat_sublimation(double T) { return or_latent_heat(T) + 3.337e5; }

/* SaturationH2O.h:207-210 */
double or_latent_heat_auto(double T)
{
    return (T >= 273.16) ? or_latent_heat(T) : or_latent_heat_sublimation(T);
}

/* SaturationH2O.h:168-178 */
double or_saturation_mass_fraction(double E, double p, double M_other)
{
    if (E == OR_NO_SATURATION) return 1.0;
    if (!(p > 0.0)) return 0.0;
    if (E >= p) return 1.0;
    const double x = E / p;
    const double num = x * OR_M_H2O;
    const double den = num + (1.0 - x) * M_other;
    return (den > 0.0) ? num / den : 1.0;
}

/* SaturationH2O.h:298-301 */
double or_saturation_mass_fraction_at(double T, double p, double M_other)
{
    return or_saturation_mass_fraction(or_saturation_pressure_auto(T), p, M_other);
}

/* SaturationH2O.h:189-202 */
double or_dew_point(double e)
{
    if (!(e > 0.0)) return 0.0;
    if (e >= 220640.0) return OR_T_CRIT;
    double lo = 150.0, hi = OR_T_CRIT;
    if (or_saturation_pressure_auto(lo) >= e) return lo;
    for (int it = 0; it < 60; it++) {
        const double mid = 0.5 * (lo + hi);
        if (or_saturation_pressure_auto(mid) < e) lo = mid; else hi = mid;
    }
    return 0.5 * (lo + hi);
}

/* SaturationH2O.h:230-239 */
double or_sat_deriv_factor_at(double E, double p, double M_other)
{
    if (E == OR_NO_SATURATION || !(p > 0.0) || E >= p) return 0.0;
    const double x = E / p;
    const double den = x * OR_M_H2O + (1.0 - x) * M_other;
    if (!(den > 0.0)) return 0.0;
    return x * OR_M_H2O * M_other / (den * den);
}

/* SaturationH2O.h:251-255 */
double or_dqsat_dT_from(double E, double L, double T, double p, double M_other)
{
    if (!(T > 0.0)) return 0.0;
    return or_sat_deriv_factor_at(E, p, M_other) * L / (OR_R_H2O * T * T);
}

/* SaturationH2O.h:257-260 */
double or_dqsat_dT(double T, double p, double M_other)
{
    return or_dqsat_dT_from(or_saturation_pressure_auto(T), or_latent_heat_auto(T), T, p,
                            M_other);
}

/* SaturationH2O.h:280-293 */
double or_moist_lapse(double T, double p, double M_other, double cp, double R_mix, double g)
{
    if (!(cp > 0.0) || !(T > 0.0) || !(R_mix > 0.0)) return 0.0;
    const double A = or_sat_deriv_factor_at(or_saturation_pressure_auto(T), p, M_other);
    if (!(A > 0.0)) return g / cp;
    const double L = or_latent_heat_auto(T);
    const double num = 1.0 + L * A / (R_mix * T);
    const double den = cp + L * L * A / (OR_R_H2O * T * T);
    return (den > 0.0) ? g * num / den : g / cp;
}

/* MixtureAtm.h:123-128 */
static double shomate(double T, double A, double B, double Cc, double D, double E)
{
    const double t = or_min(or_max(T, 298.0), 2000.0) * 1.0e-3;
    const double t2 = t * t;
    return A + B * t + Cc * t2 + D * t2 * t + E / t2;
}
static double cp_H2O(double T) { return shomate(T, 30.09200, 6.832514, 6.793435, -2.534480, 0.082139) / OR_M_H2O; }
static double cp_CO2(double T) { return shomate(T, 24.99735, 55.18696, -33.69137, 7.948387, -0.136638) / OR_M_CO2; }
static double cp_bg(double T, double M_b) { return shomate(T, 28.98641, 1.853978, -9.647459, 16.63537, 0.000117) / M_b; }

/* MixtureAtm.h:152-162 */
static void split(double c, double co2, double* q_v, double* q_c, double* q_b)
{
    *q_v = or_min(or_max(c, 0.0), 1.0);
    *q_c = or_min(or_max(co2, 0.0), 1.0);
    const double sum = *q_v + *q_c;
    if (sum > 1.0) { *q_v /= sum; *q_c /= sum; }
    *q_b = or_max(0.0, 1.0 - *q_v - *q_c);
}

/* MixtureAtm.h:165-170 */
double or_R_of(double c, double co2, double R_b)
{
    double q_v, q_c, q_b;
    split(c, co2, &q_v, &q_c, &q_b);
    return q_v * OR_R_H2O + q_c * OR_R_CO2 + q_b * R_b;
}

/* MixtureAtm.h:173-178 */
double or_cp_of(double c, double co2, double T, double M_b)
{
    double q_v, q_c, q_b;
    split(c, co2, &q_v, &q_c, &q_b);
    return q_v * cp_H2O(T) + q_c * cp_CO2(T) + q_b * cp_bg(T, M_b);
}

/* MixtureAtm.h:209-217 */
double or_M_nonwater(double c, double co2, double M_b)
{
    double q_v, q_c, q_b;
    split(c, co2, &q_v, &q_c, &q_b);
    const double sum = q_c + q_b;
    if (!(sum > 0.0)) return M_b;
    const double inv = (q_c / sum) / OR_M_CO2 + (q_b / sum) / M_b;
    return (inv > 0.0) ? 1.0 / inv : M_b;
}

/* MixtureAtm.h:181-187 (M_of) and :220-225 (x_H2O_of): the water vapour mole fraction */
double or_x_H2O_of(double c, double co2, double M_b)
{
    double q_v, q_c, q_b;
    split(c, co2, &q_v, &q_c, &q_b);
    const double inv = q_v / OR_M_H2O + q_c / OR_M_CO2 + q_b / M_b;
    const double M = (inv > 0.0) ? 1.0 / inv : M_b;
    return q_v * M / OR_M_H2O;
}

/* MixtureAtm.h:82-109.  x8 = H2O, CO2, N2, CH4, NH3, H2, CO, SO2 mole fractions;
 * out7 = M_mean, R_mix, q_H2O, q_CO2, q_bg, M_bg, R_bg. */
void or_resolve(const double* x, double* out)
{
    const double m_H2O = x[0] * OR_M_H2O;
    const double m_CO2 = x[1] * OR_M_CO2;
    const double m_bg = x[2] * 0.028014 + x[3] * 0.016043 + x[4] * 0.017031
                      + x[5] * 0.002016 + x[6] * 0.028010 + x[7] * 0.064066;
    const double M_mean = m_H2O + m_CO2 + m_bg;
    out[0] = M_mean;
    out[1] = OR_R_STAR / M_mean;
    out[2] = m_H2O / M_mean;
    out[3] = m_CO2 / M_mean;
    out[4] = m_bg / M_mean;
    const double x_bg = x[2] + x[3] + x[4] + x[5] + x[6] + x[7];
    out[5] = (x_bg > 0.0) ? (m_bg / x_bg) : 0.028014;
    out[6] = OR_R_STAR / out[5];
}
