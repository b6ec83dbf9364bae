// thermo.cuh - water saturation physics and mixture properties for the device.
//
// Restates atmosphere/SaturationH2O.h:46-303 (IAPWS-95 saturation line after Wagner &
// Pruss, IAPWS-2011 sublimation curve, Watson latent heat, the exact non-dilute saturation
// mass fraction, the exact derivative factor and the full moist-lapse expression) and
// atmosphere/MixtureAtm.h:33-227 (Shomate heat capacities, mass-weighted R and cp).  FP64
// throughout; the transcendentals are CUDA's own exp/log/sqrt.  Host+device so the host
// can build tables with the same code.
#pragma once

#include <cmath>
#include "common.cuh"

namespace athad {
namespace thermo {

constexpr double T_CRIT = 647.096;          // MixtureAtm.h:40
constexpr double NO_SATURATION = -1.0;      // SaturationH2O.h:50
constexpr double T_TRIPLE = 273.16;
constexpr double R_STAR = 8.314462618;
constexpr double M_H2O = 0.018015;
constexpr double M_CO2 = 0.044010;
constexpr double R_H2O = R_STAR / M_H2O;
constexpr double R_CO2 = R_STAR / M_CO2;

// Wagner & Pruss saturation line (SaturationH2O.h:68-93)
ATHAD_HD double saturation_pressure(double T)
{
    if (T >= T_CRIT) return NO_SATURATION;
    if (T <= 0.0) return 0.0;
    const double theta = 1.0 - T / T_CRIT;
    const double sq = sqrt(theta);
    const double t15 = theta * sq;
    const double t3 = theta * theta * theta;
    const double t35 = t3 * sq;
    const double t4 = t3 * theta;
    const double t75 = t4 * t3 * sq;
    const double sum = -7.85951783 * theta + 1.84408259 * t15 + -11.7866497 * t3
                     + 22.6807411 * t35 + -15.9618719 * t4 + 1.80122502 * t75;
    return 220640.0 * exp((T_CRIT / T) * sum);
}

// IAPWS (2011) sublimation curve (SaturationH2O.h:105-120).  The three powers of theta
// share one logarithm: theta^a = exp(a ln theta), within two ulp of pow(theta, a) for the
// theta of the atmosphere (0.5..2.4), at a third of the cost of three pow calls.
ATHAD_HD double sublimation_pressure(double T)
{
    if (T <= 0.0) return 0.0;
    const double theta = T / T_TRIPLE;
    const double lt = log(theta);
    const double sum = -0.212144006e2 * exp(0.333333333e-2 * lt)
                     + 0.273203819e2 * exp(0.120666667e1 * lt)
                     + -0.610598130e1 * exp(0.170333333e1 * lt);
    return 6.11657 * exp(sum / theta);
}

ATHAD_HD double saturation_pressure_auto(double T)   // SaturationH2O.h:123-127
{
    if (T >= T_CRIT) return NO_SATURATION;
    return (T >= T_TRIPLE) ? saturation_pressure(T) : sublimation_pressure(T);
}

// Watson, SaturationH2O.h:138-147; x^0.38 as exp(0.38 ln x) (within two ulp of pow)
ATHAD_HD double latent_heat(double T)
{
    if (T >= T_CRIT) return 0.0;
    const double x = (T_CRIT - T) / (T_CRIT - 273.15);
    return (x > 0.0) ? 2.501e6 * exp(0.38 * log(x)) : 0.0;
}
ATHAD_HD double latent_heat_sublimation(double T) { return latent_heat(T) + 3.337e5; }
ATHAD_HD double latent_heat_auto(double T)
{
    return (T >= T_TRIPLE) ? latent_heat(T) : latent_heat_sublimation(T);
}

// exact mass fraction (SaturationH2O.h:168-178)
ATHAD_HD double saturation_mass_fraction(double E, double p, double M_other)
{
    if (E == NO_SATURATION) return 1.0;
    if (!(p > 0.0)) return 0.0;
    if (E >= p) return 1.0;
    const double x = E / p;
    const double num = x * M_H2O;
    const double den = num + (1.0 - x) * M_other;
    return (den > 0.0) ? num / den : 1.0;
}
ATHAD_HD double saturation_mass_fraction_at(double T, double p, double M_other)
{
    return saturation_mass_fraction(saturation_pressure_auto(T), p, M_other);
}

ATHAD_HD double sat_deriv_factor_at(double E, double p, double M_other)   // :230-239
{
    if (E == NO_SATURATION || !(p > 0.0) || E >= p) return 0.0;
    const double x = E / p;
    const double den = x * M_H2O + (1.0 - x) * M_other;
    if (!(den > 0.0)) return 0.0;
    return x * M_H2O * M_other / (den * den);
}

ATHAD_HD double dqsat_dT_from(double E, double L, double T, double p, double M_other)  // :251-255
{
    if (!(T > 0.0)) return 0.0;
    return sat_deriv_factor_at(E, p, M_other) * L / (R_H2O * T * T);
}

ATHAD_HD double dqsat_dT(double T, double p, double M_other)   // :257-260
{
    return dqsat_dT_from(saturation_pressure_auto(T), latent_heat_auto(T), T, p, M_other);
}

// full moist lapse rate (SaturationH2O.h:280-293), with E = saturation_pressure_auto(T)
// when the caller has formed it already
ATHAD_HD double moist_lapse_E(double T, double E, double p, double M_other, double cp, double R_mix, double g)
{
    if (!(cp > 0.0) || !(T > 0.0) || !(R_mix > 0.0)) return 0.0;
    const double A = sat_deriv_factor_at(E, p, M_other);
    if (!(A > 0.0)) return g / cp;
    const double L = latent_heat_auto(T);
    const double num = 1.0 + L * A / (R_mix * T);
    const double den = cp + L * L * A / (R_H2O * T * T);
    return (den > 0.0) ? g * num / den : g / cp;
}
ATHAD_HD double moist_lapse(double T, double p, double M_other, double cp, double R_mix, double g)
{
    if (!(cp > 0.0) || !(T > 0.0) || !(R_mix > 0.0)) return 0.0;
    const double A = sat_deriv_factor_at(saturation_pressure_auto(T), p, M_other);
    if (!(A > 0.0)) return g / cp;
    const double L = latent_heat_auto(T);
    const double num = 1.0 + L * A / (R_mix * T);
    const double den = cp + L * L * A / (R_H2O * T * T);
    return (den > 0.0) ? g * num / den : g / cp;
}

// Shomate heat capacities (MixtureAtm.h:123-143)
ATHAD_HD double shomate(double T, double A, double B, double Cc, double D, double E)
{
    const double t = smin(smax(T, 298.0), 2000.0) * 1.0e-3;
    const double t2 = t * t;
    return A + B * t + Cc * t2 + D * t2 * t + E / t2;
}

// MixtureAtm.h:152-162
ATHAD_HD void split(double c, double co2, double& q_v, double& q_c, double& q_b)
{
    q_v = smin(smax(c, 0.0), 1.0);
    q_c = smin(smax(co2, 0.0), 1.0);
    const double sum = q_v + q_c;
    if (sum > 1.0) { q_v /= sum; q_c /= sum; }
    q_b = smax(0.0, 1.0 - q_v - q_c);
}

ATHAD_HD double R_of(double c, double co2, double R_b)   // MixtureAtm.h:165-170
{
    double q_v, q_c, q_b;
    split(c, co2, q_v, q_c, q_b);
    return q_v * R_H2O + q_c * R_CO2 + q_b * R_b;
}

ATHAD_HD double cp_of(double c, double co2, double T, double M_b)   // MixtureAtm.h:173-178
{
    double q_v, q_c, q_b;
    split(c, co2, q_v, q_c, q_b);
    return q_v * (shomate(T, 30.09200, 6.832514, 6.793435, -2.534480, 0.082139) / M_H2O)
         + q_c * (shomate(T, 24.99735, 55.18696, -33.69137, 7.948387, -0.136638) / M_CO2)
         + q_b * (shomate(T, 28.98641, 1.853978, -9.647459, 16.63537, 0.000117) / M_b);
}

ATHAD_HD double M_nonwater(double c, double co2, double M_b)   // MixtureAtm.h:209-217
{
    double q_v, q_c, q_b;
    split(c, co2, q_v, q_c, q_b);
    const double sum = q_c + q_b;
    if (!(sum > 0.0)) return M_b;
    const double inv = (q_c / sum) / M_CO2 + (q_b / sum) / M_b;
    return (inv > 0.0) ? 1.0 / inv : M_b;
}

// the water vapour mole fraction, MixtureAtm.h:181-187 (M_of) and :220-225 (x_H2O_of)
ATHAD_HD double x_H2O_of(double c, double co2, double M_b)
{
    double q_v, q_c, q_b;
    split(c, co2, q_v, q_c, q_b);
    const double inv = q_v / M_H2O + q_c / M_CO2 + q_b / M_b;
    const double M = (inv > 0.0) ? 1.0 / inv : M_b;
    return q_v * M / M_H2O;
}

// SaturationH2O::dewPoint (SaturationH2O.h:189-202): bisection of the saturation curve
// (liquid above the triple point, ice below) on [150 K, T_crit], 60 halvings
// d ln p_sat / dT of saturation_pressure_auto, for the dew point's Newton step: the
// Wagner-Pruss line above the triple point (ln p = ln p_c + (T_c/T) S(theta)), the IAPWS
// sublimation curve below it (ln p = ln p_t + sum b_i vartheta^(m_i - 1))
ATHAD_HD double dlnp_sat_dT(double T)
{
    if (T >= T_TRIPLE) {
        const double theta = 1.0 - T / T_CRIT;
        const double sq = sqrt(theta);
        const double t2 = theta * theta, t3 = t2 * theta;
        const double S = -7.85951783 * theta + 1.84408259 * theta * sq + -11.7866497 * t3
                       + 22.6807411 * t3 * sq + -15.9618719 * t3 * theta + 1.80122502 * t3 * t3 * theta * sq;
        const double dS = -7.85951783 + 1.5 * 1.84408259 * sq + 3.0 * -11.7866497 * t2
                        + 3.5 * 22.6807411 * t2 * sq + 4.0 * -15.9618719 * t3 + 7.5 * 1.80122502 * t3 * t3 * sq;
        return -(T_CRIT / (T * T)) * S - dS / T;
    }
    const double th = T / T_TRIPLE;
    const double lt = log(th);
    return (-0.212144006e2 * (0.333333333e-2 - 1.0) * exp((0.333333333e-2 - 2.0) * lt)
            + 0.273203819e2 * (0.120666667e1 - 1.0) * exp((0.120666667e1 - 2.0) * lt)
            + -0.610598130e1 * (0.170333333e1 - 1.0) * exp((0.170333333e1 - 2.0) * lt)) / T_TRIPLE;
}

// SaturationH2O::dewPoint (the temperature whose saturation pressure is e): the reference
// bisects [150 K, T_crit] 60 times; here a Newton iteration on ln p_sat(T) = ln e, kept
// inside the bisection bracket it narrows (a step leaving it bisects instead), stops when a
// step moves T by under 1e-12 K.  Both end at the root to within a few ulps; the same
// results below 150 K, at and above the critical pressure and for e <= 0.
ATHAD_HD double dew_point(double e)
{
    if (!(e > 0.0)) return 0.0;
    if (e >= 220640.0) return T_CRIT;
    double lo = 150.0, hi = T_CRIT;
    if (saturation_pressure_auto(lo) >= e) return lo;
    const double ln_e = log(e);
    // Clausius-Clapeyron start from the triple point (6.11657 hPa; L/R_v = 2.5e6 / 461.5 K)
    double T = 1.0 / (1.0 / T_TRIPLE - log(e / 6.11657) / (2.5e6 / 461.5));
    if (!(T > lo && T < hi)) T = 0.5 * (lo + hi);
    for (int it = 0; it < 60; it++) {
        const double p = saturation_pressure_auto(T);
        if (p < e) lo = T; else hi = T;
        double Tn = T - (log(p) - ln_e) / dlnp_sat_dT(T);
        if (fabs(Tn - T) <= 1.0e-12 && Tn >= lo && Tn <= hi) return Tn;   // converged
        if (!(Tn > lo && Tn < hi)) Tn = 0.5 * (lo + hi);
        T = Tn;
        if (hi - lo <= 1.0e-12) break;
    }
    return T;
}

}  // namespace thermo

}  // namespace athad
