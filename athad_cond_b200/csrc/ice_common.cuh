// ice_common.cuh - device pieces shared by the ice / precipitation schemes (k_ice.cu,
// k_ice_cat.cu): IceSchemeCommon's saturation, condensability and evaporation of a cell
// (IceSchemeCommon.h:71-190).  Compiled without fused multiply-add in every includer.
#pragma once
#include "kernels.cuh"
#include "thermo.cuh"

namespace athad {
namespace ice {

__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }   // std::max
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }   // std::min

// IceSchemeCommon::qSatWater / qSatIce (:71-84) for the saturation pressure E of cell c
__device__ __forceinline__ double q_sat_at(const IceArgs& a, long long c, double E)
{
    return thermo::saturation_mass_fraction(E, a.p_stat[c], thermo::M_nonwater(a.c[c], a.co2[c], a.M_bg));
}

// IceSchemeCommon::canCondense (:108-111); q_sat receives qSatWater where it was formed
__device__ __forceinline__ bool can_condense(const IceArgs& a, long long c, double t_u, double& q_sat)
{
    if (t_u >= thermo::T_CRIT) return false;
    q_sat = q_sat_at(a, c, thermo::saturation_pressure(t_u));
    return q_sat < 1.0;
}

// IceSchemeCommon::evaporateWhereImpossible (:121-190) on cell c
__device__ inline void evaporate_cell(const IceArgs& a, long long c, double t_u)
{
    const double q_cond = dmax(0.0, a.cloud[c]) + dmax(0.0, a.ice[c]) + dmax(0.0, a.gr[c]);
    if (q_cond > 0.0) {
        const double c_max = dmax(0.0, 1.0 - a.co2[c]);
        const double c_new = dmin(c_max, a.c[c] + q_cond);
        const double q_used = dmax(0.0, c_new - a.c[c]);
        a.c[c] = c_new;
        a.cloud[c] = 0.0; a.ice[c] = 0.0; a.gr[c] = 0.0;
        if (t_u < thermo::T_CRIT) {
            const double cp_loc = thermo::cp_of(a.c[c], a.co2[c], t_u, a.M_bg);
            if (cp_loc > 0.0) {
                double T_new = t_u - thermo::latent_heat(t_u) * q_used / cp_loc;
                if (T_new < 1.0) T_new = 1.0;
                a.t[c] = T_new / a.t_0;
            }
        }
    }
    const double rho = dmax(1.0e-6, a.r_humid[c]);
    const double q_p = dmax(0.0, a.P_rain[c]) / (1.6 * rho) + dmax(0.0, a.P_snow[c]) / (0.96 * rho)
                     + dmax(0.0, a.P_graupel[c]) / (2.0 * rho);
    if (q_p > 0.0) {
        const double c_max = dmax(0.0, 1.0 - a.co2[c]);
        a.c[c] = dmin(c_max, a.c[c] + q_p);
    }
    a.P_rain[c] = 0.0; a.P_snow[c] = 0.0; a.P_graupel[c] = 0.0; a.Precipitation[c] = 0.0;
    a.S_v[c] = 0.0; a.S_c[c] = 0.0; a.S_i[c] = 0.0; a.S_r[c] = 0.0; a.S_s[c] = 0.0;
    a.S_g[c] = 0.0; a.S_c_c[c] = 0.0;
}

}  // namespace ice
}  // namespace athad
