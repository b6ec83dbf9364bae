// k_surface.cu - the surface-flux modules of the moist iteration on sm_100a, flat terrain:
//
//   water_vapour_evaporation_kernel  ThermoAtm::waterVapourEvaporation (ThermoAtm.h:115-398):
//       the sea surface as a saturation boundary (:186-262), one thread per (j, k) column:
//       the surface vapour relaxes toward the sea's saturation mass fraction, the change
//       spreads over levels 1-3 with weights e^-i (capped at each level's saturation), and
//       the Dalton, Meyer and Rohwer rates of the saturation deficit are reported.  The
//       Earth branch after that block (:264-362) is unreachable in the reference: not built.
//   latent_sensible_kernel           ThermoAtm::latentSensibleHeat (ThermoAtm.h:36-112):
//       Q_Latent zeroed at the surface, Q_Sensible = cp_l t_0 |grad t| / sqrt(3) inside.
//
// Compiled without fused multiply-add; the saturation curves are CUDA's exp/log/sqrt.
#include "kernels.cuh"
#include "thermo.cuh"

namespace athad {

namespace {

using namespace thermo;

__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }

__global__ void __launch_bounds__(128) water_vapour_evaporation_kernel(SurfaceArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= d.km) return;
    const long long c0 = idx3(d, 0, j, k);
    const long long q2 = (long long)j * d.pitch + k;
    if (a.t[c0] * a.t_0 >= T_CRIT) {             // no interface above the critical point
        a.evap_dalton[q2] = 0.0; a.evap_meyer[q2] = 0.0; a.evap_rohwer[q2] = 0.0; a.evap[q2] = 0.0;
        return;
    }
    const double hPa_to_mmHg = 0.750062, K_Meyer = 11.0;
    const double T_s = dmax(180.0, a.t[c0] * a.t_0);
    const double p_s = a.p_stat[c0];
    const double c_s = a.c[c0];
    const double M_nw = M_nonwater(c_s, a.co2[c0], a.M_bg);
    const double E_s = saturation_pressure_auto(T_s);
    const double q_sea = saturation_mass_fraction(E_s, p_s, M_nw);
    const double u = a.u[c0], v = a.v[c0], w = a.w[c0];
    const double vel = sqrt((u * u + v * v + w * w) / 3.0) * a.u_0;
    const double u_kmh_d = vel * 3.6;
    const double e_air = (q_sea > 0.0 && q_sea < 1.0)
        ? c_s * p_s * M_nw / (c_s * M_nw + (1.0 - c_s) * M_H2O)
        : 0.0;
    const double sd_d = dmax(0.0, E_s - e_air);
    // AtomUtils::C_Dalton (lib/Utils.cpp:157-172): v_max = 10 m/s, c_Dalton_max = 0.053
    const double c_dalton = a.coeff_Dalton * sqrt(0.053 * 0.053 * vel / 10.0);
    const double ed = c_dalton * 24.0 * sd_d;
    a.evap_dalton[q2] = ed;
    a.evap_meyer[q2] = K_Meyer * hPa_to_mmHg * (1.0 + u_kmh_d / 16.0) / 30.0 * sd_d;
    a.evap_rohwer[q2] = 0.771 * (1.465 - 0.000732 * p_s * hPa_to_mmHg)
                      * (0.44 + 0.0733 * u_kmh_d) * hPa_to_mmHg * sd_d;
    a.evap[q2] = ed;
    a.c_fix[q2] = c_s;
    a.c[c0] = c_s + (q_sea - c_s) * a.w_norm;
    for (int i = 1; i <= 3 && i < d.im; i++) {
        const long long ci = idx3(d, i, j, k);
        const double T_i = dmax(180.0, a.t[ci] * a.t_0);
        const double p_i = a.p_stat[ci];
        const double c_i = a.c[ci];
        const double q_s_i = saturation_mass_fraction_at(T_i, p_i, M_nonwater(c_i, a.co2[ci], a.M_bg));
        a.c[ci] = dmin(c_i + (q_sea - c_s) * a.weight[i - 1], q_s_i);
    }
}

__global__ void __launch_bounds__(128) latent_sensible_kernel(SurfaceArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int i = blockIdx.z;
    if (k >= d.km) return;
    const long long c = idx3(d, i, j, k);
    if (i == 0) {
        a.q_latent[c] = 0.0;
        a.q_sensible[c] = 0.0;
        return;
    }
    if (i >= d.im - 1 || j < 1 || j >= d.jm - 1 || k < 1 || k >= d.km - 1) return;
    double sinthe = a.sin_w[j];
    if (fabs(sinthe) < 1e-10) sinthe = 1e-10;
    const double rm = a.rad[i];
    const double exp_rm = 1.0 / (rm + 1.0);
    const double inv_rm = 1.0 / rm;
    const double inv_rmsinthe = 1.0 / (rm * sinthe);
    const double* t = a.t;
    const double dtdr = (t[c + d.plane] - t[c - d.plane]) * (1.0 / (2.0 * a.dr)) * exp_rm;
    const double dtdthe = (t[c + d.pitch] - t[c - d.pitch]) * (1.0 / (2.0 * a.dthe)) * inv_rm;
    const double dtdphi = (t[c + 1] - t[c - 1]) * (1.0 / (2.0 * a.dphi)) * inv_rmsinthe;
    a.q_sensible[c] = a.cp_l * a.t_0 * (1.0 / sqrt(3.0)) * sqrt(dtdr * dtdr + dtdthe * dtdthe + dtdphi * dtdphi);
}

}  // namespace

void launch_water_vapour_evaporation(const SurfaceArgs& a, cudaStream_t st)
{
    water_vapour_evaporation_kernel<<<dim3((a.d.km + 127) / 128, a.d.jm), 128, 0, st>>>(a);
}

void launch_latent_sensible_heat(const SurfaceArgs& a, cudaStream_t st)
{
    latent_sensible_kernel<<<dim3((a.d.km + 127) / 128, a.d.jm, a.d.im - 1), 128, 0, st>>>(a);
}

}  // namespace athad
