// k_rad.cu - MultiLayerRadiation::run (MultiLayerRadiation.h:56-388) of the ATHAD_COND
// atmosphere on sm_100a, and the radiative heating of radiation mode 2
// (cAtmosphereModel.cpp:864-879), flat terrain.
//
// One thread per (j, k) column, k on threadIdx.x: the layer emissivities from the column
// mass with pressure broadening and the cloud liquid/ice paths, the cloud short-wave albedo
// bump, four grey upward/downward sweeps that set each air layer to its radiative
// equilibrium, a final sweep, and the linearised surface energy balance.  The sweeps are
// recurrences along the column; their running flux stays in a register and the per-layer
// values the next pass needs go to the radiation field (upward flux) and two scratch fields
// (layer temperature in K, downward flux), all coalesced across the warp's columns.
// Compiled without fused multiply-add; pow and exp are CUDA's.
#include "kernels.cuh"
#include "thermo.cuh"

namespace athad {

namespace {

__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }

// T^4 as two squarings and x^(1/4) as two square roots, where the reference calls
// pow(T, 4.0) and pow(x, 0.25): each within two ulps of the exact power (sqrt is correctly
// rounded), at a few instructions instead of a logarithm and an exponential; the relaxation
// evaluates them 560 times per column
__device__ __forceinline__ double pow4(double T) { const double t2 = T * T; return t2 * t2; }
__device__ __forceinline__ double root4(double x) { return sqrt(sqrt(x)); }

__global__ void __launch_bounds__(128) mlr_columns_kernel(RadArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= d.km) return;
    const long long sI = d.plane;
    const long long c0 = idx3(d, 0, j, k);
    const int i_trop = d.im - 1;
    const double t_0 = a.t_0, sigma = a.sigma;
    // short-wave insolation: pole-to-equator parabola, mirrored (:99-114)
    const int j_max = d.jm - 1, j_half = j_max / 2;
    const int jj = (j > j_half) ? j_max - j : j;
    const double x = (double)jj / (double)j_half;
    const double sw = (a.rad_pole_short - a.rad_equator_short) * (x * x - 2.0 * x) + a.rad_pole_short;
    double* T = a.T;
    double* up = a.radiation;
    double* dn = a.dn;
    double* eps = a.epsilon;
    // emissivities and condensate paths (:130-190)
    const double p_ref = 1.0e5, inv_g = 1.0 / a.g;
    double lwp_col = 0.0, iwp_col = 0.0;
    for (int i = 0; i <= i_trop; i++) {
        const long long c = c0 + i * sI;
        const double ps = a.p_stat[c];
        double dp_Pa = (i < i_trop) ? (ps - a.p_stat[c + sI]) * 100.0 : ps * 100.0;
        if (dp_Pa < 0.0) dp_Pa = 0.0;
        const double q_v = dmax(0.0, a.c[c]);
        const double q_c = dmax(0.0, a.co2[c]);
        const double q_b = dmax(0.0, 1.0 - q_v - q_c);
        const double u_col = dp_Pa * inv_g;
        const double broad = ps * 100.0 / p_ref;
        const double tau_gas = (a.kappa_H2O * q_v + a.kappa_CO2 * q_c + a.kappa_bg * q_b) * u_col * broad;
        const double dz = (i < i_trop) ? a.step_f[i] : a.step_f[i - 1];
        const double tv = a.t[c];
        const double T_i = tv * t_0;
        T[c] = T_i;
        const double R_i = thermo::R_of(q_v, q_c, a.R_bg);
        const double rho_i = (T_i > 0.0) ? (ps * 100.0) / (R_i * T_i) : 0.0;
        const double LWP_i = dmax(0.0, a.cloud[c]) * rho_i * dz * 1000.0;
        const double IWP_i = dmax(0.0, a.ice[c]) * rho_i * dz * 1000.0;
        lwp_col += LWP_i;
        iwp_col += IWP_i;
        const double tau = tau_gas + 0.12 * LWP_i + 0.055 * IWP_i;
        eps[c] = (tau > 700.0) ? 1.0 : (1.0 - exp(-tau));
    }
    const long long q2 = (long long)j * d.pitch + k;
    a.epsilon_2D[q2] = eps[c0];
    double albedo = a.albedo_surface;
    {
        const double cwp_sw = lwp_col + 0.50 * iwp_col;
        const double tau = cwp_sw / 100.0;
        const double refl = tau / (tau + 2.0);
        if (a.albedo_cloud > albedo) albedo = albedo + (a.albedo_cloud - albedo) * refl;
    }
    a.albedo[q2] = albedo;
    // four relaxation sweeps and the final one (:205-262)
    const double T_s0 = T[c0];
    const double up0 = sigma * pow4(T_s0);
    for (int it = 0; it <= 4; it++) {
        double u = up0;
        for (int i = 1; i <= i_trop; i++) {
            const long long c = c0 + i * sI;
            const double e = eps[c];
            u = u * (1.0 - e) + e * sigma * pow4(T[c]);
            up[c] = u;
        }
        double dd = 0.0;
        for (int i = i_trop; i >= 1; i--) {
            const long long c = c0 + i * sI;
            const double e = eps[c];
            dd = dd * (1.0 - e) + e * sigma * pow4(T[c]);
            dn[c] = dd;
        }
        if (it == 4) break;
        for (int i = 1; i <= i_trop; i++) {
            const long long c = c0 + i * sI;
            const double u_below = (i == 1) ? up0 : up[c - sI];
            const double d_above = (i == i_trop) ? 0.0 : dn[c + sI];
            const double emit = 0.5 * (u_below + d_above);
            if (emit > 0.0 && is_finite_bits(emit)) T[c] = root4(emit / sigma);
        }
    }
    for (int i = 1; i <= i_trop; i++) {
        const long long c = c0 + i * sI;
        a.t[c] = T[c] / t_0;
    }
    // the surface energy balance (:268-284)
    const double L_down = dn[c0 + sI];
    const double SW_abs = (1.0 - albedo) * sw;
    const double T_air1 = T[c0 + sI];
    const double c_H = 15.0;
    const double dsigT4 = 4.0 * sigma * T_s0 * T_s0 * T_s0;
    const double T_s = (SW_abs + a.geothermal_flux + L_down - sigma * pow4(T_s0)
                       + dsigT4 * T_s0 + c_H * T_air1) / (dsigT4 + c_H);
    a.t[c0] = T_s / t_0;
    up[c0] = sigma * pow4(T_s);
}

// radiation mode 2: t := t_before (1 - omega) + t_RE omega
__global__ void __launch_bounds__(256) rad_blend_kernel(long long n, const double* __restrict__ t_before,
                                                        double* __restrict__ t, double omega)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        t[q] = t_before[q] * (1.0 - omega) + t[q] * omega;
}

// cAtmosphereModel::planetaryShortWave's row sums (cAtmosphereModel.cpp:244-246): one thread
// per row, the longitudes in order, so the host finishes the budget bit for bit
__global__ void albedo_rows_kernel(Dims d, const double* __restrict__ albedo, double* __restrict__ out)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= d.jm) return;
    const double* row = albedo + (long long)j * d.pitch;
    double s = 0.0;
    for (int k = 0; k < d.km; k++) s += row[k];
    out[j] = s;
}

}  // namespace

void launch_albedo_rows(const Dims& d, const double* albedo, double* out, cudaStream_t st)
{
    albedo_rows_kernel<<<(d.jm + 127) / 128, 128, 0, st>>>(d, albedo, out);
}

void launch_multilayer_radiation(const RadArgs& a, cudaStream_t st)
{
    mlr_columns_kernel<<<dim3((a.d.km + 127) / 128, a.d.jm), 128, 0, st>>>(a);
}

void launch_rad_blend(const Dims& d, const double* t_before, double* t, double omega, cudaStream_t st)
{
    rad_blend_kernel<<<148 * 8, 256, 0, st>>>(d.fstride, t_before, t, omega);
}

}  // namespace athad
