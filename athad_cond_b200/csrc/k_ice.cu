// k_ice.cu - the two-category ice scheme (TwoCatIceScheme::run, TwoCatIceScheme.h:89-109,
// the configuration's CategoryIceScheme = 2) of the ATHAD_COND atmosphere on sm_100a, flat
// terrain:
//
//   ice_init_kernel      initArrays (:126-158): non-negative water species, the falling
//                        fluxes restarted from the time level n;
//   ice_columns_kernel   computeColumns (:162-484): one thread per (j, k) column walks the
//                        column top-down, up to three passes until the rain flux at i = 1
//                        settles; per cell the COSMO sources and sinks, the cloud-water and
//                        cloud-ice limiters and the capped flux integration;
//   ice_bc_*_kernel      applyBoundaryConditions (:489-492): IceSchemeCommon::extrapolateBC
//                        (IceSchemeCommon.h:27-52) of P_rain and P_snow, radial lid, poles,
//                        then the seam with its average (launch_precip_bc, shared with the
//                        other schemes of k_ice_cat.cu, which choose the average per field).
//
// A column reads nothing of other columns, so the columns run independently.  The reference
// keeps N_i, m_i, S_nuc and S_i_dep from one cell to the next where a branch does not
// assign them; the thread carries them the same way.  Compiled without fused multiply-add;
// exp, log and the saturation curves are CUDA's.  The reference's pow calls become powers of
// one root per cell (Rain^(1/18), Snow^(1/26)), cbrt and x * sqrt(x): the same exponents
// within a few ulp.
#include "ice_common.cuh"

namespace athad {

namespace {

using namespace thermo;

// TwoCatIce constants, TwoCatIceScheme.h:17-71
constexpr double kNi0 = 1.0e2, kMi0 = 1.0e-12, kMiMax = 1.0e-9, kMs0 = 3.0e-9;
constexpr double kCiDep = 1.3e-5, kCcAu = 1.0e-3, kQcCrit = 5.0e-4, kCiAu = 1.0e-3;
constexpr double kCac = 0.24, kCrim = 18.6, kCrimSnow = 18.6 / 5.0, kCagg = 10.3;
constexpr double kCiCri = 0.24, kCrCri = 3.2e-5, kAev = 1.0e-3, kBev = 5.9;
constexpr double kCsDep = 1.8e-2, kBsDep = 12.3, kCsMelt = 8.43e-5, kBsMelt = 12.05;
constexpr double kCrFrz = 3.75e-2;
constexpr double kTnuc = 267.15, kTd = 248.15, kThn = 236.15, kTrFrz = 271.15;
constexpr int kIterPrecEnd = 3, kIcheck = 1;

using ice::dmax;
using ice::dmin;
using ice::q_sat_at;
using ice::evaporate_cell;

__global__ void __launch_bounds__(256) ice_init_kernel(IceArgs a)
{
    const long long n = a.d.fstride;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        a.c[c] = dmax(0.0, a.c[c]);
        a.cloud[c] = dmax(0.0, a.cloud[c]);
        a.ice[c] = dmax(0.0, a.ice[c]);
        const double pr = dmax(0.0, a.P_rainn[c]);
        const double ps = dmax(0.0, a.P_snown[c]);
        a.P_rainn[c] = pr; a.P_snown[c] = ps;
        a.P_rain[c] = pr; a.P_snow[c] = ps;
    }
}

__global__ void __launch_bounds__(128) ice_columns_kernel(IceArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k < 1 || k >= d.km - 1 || j < 1 || j >= d.jm - 1) return;
    const long long sI = d.plane;
    const double t_0 = a.t_0;
    const double P_max = 50.0 / 86400.0;
    const double Rain_check = a.P_rain[idx3(d, kIcheck, j, k)];
    double m_i = kMiMax, N_i = 0.0, S_nuc = 0.0, S_i_dep = 0.0;
    for (int iter_prec = 1; iter_prec <= kIterPrecEnd; iter_prec++) {
        a.P_rain[idx3(d, d.im - 1, j, k)] = 0.0;
        a.P_snow[idx3(d, d.im - 1, j, k)] = 0.0;
        for (int i = d.im - 2; i >= 0; i--) {
            const long long c = idx3(d, i, j, k);
            const double t_u = a.t[c] * t_0;
            // IceSchemeCommon::canCondense (IceSchemeCommon.h:108-111); its q_sat is the
            // scheme's own
            if (t_u >= T_CRIT) {
                evaporate_cell(a, c, t_u);
                continue;
            }
            const double q_sat = q_sat_at(a, c, saturation_pressure(t_u));
            if (!(q_sat < 1.0)) {
                evaporate_cell(a, c, t_u);
                continue;
            }
            const double Rain = a.P_rain[c], Snow = a.P_snow[c];
            // the rain powers 4/9, 7/9, 13/9 and 1/6 from one logarithm: r18 = Rain^(1/18)
            double R49 = 0.0, R79 = 0.0, R139 = 0.0, R16 = 0.0;
            if (Rain > 1e-12) {
                const double r18 = exp(log(Rain) * (1.0 / 18.0));
                const double rb = r18 * r18;
                const double r2 = rb * rb;
                const double r4 = r2 * r2;
                R49 = r4; R79 = Rain / r2; R139 = Rain * r4; R16 = rb * r18;
            }
            // the snow powers 5/26 and 8/13 = 16/26 from one logarithm: s26 = Snow^(1/26)
            double S526 = 0.0, S813 = 0.0;
            if (Snow > 1e-12) {
                const double s26 = exp(log(Snow) * (1.0 / 26.0));
                const double s2 = s26 * s26;
                const double s4 = s2 * s2;
                const double s8 = s4 * s4;
                S526 = s4 * s26; S813 = s8 * s8;
            }
            const double q_Ice = q_sat_at(a, c, sublimation_pressure(t_u));
            const double step = a.step_f[i];
            const double rh = a.r_humid[c];
            const double mass_layer = rh * step;
            const double dt_snow_dim = step / 0.96;
            const double cv = a.c[c], cl = a.cloud[c], ic = a.ice[c];
            if (!(t_u > t_0) && !(t_u <= kThn)) {
                N_i = kNi0 * exp(0.2 * (t_0 - t_u));
                m_i = dmin((rh * ic) / N_i, kMiMax);
                if (m_i > kMiMax) m_i = kMiMax;
                if (m_i < kMi0) m_i = kMi0;
            }
            if (ic == 0.0) {
                if ((t_u < kTd && cv >= q_Ice) || ((kTd <= t_u && t_u <= kTnuc) && cv >= q_sat))
                    S_nuc = kMi0 / (rh * dt_snow_dim) * N_i;
            } else {
                S_nuc = 0.0;
            }
            double S_c_frz = (t_u < kThn) ? cl / dt_snow_dim : 0.0;
            if (cv > q_Ice) S_i_dep = kCiDep * N_i * cbrt(m_i) * (cv - q_Ice);
            if (cv < q_Ice) S_i_dep = dmax(-ic / dt_snow_dim, (cv - q_Ice) / dt_snow_dim);
            double S_c_au = (cl > kQcCrit) ? kCcAu * (cl - kQcCrit) : 0.0;
            double S_i_au = (ic > 0.0) ? dmax(kCiAu * ic, 0.0) : 0.0;
            double S_d_au = 0.0;
            if (S_i_dep > 0.0) {
                const double r = cbrt(kMs0 / m_i);
                S_d_au = S_i_dep / (1.5 * (r * r - 1.0));
            }
            double S_ac = (t_u >= t_0 && cl > kQcCrit) ? kCac * (cl - kQcCrit) * R79 : 0.0;
            double S_rim = (t_u < t_0) ? kCrimSnow * cl * Snow : 0.0;
            double S_shed = (t_u >= t_0) ? kCrim * cl * Snow : 0.0;
            double S_s_melt = 0.0, S_i_melt = 0.0;
            if (t_u > t_0) {
                if (Snow > 1e-12) {
                    S_s_melt = kCsMelt * (1.0 + kBsMelt * S526) * (t_u - t_0) * cbrt(Snow);
                    S_s_melt = dmin(S_s_melt, Snow / mass_layer);
                }
                S_i_melt = ic / dt_snow_dim;
            }
            double S_agg = 0.0, S_i_cri = 0.0, S_r_cri = 0.0;
            if (t_u <= t_0) {
                S_agg = kCagg * ic * Snow;
                S_i_cri = kCiCri * ic * R79;
                S_r_cri = kCrCri * ic / m_i * R139;
            }
            double S_ev = 0.0;
            if (t_u > t_0 && Rain > 1e-12 && cv < q_sat) {
                S_ev = kAev * (1.0 + kBev * R16) * (q_sat - cv) * R49;
                S_ev = dmin(S_ev, Rain / mass_layer);
            }
            double S_s_dep = 0.0;
            if (t_u < t_0 && Snow > 1e-12) {
                S_s_dep = kCsDep * (1.0 + kBsDep * S526) * (cv - q_Ice) * S813;
                if (S_s_dep < 0.0) S_s_dep = dmax(S_s_dep, -Snow / mass_layer);
            }
            double S_r_frz = 0.0;
            if (t_u <= t_0) {
                const double t_frz = dmax(kTrFrz - t_u, 0.0);
                // x^(3/2) = x * sqrt(x) for x >= 0; Rain >= 0 after the init kernel and the flux caps
                S_r_frz = kCrFrz * (t_frz * sqrt(t_frz)) * (Rain * sqrt(Rain));
            }
            // the cloud-water and cloud-ice limiters (:413-434)
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
            const double S_c_c = a.S_c_c[c];
            a.S_v[c] = -S_c_c + S_ev - S_i_dep - S_s_dep - S_nuc;
            a.S_c[c] = S_c_c - S_c_au - S_ac - S_c_frz + S_i_melt - S_rim - S_shed;
            a.S_i[c] = S_nuc + S_c_frz + S_i_dep - S_i_melt - S_i_au - S_d_au - S_agg - S_i_cri;
            a.S_r[c] = S_c_au + S_ac - S_ev + S_shed - S_r_cri - S_r_frz + S_s_melt;
            a.S_s[c] = S_i_au + S_d_au + S_agg + S_rim + S_s_dep + S_i_cri + S_r_cri + S_r_frz - S_s_melt;
            // the fluxes, integrated top-down and capped at 50 mm/d (:478-509)
            const double dP_rain = (S_c_au + S_ac + S_shed + S_s_melt - S_ev - S_r_frz) * mass_layer;
            const double pr = dmin(P_max, dmax(0.0, a.P_rain[c + sI] + dP_rain));
            a.P_rain[c] = pr;
            const double dP_snow = (S_i_au + S_d_au + S_rim + S_agg + S_r_frz - S_s_melt) * mass_layer;
            const double ps = (t_u < t_0 && t_u >= a.t_000) ? dmin(P_max, dmax(0.0, a.P_snow[c + sI] + dP_snow)) : 0.0;
            a.P_snow[c] = ps;
            a.Precipitation[c] = dmin(P_max, pr + ps);
        }
        const double P_rain_diff = fabs(a.P_rain[idx3(d, kIcheck, j, k)] - Rain_check) * 8.64e4;
        if (P_rain_diff <= 1.0e-3) break;
    }
}

// extrapolateBC with c43 = 1, c13 = 0 (const int members, cAtmosphereModel.h:158), for the
// field b.P[blockIdx.z]: radial lid, then poles, then the seam (averaged where b.avg is set)
struct PrecipBc { double* P[3]; int avg[3]; };

__global__ void ice_bc_lid_kernel(Dims d, PrecipBc b)
{
    double* P = b.P[blockIdx.z];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= d.km) return;
    P[idx3(d, d.im - 1, j, k)] = 1.0 * P[idx3(d, d.im - 2, j, k)] - 0.0 * P[idx3(d, d.im - 3, j, k)];
}
__global__ void ice_bc_pole_kernel(Dims d, PrecipBc b)
{
    double* P = b.P[blockIdx.z];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (k >= d.km) return;
    P[idx3(d, i, 0, k)] = 1.0 * P[idx3(d, i, 1, k)] - 0.0 * P[idx3(d, i, 2, k)];
    P[idx3(d, i, d.jm - 1, k)] = 1.0 * P[idx3(d, i, d.jm - 2, k)] - 0.0 * P[idx3(d, i, d.jm - 3, k)];
}
__global__ void ice_bc_seam_kernel(Dims d, PrecipBc b)
{
    double* P = b.P[blockIdx.z];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= d.jm) return;
    double* row = P + idx3(d, i, j, 0);
    const double r0 = 1.0 * row[1] - 0.0 * row[2];
    const double r1 = 1.0 * row[d.km - 2] - 0.0 * row[d.km - 3];
    if (b.avg[blockIdx.z]) {
        const double m = (r0 + r1) * 0.5;
        row[0] = m;
        row[d.km - 1] = m;
    } else {
        row[0] = r0;
        row[d.km - 1] = r1;
    }
}

}  // namespace

void launch_two_cat_ice(const IceArgs& a, cudaStream_t st)
{
    const Dims& d = a.d;
    ice_init_kernel<<<148 * 8, 256, 0, st>>>(a);
    ice_columns_kernel<<<dim3((d.km + 127) / 128, d.jm), 128, 0, st>>>(a);
    double* P[3] = {a.P_rain, a.P_snow, nullptr};
    const int avg[3] = {1, 1, 0};
    launch_precip_bc(d, P, avg, 2, st);
}

void launch_precip_bc(const Dims& d, double* const* P, const int* avg, int n, cudaStream_t st)
{
    PrecipBc b;
    for (int q = 0; q < 3; q++) {
        b.P[q] = (q < n) ? P[q] : nullptr;
        b.avg[q] = (q < n) ? avg[q] : 0;
    }
    ice_bc_lid_kernel<<<dim3((d.km + 127) / 128, d.jm, n), 128, 0, st>>>(d, b);
    ice_bc_pole_kernel<<<dim3((d.km + 127) / 128, d.im, n), 128, 0, st>>>(d, b);
    ice_bc_seam_kernel<<<dim3((d.jm + 127) / 128, d.im, n), 128, 0, st>>>(d, b);
}

}  // namespace athad
