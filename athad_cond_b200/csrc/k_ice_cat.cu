// k_ice_cat.cu - the ice / precipitation schemes of the other CategoryIceScheme values
// (cAtmosphereModel.cpp:581-596, 1230-1245) on sm_100a, flat terrain:
//
//   ZeroCatIceScheme::run   (ZeroCatIceScheme.h:37-230)   rain only, uncapped flux;
//   OneCatIceScheme::run    (OneCatIceScheme.h:50-378)    rain and snow;
//   ThreeCatIceScheme::run  (ThreeCatIceScheme.h:70-470)  rain, snow and graupel, the fluxes
//                                                         normalised by the surface flux.
//
// Each is an elementwise init kernel (initArrays), one thread per (j, k) column walking it
// top-down in up to two passes until the rain flux at level 23 settles (the reference's
// hard-coded convergence level), then IceSchemeCommon::extrapolateBC (launch_precip_bc).
// Cells where no condensed phase can exist evaporate their condensate, as in TwoCat.
//
// OneCat walks its columns in one serial order (k outer, j inner) and keeps the
// autoconversion rate S_au from the last cell with cloud water wherever a cell has none,
// across columns.  A column's cells change neither t nor cloud where they can condense, so
// the cells that assign S_au, and the values they assign, are the same in both passes and do
// not depend on what the column entered with: the value a column leaves behind is its last
// such cell's, or the one it entered with if it has none.  So:
//   one_cat_exit_kernel     per column, the S_au of its last condensable cell with cloud water;
//   one_cat_scan_kernel     one block: per column the value it enters with, the exit of the
//                           last earlier column (serial order) that has one; 0 before the first,
//                           where the reference reads an uninitialised variable;
//   one_cat_columns_kernel  the columns, each starting from its entry value.
//
// Compiled without fused multiply-add; the powers, exp, sin and cos are CUDA's (the oracle's
// are glibc's: the same values within a few ulp).
#include "ice_common.cuh"

namespace athad {

namespace {

using namespace thermo;
using ice::dmax;
using ice::dmin;
using ice::q_sat_at;
using ice::can_condense;
using ice::evaporate_cell;

constexpr int kCheckLevel = 23;   // the schemes' P_rain.x[23] convergence test
constexpr int kIterPrecEnd = 2;   // ZeroCatIce/OneCatIce/ThreeCatIce::iter_prec_end
constexpr double kPmaxFlux = 3.0e-3;

enum { kInitZero = 0, kInitOne = 1, kInitThree = 2 };

// initArrays: ZeroCat (:69-94) clamps c and cloud and restarts the fluxes from the clamped
// time level n; OneCat (:89-104) clamps c, cloud, ice with `if (x < 0) x = 0` (a NaN stays)
// and restarts from level n unclamped; ThreeCat (:119-144) clamps c, cloud, ice, gr with
// std::max and restarts from level n unclamped.
template <int MODE>
__global__ void __launch_bounds__(256) cat_init_kernel(IceArgs a)
{
    const long long n = a.d.fstride;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        if (MODE == kInitZero) {
            a.c[c] = dmax(0.0, a.c[c]);
            a.cloud[c] = dmax(0.0, a.cloud[c]);
            a.P_rain[c] = dmax(0.0, a.P_rainn[c]);
            a.P_snow[c] = dmax(0.0, a.P_snown[c]);
        } else if (MODE == kInitOne) {
            if (a.c[c] < 0.0) a.c[c] = 0.0;
            if (a.cloud[c] < 0.0) a.cloud[c] = 0.0;
            if (a.ice[c] < 0.0) a.ice[c] = 0.0;
            a.P_rain[c] = a.P_rainn[c];
            a.P_snow[c] = a.P_snown[c];
        } else {
            a.c[c] = dmax(0.0, a.c[c]);
            a.cloud[c] = dmax(0.0, a.cloud[c]);
            a.ice[c] = dmax(0.0, a.ice[c]);
            a.gr[c] = dmax(0.0, a.gr[c]);
            a.P_rain[c] = a.P_rainn[c];
            a.P_snow[c] = a.P_snown[c];
        }
    }
}

// IceSchemeCommon::depositionThrottle (IceSchemeCommon.h:203-237): deposition onto cloud ice
// and the ice -> snow autoconversions, with the ice number density and mean particle mass
struct IceSnowRates { double S_i_dep, S_i_au, S_d_au, N_i, m_i; };

__device__ __forceinline__ IceSnowRates deposition_throttle(const IceArgs& a, long long c, double t_u,
                                                            double q_Ice, double dt_snow_dim)
{
    constexpr double N_i_0 = 1.0e2, m_i_0 = 1.0e-12, m_i_max = 1.0e-9, m_s_0 = 3.0e-9;
    constexpr double c_i_dep = 1.3e-5, c_i_au = 1.0e-3, t_hn = 236.15;
    IceSnowRates r{0.0, 0.0, 0.0, 0.0, 1.0e-9};
    const double cv = a.c[c], ice = a.ice[c];
    double N_i = 0.0, m_i = m_i_max;
    if (t_u <= a.t_0 && t_u > t_hn) {
        N_i = N_i_0 * exp(0.2 * (a.t_0 - t_u));
        m_i = dmin(a.r_humid[c] * ice / N_i, m_i_max);
        m_i = dmax(m_i_0, dmin(m_i, m_i_max));
    }
    if (cv > q_Ice)      r.S_i_dep = c_i_dep * N_i * pow(m_i, 1.0 / 3.0) * (cv - q_Ice);
    else if (cv < q_Ice) r.S_i_dep = dmax(-ice / dt_snow_dim, (cv - q_Ice) / dt_snow_dim);
    if (ice > 0.0)       r.S_i_au = dmax(c_i_au * ice, 0.0);
    if (r.S_i_dep > 0.0) r.S_d_au = r.S_i_dep / (1.5 * (pow(m_s_0 / m_i, 2.0 / 3.0) - 1.0));
    r.N_i = N_i;
    r.m_i = m_i;
    return r;
}

// the interior column of this thread: (j, k) with 1 <= j < jm-1, 1 <= k < km-1
__device__ __forceinline__ bool column_of(const Dims& d, int& j, int& k)
{
    k = blockIdx.x * blockDim.x + threadIdx.x;
    j = blockIdx.y;
    return k >= 1 && k < d.km - 1 && j >= 1 && j < d.jm - 1;
}

// ---------------------------------------------------------------------------------------
// ZeroCatIceScheme::computeColumns (ZeroCatIceScheme.h:98-181)
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) zero_cat_columns_kernel(IceArgs a)
{
    const Dims& d = a.d;
    int j, k;
    if (!column_of(d, j, k)) return;
    constexpr double tau_r_inv = 1.0 / 3.3e3, q_c_crit = 5.0e-4, b_ev = 8.05, c_ac = 0.24;
    const long long sI = d.plane;
    const double t_0 = a.t_0;
    const long long chk = idx3(d, kCheckLevel, j, k);
    for (int iter_prec = 1; iter_prec <= kIterPrecEnd; iter_prec++) {
        const double Rain_check = a.P_rain[chk];
        a.P_rain[idx3(d, d.im - 1, j, k)] = 0.0;
        a.P_snow[idx3(d, d.im - 1, j, k)] = 0.0;
        for (int i = d.im - 2; i >= 0; i--) {
            const long long c = idx3(d, i, j, k);
            const double t_u = a.t[c] * t_0;
            double q_sat;
            if (!can_condense(a, c, t_u, q_sat)) {
                evaporate_cell(a, c, t_u);
                continue;
            }
            const double Rain = a.P_rain[c];
            const double cl = a.cloud[c];
            const bool warm_rain = (t_u >= t_0 && Rain > 0.0);
            const double S_ac = warm_rain ? c_ac * cl * pow(Rain, 7.0 / 9.0) : 0.0;   // accretion
            const double S_au = (cl > q_c_crit) ? (cl - q_c_crit) * tau_r_inv : 0.0; // Kessler
            double S_ev = 0.0;                                                        // evaporation
            if (warm_rain) {
                const double a_ev = 2.76e-3 * exp(0.055 * (t_0 - t_u));
                S_ev = a_ev * (1.0 + b_ev * pow(Rain, 1.0 / 6.0)) * (q_sat - a.c[c]) * pow(Rain, 4.0 / 9.0);
            }
            const double S_c_c = a.S_c_c[c];
            a.S_v[c] = -S_c_c + S_ev;
            a.S_c[c] = S_c_c - S_au - S_ac;
            a.S_r[c] = S_au + S_ac - S_ev;
            // the flux from the cell above's S_r, uncapped (:158-163)
            const double pr = (t_u >= t_0)
                ? dmax(0.0, a.P_rain[c + sI] + a.r_humid[c + sI] * a.S_r[c + sI] * a.step_f[i]) : 0.0;
            a.P_rain[c] = pr;
            a.Precipitation[c] = pr;
        }
        if (fabs(a.P_rain[chk] - Rain_check) * 8.64e4 <= 1.0e-3) break;
    }
}

// ---------------------------------------------------------------------------------------
// OneCatIceScheme::computeColumns (OneCatIceScheme.h:108-349)
// ---------------------------------------------------------------------------------------
constexpr double kOneTauR = 3.3e3, kOneQcCrit = 5.0e-4;

// epsilon(T), the share of autoconversion that nucleates snow (:172-176)
__device__ __forceinline__ double one_cat_eps(const IceArgs& a, double t_u, double t_m2)
{
    return (t_u > a.t_00 && t_u <= a.t_0) ? 0.5 * (1.0 + sin(M_PI * (t_m2 - t_u) / (a.t_0 - a.t_00))) : 0.0;
}
// S_au where the cell has cloud water (:179)
__device__ __forceinline__ double one_cat_sau(double eps_t, double cl)
{
    return (1.0 - eps_t) / kOneTauR * dmax(0.0, cl - kOneQcCrit);
}

__device__ __forceinline__ long long serial_index(const Dims& d, int j, int k)
{
    return (long long)(k - 1) * (d.jm - 2) + (j - 1);
}

__global__ void __launch_bounds__(128) one_cat_exit_kernel(IceArgs a)
{
    const Dims& d = a.d;
    int j, k;
    if (!column_of(d, j, k)) return;
    const double t_m2 = 0.5 * (a.t_0 + a.t_00);
    double v = 0.0, has = 0.0;
    // the last cell of the top-down walk that assigns S_au: the first one bottom-up
    for (int i = 0; i <= d.im - 2; i++) {
        const long long c = idx3(d, i, j, k);
        const double t_u = a.t[c] * a.t_0;
        double q_sat;
        if (!can_condense(a, c, t_u, q_sat)) continue;
        const double cl = a.cloud[c];
        if (cl > 0.0) {
            v = one_cat_sau(one_cat_eps(a, t_u, t_m2), cl);
            has = 1.0;
            break;
        }
    }
    const long long n = serial_index(d, j, k);
    a.sau_exit[n] = v;
    a.sau_has[n] = has;
}

// one block of kScanThreads: each thread a contiguous run of columns in the serial order, an
// inclusive max-scan of the last column with a value over the runs, then each run's entries
constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads) one_cat_scan_kernel(IceArgs a, long long N)
{
    __shared__ long long last[kScanThreads];
    const int t = threadIdx.x;
    const long long chunk = (N + kScanThreads - 1) / kScanThreads;
    const long long lo = min(N, (long long)t * chunk);
    const long long hi = min(N, lo + chunk);
    long long mine = -1;
    for (long long n = lo; n < hi; n++)
        if (a.sau_has[n] != 0.0) mine = n;
    last[t] = mine;
    __syncthreads();
    for (int off = 1; off < kScanThreads; off <<= 1) {
        const long long v = (t >= off) ? last[t - off] : -1;
        __syncthreads();
        if (v > last[t]) last[t] = v;
        __syncthreads();
    }
    long long cur = (t > 0) ? last[t - 1] : -1;
    for (long long n = lo; n < hi; n++) {
        a.sau_entry[n] = (cur >= 0) ? a.sau_exit[cur] : 0.0;
        if (a.sau_has[n] != 0.0) cur = n;
    }
}

__global__ void __launch_bounds__(128) one_cat_columns_kernel(IceArgs a)
{
    const Dims& d = a.d;
    int j, k;
    if (!column_of(d, j, k)) return;
    // OneCatIce constants, OneCatIceScheme.h:17-37
    constexpr double c_ac = 0.24, c_rim = 0.69, b_ev = 5.98, a_melt = 3.90e-6, b_melt = 10.50;
    constexpr double a_if = 1.92e-6, a_cf = 3.97e-5, E_cf = 5.0e-3;
    constexpr double N_cf_0_surf = 2.0e5, N_cf_0_top = 1.0e4, a_mc = 0.08, a_mv = 0.02;
    const long long sI = d.plane;
    const double t_0 = a.t_0, t_00 = a.t_00, t_000 = a.t_000;
    const double t_m1 = 0.5 * (t_0 + t_000), t_m2 = 0.5 * (t_0 + t_00);
    const double p_surf = a.p_stat[idx3(d, 0, j, k)];
    const long long chk = idx3(d, kCheckLevel, j, k);
    double S_au = a.sau_entry[serial_index(d, j, k)];
    for (int iter_prec = 1; iter_prec <= kIterPrecEnd; iter_prec++) {
        const double Rain_check = a.P_rain[chk];
        a.P_rain[idx3(d, d.im - 1, j, k)] = 0.0;
        a.P_snow[idx3(d, d.im - 1, j, k)] = 0.0;
        for (int i = d.im - 2; i >= 0; i--) {
            const long long c = idx3(d, i, j, k);
            const double t_u = a.t[c] * t_0;
            double q_sat;
            if (!can_condense(a, c, t_u, q_sat)) {
                evaporate_cell(a, c, t_u);
                continue;
            }
            const double Rain = a.P_rain[c], Snow = a.P_snow[c];
            const double q_Ice = q_sat_at(a, c, sublimation_pressure(t_u));
            const double step = a.step_f[i];
            const IceSnowRates thr = deposition_throttle(a, c, t_u, q_Ice, step / 0.96);
            // mass-size relation of circular plates (:160-164)
            const double a_m = (t_u < t_0 && t_u >= t_m1)
                ? a_mc - a_mv * (1.0 + cos(2.0 * M_PI * (t_u - t_m1) / (t_0 - t_000))) : a_mc;
            const double eps_t = one_cat_eps(a, t_u, t_m2);
            const double cl = a.cloud[c];
            if (cl > 0.0) S_au = one_cat_sau(eps_t, cl);
            const double S_ac = (1.0 - eps_t) * c_ac * cl * pow(Rain, 7.0 / 9.0);
            const double rim = (cl > kOneQcCrit) ? (c_rim / 5.0) / a_m * (cl - kOneQcCrit) * Snow : 0.0;
            const double S_rim = (t_u < t_0) ? rim : 0.0;
            const double S_shed = (t_u >= t_0) ? rim : 0.0;
            const double a_ev = 2.76e-3 * exp(0.055 * (t_0 - t_u));
            const double S_ev = a_ev * (1.0 + b_ev * pow(Rain, 1.0 / 6.0)) * (q_sat - a.c[c])
                              * pow(Rain, 4.0 / 9.0);
            const double S_melt = a_melt / pow(a_mc, -0.5)
                                * (1.0 + b_melt * pow(a_mc, -0.25) * pow(Snow, 0.9 / 4.3))
                                * ((t_u - t_0) * pow(Snow, 5.0 / 8.6));
            // freezing of rain (:254-274)
            const double p_u = a.p_stat[c];
            double N_cf_0 = N_cf_0_surf + (N_cf_0_surf - N_cf_0_top) / (p_surf - 500.0) * (p_u - p_surf);
            if (p_u <= 500.0) N_cf_0 = N_cf_0_top;
            const double N_cf = (t_u < 270.16) ? N_cf_0 * pow(270.16 - t_u, 1.3) : 0.0;
            double S_frz = 0.0;
            if (t_u <= t_0 && t_u >= t_00) {
                const double S_if_frz = a_if * (exp(a_if * (t_u - t_0)) - 1.0) * pow(Rain, 14.0 / 9.0);
                const double S_cf_frz = a_cf * E_cf * N_cf * pow(Rain, 13.0 / 9.0);
                S_frz = S_if_frz + S_cf_frz;
            }
            const double S_c_c = a.S_c_c[c];
            a.S_v[c] = -S_c_c + S_ev;
            a.S_c[c] = S_c_c - S_au - S_ac - S_rim - S_shed;
            a.S_r[c] = S_au + S_ac - S_ev + S_shed - S_frz + S_melt;
            a.S_s[c] = thr.S_i_au + thr.S_d_au + S_rim + S_frz - S_melt;
            // the capped fluxes from the cell above's sources (:285-329)
            const double rh_up = a.r_humid[c + sI];
            double pr = (t_u >= t_0) ? a.P_rain[c + sI] + rh_up * a.S_r[c + sI] * step : 0.0;
            if (pr < 0.0) pr = 0.0;
            if (pr > kPmaxFlux) pr = kPmaxFlux;
            a.P_rain[c] = pr;
            double ps = (t_u < t_0 && t_u >= t_00) ? a.P_snow[c + sI] + rh_up * a.S_s[c + sI] * step : 0.0;
            if (ps < 0.0) ps = 0.0;
            if (ps > kPmaxFlux) ps = kPmaxFlux;
            a.P_snow[c] = ps;
            a.Precipitation[c] = pr + ps;
        }
        if (fabs(a.P_rain[chk] - Rain_check) * 8.64e4 <= 1.0e-3) break;
    }
}

// ---------------------------------------------------------------------------------------
// ThreeCatIceScheme::computeColumns (ThreeCatIceScheme.h:147-420)
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) three_cat_columns_kernel(IceArgs a)
{
    const Dims& d = a.d;
    int j, k;
    if (!column_of(d, j, k)) return;
    // ThreeCatIce constants, ThreeCatIceScheme.h:17-66
    constexpr double m_i_0 = 1.0e-12;
    constexpr double c_c_au = 4.0e-4, c_ac = 0.24, c_rim = 18.6, c_agg = 10.3, c_i_cri = 0.24;
    constexpr double c_r_cri = 3.2e-5, b_ev = 5.9, c_r_frz = 3.75e-2;
    constexpr double z_csg = 0.5, c_g_rim = 4.43, c_g_agg = 2.46;
    constexpr double t_nuc = 267.15, t_d = 248.15, t_hn = 236.15, t_r_frz = 271.15;
    constexpr double P_norm_floor = 1.0e-6;
    const long long sI = d.plane;
    const double t_0 = a.t_0;
    const long long c0 = idx3(d, 0, j, k);
    const long long chk = idx3(d, kCheckLevel, j, k);
    a.P_rain[chk] = 0.0;
    for (int iter_prec = 1; iter_prec <= kIterPrecEnd; iter_prec++) {
        const double Rain_check = a.P_rain[chk];
        a.P_rain[idx3(d, d.im - 1, j, k)] = 0.0;
        a.P_snow[idx3(d, d.im - 1, j, k)] = 0.0;
        a.P_graupel[idx3(d, d.im - 1, j, k)] = 0.0;
        for (int i = d.im - 2; i >= 0; i--) {
            const long long c = idx3(d, i, j, k);
            const double t_u = a.t[c] * t_0;
            double q_sat;
            if (!can_condense(a, c, t_u, q_sat)) {
                evaporate_cell(a, c, t_u);
                continue;
            }
            // precipitation normalised by the (floored) surface flux (:205-214)
            const double Rain = a.P_rain[c] / dmax(a.P_rain[c0], P_norm_floor);
            const double Snow = a.P_snow[c] / dmax(a.P_snow[c0], P_norm_floor);
            const double Graupel = a.P_graupel[c] / dmax(a.P_graupel[c0], P_norm_floor);
            const double Rain_79 = (Rain > 0.0) ? pow(Rain, 7.0 / 9.0) : 0.0;
            const double Rain_89 = (Rain > 0.0) ? pow(Rain, 8.0 / 9.0) : 0.0;
            const double Rain_139 = (Rain > 0.0) ? pow(Rain, 13.0 / 9.0) : 0.0;
            const double Rain_16 = (Rain > 0.0) ? pow(Rain, 1.0 / 6.0) : 0.0;
            const double Rain_49 = (Rain > 0.0) ? pow(Rain, 4.0 / 9.0) : 0.0;
            const double r_q_r = a.A_r * a.B_rad_neg89 * Rain_89;
            const double r_q_s = a.A_s * a.B_s_neg1213 * ((Snow > 0.0) ? pow(Snow, 12.0 / 13.0) : 0.0);
            const double r_q_g = a.A_g * a.B_g_neg1213 * ((Graupel > 0.0) ? pow(Graupel, 12.0 / 13.0) : 0.0);
            const double p_u_0 = 1e2 * a.p_stat[c];
            const double r_h_i = a.r_humid[c];
            const double c_ijk = a.c[c], cl_i = a.cloud[c], ice_i = a.ice[c];
            const double step_i = a.step_f[i];
            const double q_Ice = q_sat_at(a, c, sublimation_pressure(t_u));
            const double dt_rain_dim = step_i / 1.6;
            const double dt_snow_dim = step_i / 0.96;
            const double rh_rqs_08 = (r_q_s > 0.0) ? pow(r_h_i * r_q_s, 0.8) : 0.0;
            const double rh_rqg_06 = (r_q_g > 0.0) ? pow(r_h_i * r_q_g, 0.6) : 0.0;
            const double rh_rqg_95 = (r_q_g > 0.0) ? pow(r_h_i * r_q_g, 0.94878) : 0.0;
            const IceSnowRates thr = deposition_throttle(a, c, t_u, q_Ice, dt_snow_dim);
            double S_nuc = 0.0;                                                   // nucleation
            if (ice_i == 0.0) {
                if ((t_u < t_d && c_ijk >= q_Ice) || (t_d <= t_u && t_u <= t_nuc && c_ijk >= q_sat))
                    S_nuc = m_i_0 / (r_h_i * dt_snow_dim) * thr.N_i;
            }
            const double S_c_frz = (t_u < t_hn && cl_i > 0.0) ? cl_i / dt_rain_dim : 0.0;
            const double S_c_au = (t_u >= t_0 && cl_i > 0.0) ? dmax(c_c_au * (cl_i - 0.0002), 0.0) : 0.0;
            const double S_ac = (t_u >= t_0) ? c_ac * cl_i * Rain_79 : 0.0;
            const bool cold = t_u < t_0;
            const double S_s_rim = cold ? c_rim * cl_i * Snow : 0.0;
            const double S_g_rim = cold ? c_rim * cl_i * rh_rqg_95 : 0.0;
            const double S_s_shed = cold ? 0.0 : c_rim * cl_i * Snow;
            const double S_g_shed = cold ? 0.0 : c_g_rim * cl_i * rh_rqg_95;
            double S_s_agg = 0.0, S_g_agg = 0.0, S_i_cri = 0.0, S_r_cri = 0.0;
            if (t_u <= t_0) {
                S_s_agg = c_agg * ice_i * Snow;
                S_g_agg = c_g_agg * ice_i * rh_rqg_95;
                S_i_cri = c_i_cri * ice_i * Rain_79;
                S_r_cri = c_r_cri * ice_i / thr.m_i * Rain_139;
            }
            double S_ev = 0.0;
            if (t_u >= t_0 && Rain > 0.0) {
                const double a_ev = 2.76e-3 * exp(0.055 * (t_0 - t_u));
                S_ev = a_ev * (1.0 + b_ev * Rain_16) * (q_sat - c_ijk) * Rain_49;
            }
            // deposition / sublimation of snow and graupel (:303-339)
            const double inv_p_u_0 = 1.0 / p_u_0;
            const double c_minus_qIce = c_ijk - q_Ice;
            const double d_v = (t_u >= t_0)
                ? 101325.0 * inv_p_u_0 * (2.22e-5 + 1.46e-7 * (t_u - t_0))
                : 101325.0 * inv_p_u_0 * (2.22e-5 + 1.25e-7 * (t_u - t_0));
            const double l_h = 0.024 + 8.0e-5 * (t_u - t_0);
            const double q_sat_t_0 = saturation_mass_fraction(a.E_sat_t_0_Pa, p_u_0,
                                                              M_nonwater(c_ijk, a.co2[c], a.M_bg));
            const double t_crit = (c_ijk >= q_sat_t_0)
                ? t_0 - (1.0 / l_h) * a.ls * d_v * r_h_i * (c_ijk - q_sat_t_0) : t_0;
            double S_s_dep, S_g_dep;
            if (t_u < t_0) {
                S_s_dep = (2.91955 - 0.0109928 * t_u + 15871.3 * inv_p_u_0 + 1.74744e-6 * p_u_0)
                        * c_minus_qIce * rh_rqs_08;
                S_g_dep = 0.0;
            } else if (t_u < t_crit) {
                S_s_dep = (0.28003 - 0.146293e-6 * p_u_0) * c_minus_qIce * rh_rqs_08;
                S_g_dep = (0.0418521 - 4.7524e-8 * p_u_0) * c_minus_qIce * rh_rqg_06;
            } else {
                S_s_dep = (2.41897 + 31282.3 * inv_p_u_0) * c_minus_qIce * rh_rqs_08;
                S_g_dep = (0.153907 - 7.86703e-7 * p_u_0) * c_minus_qIce * rh_rqg_06;
            }
            double S_s_melt = 0.0, S_g_melt = 0.0;                                // melting
            if (t_u >= t_0) {
                const double melt_driver = (t_u - t_0) + 2.95e+3 * (c_ijk - q_sat_t_0);
                S_s_melt = melt_driver * (0.612654e-3 + 79.6863 * inv_p_u_0) * rh_rqs_08;
                S_g_melt = melt_driver * (7.39441e-5 + 12.31698 * inv_p_u_0) * rh_rqg_06;
            }
            const double S_i_melt = (t_u > t_0 && ice_i > 0.0) ? ice_i / dt_snow_dim : 0.0;
            double S_r_frz;                                                       // freezing
            if (t_u > t_hn) {
                const double t_frz = dmax(t_r_frz - t_u, 0.0);
                S_r_frz = c_r_frz * pow(t_frz, 1.5) * pow(r_h_i * r_q_r, 27.0 / 16.0);
            } else {
                S_r_frz = Rain / dt_rain_dim;
            }
            const double S_csg = (t_u <= t_0 && cl_i > 0.0002)
                ? z_csg * cl_i * ((r_q_s > 0.0) ? pow(r_h_i * r_q_s, 0.75) : 0.0) : 0.0;
            const double S_c_c = a.S_c_c[c];
            a.S_v[c] = -S_c_c + S_ev - thr.S_i_dep - S_s_dep - S_g_dep - S_nuc;
            a.S_c[c] = S_c_c - S_c_au - S_ac - S_c_frz + S_i_melt - S_s_rim - S_g_rim - S_s_shed - S_g_shed;
            a.S_i[c] = S_nuc + S_c_frz + thr.S_i_dep - S_i_melt - thr.S_i_au - thr.S_d_au - S_s_agg - S_g_agg
                     - S_i_cri;
            a.S_r[c] = S_c_au + S_ac - S_ev + S_s_shed + S_g_shed - S_r_cri - S_r_frz + S_s_melt + S_g_melt;
            a.S_s[c] = thr.S_i_au + thr.S_d_au + S_s_agg + S_s_rim + S_s_dep + S_i_cri + S_r_cri - S_s_melt
                     - S_csg;
            a.S_g[c] = S_g_agg + S_g_rim + S_g_dep + S_i_cri + S_r_cri + S_r_frz - S_g_melt + S_csg;
            // the capped top-down fluxes (:395-412)
            const double rh_up = a.r_humid[c + sI];
            const double pr = (t_u >= t_0)
                ? dmin(kPmaxFlux, dmax(0.0, a.P_rain[c + sI] + rh_up * a.S_r[c + sI] * step_i)) : 0.0;
            const double ps = (t_u < t_0 && t_u >= a.t_000)
                ? dmin(kPmaxFlux, dmax(0.0, a.P_snow[c + sI] + rh_up * a.S_s[c + sI] * step_i)) : 0.0;
            const double pg = (t_u < t_0 && t_u >= a.t_00)
                ? dmin(kPmaxFlux, dmax(0.0, a.P_graupel[c + sI] + rh_up * a.S_g[c + sI] * step_i)) : 0.0;
            a.P_rain[c] = pr;
            a.P_snow[c] = ps;
            a.P_graupel[c] = pg;
            a.Precipitation[c] = pr + ps + pg;
        }
        if (fabs(a.P_rain[chk] - Rain_check) * 8.64e4 <= 1.0e-3) break;
    }
}

dim3 column_grid(const Dims& d) { return dim3((d.km + 127) / 128, d.jm); }

}  // namespace

void launch_zero_cat_ice(const IceArgs& a, cudaStream_t st)
{
    cat_init_kernel<kInitZero><<<148 * 8, 256, 0, st>>>(a);
    zero_cat_columns_kernel<<<column_grid(a.d), 128, 0, st>>>(a);
    double* P[3] = {a.P_rain, a.P_snow, nullptr};
    const int avg[3] = {1, 0, 0};   // ZeroCat's snow keeps the seam unaveraged (:206-209)
    launch_precip_bc(a.d, P, avg, 2, st);
}

void launch_one_cat_ice(const IceArgs& a, cudaStream_t st)
{
    const long long N = (long long)(a.d.jm - 2) * (a.d.km - 2);
    cat_init_kernel<kInitOne><<<148 * 8, 256, 0, st>>>(a);
    one_cat_exit_kernel<<<column_grid(a.d), 128, 0, st>>>(a);
    one_cat_scan_kernel<<<1, kScanThreads, 0, st>>>(a, N);
    one_cat_columns_kernel<<<column_grid(a.d), 128, 0, st>>>(a);
    double* P[3] = {a.P_rain, a.P_snow, nullptr};
    const int avg[3] = {1, 1, 0};
    launch_precip_bc(a.d, P, avg, 2, st);
}

void launch_three_cat_ice(const IceArgs& a, cudaStream_t st)
{
    cat_init_kernel<kInitThree><<<148 * 8, 256, 0, st>>>(a);
    three_cat_columns_kernel<<<column_grid(a.d), 128, 0, st>>>(a);
    double* P[3] = {a.P_rain, a.P_snow, a.P_graupel};
    const int avg[3] = {1, 1, 1};
    launch_precip_bc(a.d, P, avg, 3, st);
}

}  // namespace athad
