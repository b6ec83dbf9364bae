// k_columns.cu - per-cell and per-column moist physics of the ATHAD_COND atmosphere on
// sm_100a: SaturationAdjustment::run (SaturationAdjustment.h:25-459) and
// ThermoAtm::densities (ThermoAtm.h:1436-1666), flat terrain.
//
// Both are FP64-pipe bound (IAPWS transcendentals inside a Newton iteration, a sequential
// column ODE), so they run one thread per cell / per column with k on threadIdx.x for
// coalesced access; the column reduction that builds rho_bar uses a fixed-order warp
// reduction and pairs rows j and jm-1-j so it is deterministic and mirror-invariant.
#include "kernels.cuh"
#include "thermo.cuh"

namespace athad {

using namespace thermo;

// IceSchemeCommon::evaporateWhereImpossible, IceSchemeCommon.h:121-190
__host__ __device__ void evaporate_where_impossible(const ColumnArgs& a, long long c, double t_u,
                                                    double& cv, double& cld, double& ic, double& T_nd)
{
    const double co2 = a.co2[c];
    const double q_cond = smax(0.0, cld) + smax(0.0, ic) + smax(0.0, a.gr[c]);
    if (q_cond > 0.0) {
        const double c_max = smax(0.0, 1.0 - co2);
        const double c_new = smin(c_max, cv + q_cond);
        const double q_used = smax(0.0, c_new - cv);
        cv = c_new;
        cld = 0.0; ic = 0.0;
        a.gr[c] = 0.0;
        if (t_u < T_CRIT) {
            const double cp_loc = cp_of(cv, co2, t_u, a.M_bg);
            if (cp_loc > 0.0) {
                double T_new = t_u - latent_heat(t_u) * q_used / cp_loc;
                if (T_new < 1.0) T_new = 1.0;
                T_nd = T_new / a.t_0;
            }
        }
    }
    {
        const double rho = smax(1.0e-6, a.r_humid[c]);
        const double q_p = smax(0.0, a.P_rain[c]) / (1.6 * rho)
                         + smax(0.0, a.P_snow[c]) / (0.96 * rho)
                         + smax(0.0, a.P_graupel[c]) / (2.0 * rho);
        if (q_p > 0.0) {
            const double c_max = smax(0.0, 1.0 - co2);
            cv = smin(c_max, cv + q_p);
        }
    }
    a.P_rain[c] = 0.0; a.P_snow[c] = 0.0; a.P_graupel[c] = 0.0; a.Precipitation[c] = 0.0;
    a.S_v[c] = 0.0; a.S_c[c] = 0.0; a.S_i[c] = 0.0; a.S_r[c] = 0.0; a.S_s[c] = 0.0;
    a.S_g[c] = 0.0; a.S_c_c[c] = 0.0;
}

// The Newton step's saturation curves (thermo.cuh: SaturationH2O.h:68-120, 168-178,
// 230-255) with the reciprocals they divide by formed once: 1/T per Newton step, shared by
// the saturation and sublimation curves and the derivative factor, and 1/p per cell.  A
// product by a reciprocal instead of a quotient moves a result by at most an ulp or two.
__host__ __device__ __forceinline__ double p_sat_r(double T, double invT)
{
    if (T >= T_CRIT) return NO_SATURATION;
    if (T <= 0.0) return 0.0;
    const double theta = 1.0 - T * (1.0 / T_CRIT);
    const double sq = sqrt(theta);
    const double t15 = theta * sq;
    const double t3 = theta * theta * theta;
    const double t35 = t3 * sq;
    const double t4 = t3 * theta;
    const double t75 = t4 * t3 * sq;
    const double sum = -7.85951783 * theta + 1.84408259 * t15 + -11.7866497 * t3
                     + 22.6807411 * t35 + -15.9618719 * t4 + 1.80122502 * t75;
    return 220640.0 * exp((T_CRIT * invT) * sum);
}
__host__ __device__ __forceinline__ double p_subl_r(double T, double invT)
{
    if (T <= 0.0) return 0.0;
    const double lt = log(T * (1.0 / T_TRIPLE));
    const double sum = -0.212144006e2 * exp(0.333333333e-2 * lt)
                     + 0.273203819e2 * exp(0.120666667e1 * lt)
                     + -0.610598130e1 * exp(0.170333333e1 * lt);
    return 6.11657 * exp(sum * (T_TRIPLE * invT));
}
__host__ __device__ __forceinline__ double q_sat_r(double E, double p, double inv_p, double M_other)
{
    if (E == NO_SATURATION) return 1.0;
    if (!(p > 0.0)) return 0.0;
    if (E >= p) return 1.0;
    const double x = E * inv_p;
    const double num = x * M_H2O;
    const double den = num + (1.0 - x) * M_other;
    return (den > 0.0) ? num / den : 1.0;
}
__host__ __device__ __forceinline__ double dqsat_r(double E, double L, double T, double invT, double p,
                                                   double inv_p, double M_other)
{
    if (!(T > 0.0)) return 0.0;
    if (E == NO_SATURATION || !(p > 0.0) || E >= p) return 0.0;
    const double x = E * inv_p;
    const double den = x * M_H2O + (1.0 - x) * M_other;
    if (!(den > 0.0)) return 0.0;
    return x * M_H2O * M_other / (den * den) * L * (invT * invT) * (1.0 / R_H2O);
}
// The mixture heat capacity of the Newton step (MixtureAtm.h:123-178) with the three
// Shomate polynomials sharing t, t^2, t^3 and 1/t^2, and products by the reciprocal molar
// masses: one division instead of six.  Split in two: the specific heats of the three
// components at T (shomate_r), and their mixture (cp_mix), so a Newton step that moves the
// composition but not T reuses the first.
struct SpecificHeats { double h2o, co2, bg; };
__host__ __device__ __forceinline__ SpecificHeats shomate_r(double T, double inv_M_b)
{
    const double t = smin(smax(T, 298.0), 2000.0) * 1.0e-3;
    const double t2 = t * t, t3 = t2 * t, it2 = 1.0 / t2;
    const double h2o = 30.09200 + 6.832514 * t + 6.793435 * t2 + -2.534480 * t3 + 0.082139 * it2;
    const double co2s = 24.99735 + 55.18696 * t + -33.69137 * t2 + 7.948387 * t3 + -0.136638 * it2;
    const double bg = 28.98641 + 1.853978 * t + -9.647459 * t2 + 16.63537 * t3 + 0.000117 * it2;
    return {h2o * (1.0 / M_H2O), co2s * (1.0 / M_CO2), bg * inv_M_b};
}
__host__ __device__ __forceinline__ double cp_mix(double c, double co2, const SpecificHeats& h)
{
    double q_v, q_c, q_b;
    split(c, co2, q_v, q_c, q_b);
    return q_v * h.h2o + q_c * h.co2 + q_b * h.bg;
}

// adjustSaturation (:62-287) followed, for the same cell, by clampAndFade (:303-459).
// Neither reads a neighbour, so the two passes of the reference fuse into one.
// FP64 in both precision forms: with the Newton step's latent heats, heat capacities and
// derivative factors in FP32, cells converged to values 1e-7 apart from the FP64 form's
// and moved its discontinuous branches (the supersaturation test, the moist-lapse switch of
// the densities) in a few cells within 300 iterations; in FP64 the mixed form stays within
// 1e-9 of the FP64 form in c and cloud over the same iterations.
#ifndef ATHAD_SATADJ_MIN_BLOCKS
#define ATHAD_SATADJ_MIN_BLOCKS 7         // 72 registers, 7 CTAs of 128 threads per SM
#endif
// One cell (i, j, k < km) of the fused pass; returns whether the vapour hit its 1 - co2 cap.
// __host__ __device__: tests/host_columns.cu runs the same source on the host.
__host__ __device__ __forceinline__ bool satadj_cell(const ColumnArgs& a, int i, int j, int k)
{
    const Dims& d = a.d;
    bool hit = false;
    {
        const long long c = idx3(d, i, j, k);
        double cv = a.c[c], cld = a.cloud[c], ic = a.ice[c], T_nd = a.t[c];
        const double co2 = a.co2[c], p_local = a.p_stat[c];
        const double inv_t_0 = 1.0 / a.t_0;
        const double fade_K = 5.0;
        double S_c_c = a.S_c_c[c];
        if (i == 0) S_c_c = 0.0;
        if (i >= 1 && i < d.im - 1) {
            S_c_c = 0.0;
            const double q_v_old = smax(0.0, cv), q_c_old = smax(0.0, cld), q_i_old = smax(0.0, ic);
            double T = T_nd * a.t_0;
            if (T < T_CRIT) {
                const double t_range_inv = 1.0 / (a.t_0 - a.t_00);
                const double dt_dim = a.step_f[i] / 1.6;
                const double M_other = M_nonwater(cv, co2, a.M_bg);
                const double q_sat0 = saturation_mass_fraction(saturation_pressure_auto(T), p_local, M_other);
                const double alpha_entry = 1.0 / (1.0 + exp(-(T - a.t_00) / fade_K));
                if ((q_v_old > q_sat0 && alpha_entry > 0.01) ||
                    (q_v_old < q_sat0 && (q_c_old > 1e-12 || q_i_old > 1e-12))) {
                    double q_v_b = q_v_old, q_c_b = q_c_old, q_i_b = q_i_old;
                    double q_v_hyp = q_v_b;
                    const double T_original = T_nd * a.t_0;
                    // The Newton step of SaturationAdjustment.h:177-254 with the same values,
                    // fewer transcendentals: L(T) of the latent-heat update is the L(T) the
                    // previous pass computed for its gain (T has not changed in between),
                    // the sublimation latent heat is L(T) + 3.337e5 (SaturationH2O.h:150-154),
                    // and the ice curve is evaluated only where a term uses it — where the
                    // deposition weight DEP is 0 and there is no ice its terms are exactly
                    // zero, so skipping them changes no bit.
                    double L_T = latent_heat(T);
                    const double inv_p = 1.0 / p_local;
                    const double inv_M_b = 1.0 / a.M_bg;
                    SpecificHeats sh = shomate_r(T, inv_M_b);   // at the T of the step's start
                    for (int iter = 1; iter <= 20; iter++) {
                        const double CND = smax(0.0, smin(1.0, (T - a.t_00) * t_range_inv));
                        const double DEP = 1.0 - CND;
                        double d_q_v = q_v_hyp - q_v_b;
                        if (d_q_v > 0) {
                            const double max_evap = q_c_b + q_i_b;
                            if (d_q_v > max_evap) d_q_v = max_evap;
                        }
                        const double d_cnd = d_q_v * CND, d_dep = d_q_v * DEP;
                        q_v_b += d_q_v;
                        q_c_b = smax(0.0, q_c_b - d_cnd);
                        q_i_b = smax(0.0, q_i_b - d_dep);
                        const double cp_loc = cp_mix(q_v_b, co2, sh);
                        T -= (L_T * d_cnd + (L_T + 3.337e5) * d_dep) / cp_loc;
                        const double invT = 1.0 / T;
                        const double E_sat = p_sat_r(T, invT);
                        const double q_sat = q_sat_r(E_sat, p_local, inv_p, M_other);
                        const double q_sum = q_c_b + q_i_b;
                        const bool need_ice = (DEP != 0.0) || (q_i_b > 0.0) || (!(q_sum > 1e-12) && !(T >= a.t_0));
                        const double E_Ice = need_ice ? p_subl_r(T, invT) : 0.0;
                        const double q_Ice = need_ice ? q_sat_r(E_Ice, p_local, inv_p, M_other) : 0.0;
                        const double q_v_target = (q_sum > 1e-12) ? (q_c_b * q_sat + q_i_b * q_Ice) / q_sum
                                                                  : ((T >= a.t_0) ? q_sat : q_Ice);
                        sh = shomate_r(T, inv_M_b);   // the updated T: the next step starts from it
                        const double cp_g = cp_mix(q_v_b, co2, sh);
                        const double L_cnd = latent_heat(T);
                        const double L_dep = L_cnd + 3.337e5;
                        double Gain = CND * (L_cnd / cp_g) * dqsat_r(E_sat, L_cnd, T, invT, p_local, inv_p, M_other);
                        if (need_ice) Gain += DEP * (L_dep / cp_g) * dqsat_r(E_Ice, L_dep, T, invT, p_local, inv_p, M_other);
                        L_T = L_cnd;
                        const double omega = 1.0 / (1.0 + Gain);
                        q_v_hyp = q_v_b + omega * (q_v_target - q_v_b);
                        if (fabs(q_v_b / q_v_hyp - 1.0) <= 1.0e-6) break;
                    }
                    q_c_b = smax(0.0, q_c_b);
                    q_i_b = smax(0.0, q_i_b);
                    if (T > T_CRIT) T = T_CRIT;
                    if (!isnan(T) && !isnan(q_v_b)) {
                        S_c_c = alpha_entry * (q_c_b - q_c_old) / dt_dim;
                        cv = q_v_old + alpha_entry * (q_v_b - q_v_old);
                        cld = q_c_old + alpha_entry * (q_c_b - q_c_old);
                        ic = q_i_old + alpha_entry * (q_i_b - q_i_old);
                        T_nd = (T_original + alpha_entry * (T - T_original)) * inv_t_0;
                    }
                    if (T < a.t_00) { cld = 0.0; ic = 0.0; }
                }
            }
        }
        a.S_c_c[c] = S_c_c;
        // ---- clampAndFade ----
        if (cv < 0.0) cv = 0.0;
        if (cld < 0.0) cld = 0.0;
        if (ic < 0.0) ic = 0.0;
        const double c_max = smax(0.0, 1.0 - co2);
        if (cv > c_max) { cv = c_max; hit = true; }
        double T_dim = T_nd * a.t_0;
        if (T_dim > a.t_max_phys) { T_dim = a.t_max_phys; T_nd = a.t_max_phys * inv_t_0; }
        const double M_o = M_nonwater(cv, co2, a.M_bg);
        const double q_s = saturation_mass_fraction_at(T_dim, p_local, M_o);
        if (T_dim >= T_CRIT || q_s >= 1.0) {
            evaporate_where_impossible(a, c, T_dim, cv, cld, ic, T_nd);
        } else {
            const double q_sat = q_s;   // same arguments as the second evaluation (:419-423)
            if (cv > q_sat) {
                const double excess = cv - q_sat;
                cv = q_sat;
                if (T_dim >= a.t_00) {
                    cld += excess;
                    T_dim += latent_heat(T_dim) * excess / cp_of(cv, co2, T_dim, a.M_bg);
                } else {
                    ic += excess;
                    T_dim += latent_heat_sublimation(T_dim) * excess / cp_of(cv, co2, T_dim, a.M_bg);
                }
                if (T_dim > a.t_max_phys) T_dim = a.t_max_phys;
                T_nd = T_dim * inv_t_0;
            }
            if (cld > a.cloud_cap) cld = a.cloud_cap;
            if (ic > a.cloud_cap) ic = a.cloud_cap;
            const double alpha = 1.0 / (1.0 + exp(-(T_dim - a.t_00) / fade_K));
            cv *= alpha; cld *= alpha; ic *= alpha;
        }
        a.c[c] = cv; a.cloud[c] = cld; a.ice[c] = ic; a.t[c] = T_nd;
    }
    return hit;
}

__global__ void __launch_bounds__(128, ATHAD_SATADJ_MIN_BLOCKS)
saturation_adjust_kernel(const ColumnArgs a)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int i = blockIdx.z;
    bool hit = false;
    if (k < a.d.km) hit = satadj_cell(a, i, j, k);
    const unsigned nh = __popc(__ballot_sync(0xffffffffu, hit));
    if ((threadIdx.x & 31) == 0 && nh && a.counters) atomicAdd(a.counters, (unsigned long long)nh);
}

void launch_saturation_adjust(const ColumnArgs& a, cudaStream_t st)
{
    const dim3 block(128), grid((a.d.km + 127) / 128, a.d.jm, a.d.im);
    saturation_adjust_kernel<<<grid, block, 0, st>>>(a);
}

// ---------------------------------------------------------------------------------------
// densities: one thread per column, ThermoAtm.h:1484-1614
#ifndef ATHAD_DENS_BLOCK
#define ATHAD_DENS_BLOCK 128   // columns per CTA
#endif
// One (j, k) column, k < km.  __host__ __device__: tests/host_columns.cu runs the same source
// on the host.
__host__ __device__ __forceinline__ void densities_column(const ColumnArgs& a, int j, int k)
{
    const Dims& d = a.d;
    const double p_sl_factor = 1e-2 * a.r_air * a.R_mix;
    double T_prev = smax(180.0, a.t[idx3(d, 0, j, k)] * a.t_0);
    double p_prev = p_sl_factor * T_prev;
    const double p_first = p_prev;
    // saturation_pressure_auto(T_prev): formed once per level and carried to the next,
    // where T_prev is this level's T (the values, and the results, are the same as
    // evaluating it at each use)
    double E_prev = saturation_pressure_auto(T_prev);
    double q_sat_min = 1.0;
    double q_v_p = 0.0, q_c_p = 0.0;   // c and co2 of level i-1 (after any rewrite)
    double t_last = 0.0;
    // The level recurrence is sequential, so each level's loads would sit on its critical
    // path; the next level's c, co2, cloud and ice are loaded while this level computes.
    // A level writes only its own cells, so the values are those the serial order reads.
    long long c = idx3(d, 0, j, k);
    double q_v = a.c[c], q_c = a.co2[c], cl = a.cloud[c], ic = a.ice[c];
    for (int i = 0; i < d.im; i++) {
        const long long c_next = c + (long long)d.jm * d.pitch;
        double q_v_n = 0.0, q_c_n = 0.0, cl_n = 0.0, ic_n = 0.0;
        if (i + 1 < d.im) { q_v_n = a.c[c_next]; q_c_n = a.co2[c_next]; cl_n = a.cloud[c_next]; ic_n = a.ice[c_next]; }
        const double R_loc = R_of(q_v, q_c, a.R_bg);
        double T_i, p_i;
        if (i == 0) {
            T_i = T_prev; p_i = p_prev;
        } else {
            const double dz = a.height[i] - a.height[i - 1];
            const double cp_loc = cp_of(q_v_p, q_c_p, T_prev, a.M_bg);
            const double M_nw = M_nonwater(q_v_p, q_c_p, a.M_bg);
            const double q_s = saturation_mass_fraction(E_prev, p_prev, M_nw);
            const double gamma = (q_v_p >= 0.99 * q_s)
                ? moist_lapse_E(T_prev, E_prev, p_prev, M_nw, cp_loc, R_loc, a.g)
                : a.g / cp_loc;
            const double T_ad = T_prev - gamma * dz;
            T_i = smax(a.t_skin, T_ad);
            const double T_mean = 0.5 * (T_prev + T_i);
            p_i = p_prev * exp(-a.g * dz / (R_loc * T_mean));
        }
        t_last = T_i / a.t_0;
        a.t[c] = t_last;
        a.p_stat[c] = p_i;
        double q_v_now = q_v;
        const double E_i = (i == 0) ? E_prev : saturation_pressure_auto(T_i);
        if (a.set_water_profile && i > 0) {
            const double M_nw_i = M_nonwater(q_v, q_c, a.M_bg);
            const double q_s_i = saturation_mass_fraction(E_i, p_i, M_nw_i);
            if (q_s_i < q_sat_min) q_sat_min = q_s_i;
            q_v_now = smax(q_sat_min, a.c_h2o_dry_top);
            a.c[c] = q_v_now;
        }
        const double water_factor = smax(0.5, 1.0 - cl - ic);
        a.r_humid[c] = 1e2 * p_i / (R_loc * T_i * water_factor);
        const double R_dry_loc = R_of(0.0, q_c, a.R_bg);
        a.r_dry[c] = 1e2 * p_i / (R_dry_loc * T_i);
        T_prev = T_i; p_prev = p_i; E_prev = E_i;
        q_v_p = q_v_now; q_c_p = q_c;
        c = c_next; q_v = q_v_n; q_c = q_c_n; cl = cl_n; ic = ic_n;
    }
    const long long c2 = (long long)j * d.pitch + k;
    a.t_top_init[c2] = t_last;           // the value stored at level im-1
    a.p_stat_landscape[c2] = p_first;    // the value stored at level 0
}

__global__ void __launch_bounds__(ATHAD_DENS_BLOCK) densities_column_kernel(const ColumnArgs a)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= a.d.km) return;
    densities_column(a, j, k);
}

// per-(i,j) row sums of the positive densities, fixed warp order (one warp per row)
__global__ void __launch_bounds__(256) densities_rowsum_kernel(const ColumnArgs a)
{
    const Dims& d = a.d;
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= d.im * d.jm) return;
    const int i = row / d.jm, j = row % d.jm;
    const double* r = a.r_humid + idx3(d, i, j, 0);
    double s = 0.0, q = 0.0;
    for (int k = lane; k < d.km; k += 32) {
        const double v = r[k];
        if (v > 0.0) { s += v; q += 1.0; }
    }
    for (int off = 16; off >= 1; off >>= 1) {
        s = s + __shfl_xor_sync(0xffffffffu, s, off);
        q = q + __shfl_xor_sync(0xffffffffu, q, off);
    }
    if (lane == 0) { a.row_sum[row] = s; a.row_cnt[row] = q; }
}

// rho_bar(i) and its log-derivative, ThermoAtm.h:1629-1660; one thread per level
__global__ void densities_profile_kernel(const ColumnArgs a)
{
    const Dims& d = a.d;
    const int i = threadIdx.x;
    if (i < d.im) {
        double num = 0.0, den = 0.0;
        for (int j = 0; j <= d.jm / 2; j++) {
            const int jr = d.jm - 1 - j;
            if (jr < j) break;
            const double cl = a.coslat[j];
            const double s0 = a.row_sum[i * d.jm + j], c0 = a.row_cnt[i * d.jm + j];
            if (jr != j) {
                num += cl * (s0 + a.row_sum[i * d.jm + jr]);
                den += cl * (c0 + a.row_cnt[i * d.jm + jr]);
            } else {
                num += cl * s0;
                den += cl * c0;
            }
        }
        const double rb = (den > 0.0) ? num / den : 0.0;
        a.rho_base[i] = rb;
        a.row_sum[i * d.jm] = (rb > 0.0) ? log(rb) : 0.0;   // reuse as lnrho store
    }
    __syncthreads();
    if (i < d.im) {
        const double inv_2dr = a.inv_2dr, inv_dr = a.inv_dr;
        double v = 0.0;
        if (i >= 1 && i < d.im - 1) v = (a.row_sum[(i + 1) * d.jm] - a.row_sum[(i - 1) * d.jm]) * inv_2dr;
        else if (i == 0 && d.im > 1) v = (a.row_sum[1 * d.jm] - a.row_sum[0]) * inv_dr;
        else if (i == d.im - 1 && d.im > 1) v = (a.row_sum[(d.im - 1) * d.jm] - a.row_sum[(d.im - 2) * d.jm]) * inv_dr;
        a.dlnrho[i] = v;
    }
}

// The same rho_bar(i) with one CTA per level: the level's row sums and counts staged in
// shared memory by the whole CTA, then summed by one thread in the order above (the
// single-CTA form waits on a global load per row); the log-derivative follows in
// densities_dlnrho_kernel.
__global__ void __launch_bounds__(128) densities_level_kernel(const ColumnArgs a)
{
    extern __shared__ double rs[];   // [jm] row sums, [jm] counts of level i
    const Dims& d = a.d;
    const int i = blockIdx.x;
    double* rc = rs + d.jm;
    for (int j = threadIdx.x; j < d.jm; j += blockDim.x) {
        rs[j] = a.row_sum[i * d.jm + j];
        rc[j] = a.row_cnt[i * d.jm + j];
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double num = 0.0, den = 0.0;
    for (int j = 0; j <= d.jm / 2; j++) {
        const int jr = d.jm - 1 - j;
        if (jr < j) break;
        const double cl = a.coslat[j];
        if (jr != j) {
            num += cl * (rs[j] + rs[jr]);
            den += cl * (rc[j] + rc[jr]);
        } else {
            num += cl * rs[j];
            den += cl * rc[j];
        }
    }
    const double rb = (den > 0.0) ? num / den : 0.0;
    a.rho_base[i] = rb;
    a.row_sum[i * d.jm] = (rb > 0.0) ? log(rb) : 0.0;   // reuse as lnrho store
}

__global__ void densities_dlnrho_kernel(const ColumnArgs a)
{
    const Dims& d = a.d;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.im) return;
    const double inv_2dr = a.inv_2dr, inv_dr = a.inv_dr;
    double v = 0.0;
    if (i >= 1 && i < d.im - 1) v = (a.row_sum[(i + 1) * d.jm] - a.row_sum[(i - 1) * d.jm]) * inv_2dr;
    else if (i == 0 && d.im > 1) v = (a.row_sum[1 * d.jm] - a.row_sum[0]) * inv_dr;
    else if (i == d.im - 1 && d.im > 1) v = (a.row_sum[(d.im - 1) * d.jm] - a.row_sum[(d.im - 2) * d.jm]) * inv_dr;
    a.dlnrho[i] = v;
}

void launch_densities(const ColumnArgs& a, cudaStream_t st)
{
    const Dims& d = a.d;
    densities_column_kernel<<<dim3((d.km + ATHAD_DENS_BLOCK - 1) / ATHAD_DENS_BLOCK, d.jm), ATHAD_DENS_BLOCK, 0, st>>>(a);
    const int rows = d.im * d.jm;
    densities_rowsum_kernel<<<(rows + 7) / 8, 256, 0, st>>>(a);
    const size_t smem = 2 * (size_t)d.jm * sizeof(double);
    if (smem <= 48 * 1024) {
        densities_level_kernel<<<d.im, 128, smem, st>>>(a);
        densities_dlnrho_kernel<<<(d.im + 63) / 64, 64, 0, st>>>(a);
    } else {
        densities_profile_kernel<<<1, ((d.im + 31) / 32) * 32, 0, st>>>(a);
    }
}

}  // namespace athad
