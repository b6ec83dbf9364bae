// k_init.cu - the reference's deterministic initial state built on the device
// (athad_initial_state): cAtmosphereModel::RunTimeSlice for Ma = 0
// (cAtmosphereModel.cpp:468-668) on any grid with flat terrain, then run_3D_loop's
// Held-Suarez snapshot t_eq := t (:750-753).
//
// What the reference computes per row or per column from a handful of configuration
// numbers (the tropopause levels, the prescribed Hadley/Ferrel velocity profiles, the
// parabolic sea-surface temperature, the float layer thicknesses) is tabulated on the host
// in the reference's operation order; the per-cell and per-column work runs here, and the
// modules the sequence shares with the model iteration (densities, saturation adjustment,
// ice scheme, moist convection, turbulence, boundary conditions, the initial projection)
// are the context's own entry points.
//
// Mirror symmetry: the reference evaluates the surface-temperature parabola and
// interpolates the velocity rows of each hemisphere from its own end, which rounds
// differently in mirrored rows; here the northern rows are evaluated and mirrored (v
// negated), so a context's initial state is exactly north-south symmetric.  The anchor row
// of latitude phi is lround((90 - phi) / dlat), dlat = 180/(jm-1) degrees per row, and the
// southern hemisphere is j > (jm-1)/2 (VelocityInitializer.h:72, 196-201 at jm = 181).
//
// Left out, as outputs nothing in the model state reads: precipitableWater, the centrifugal
// and pressure-gradient arrays of forces (its Coriolis and buoyancy arrays are the right-hand
// side's too and are built), vegetationLand (land only) and the standard-atmosphere dew-point
// diagnostic; the file output and the printed diagnostics.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.cuh"
#include "thermo.cuh"

namespace athad {

namespace {

constexpr double kTCrit = 647.096;      // AtmMixture::T_CRIT_H2O (MixtureAtm.h:40)

struct InitArgs {
    Dims d;
    double* t; double* p_stat; double* r_dry; double* r_humid; double* c; double* co2;
    double* cloud; double* ice; double* gr; const double* P_rain;
    double* p_stat_landscape;            // 2-D [jm][pitch]
    const double* Ts;                    // [jm] surface temperature [K], mirror-exact
    const double* dz;                    // [im] get_layer_height(i) - (i-1), a float difference
    double t_0, r_air, R_mix, R_bg, M_bg, g, t_skin, M_nw, c_h2o_dry_top, t_00;
    // initCloudIce
    const double* row_sum;               // [im*jm] per-row excess sums
    double* cloud_max;                   // [im]
    const double* dt_dim;                // [im] step / 1.6
    const double* two_step;              // [im] 2 step
    double Hu_cr_max, Hu_curv, inv_p_crit, det_T_0, cloud_norm;
};

// the (i, j) tables of VelocityInitializer broadcast along k
__global__ void __launch_bounds__(256) init_velocity_kernel(Dims d, const double* tab, double* u, double* v,
                                                             double* w)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.km) return;
    const long long row = blockIdx.y, nrow = (long long)d.im * d.jm;
    const long long c = row * d.pitch + k;
    u[c] = tab[row];
    v[c] = tab[nrow + row];
    w[c] = tab[2 * nrow + row];
}

// initTemperatureData, Step 8-9 (InitValues_Atm.cpp:526-620): per column the dry adiabat
// with the isothermal skin, integrated hydrostatically from the surface
__global__ void __launch_bounds__(128) init_temperature_kernel(InitArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= d.km) return;
    const double inv_t0 = 1.0 / a.t_0;
    const double t_u_init = (a.Ts[j] * inv_t0) * a.t_0;
    double p_prev = 1e-2 * (a.r_air * a.R_mix * t_u_init);
    double T_prev = smax(100.0, t_u_init);
    for (int i = 0; i < d.im; i++) {
        const long long q = idx3(d, i, j, k);
        const double q_v = a.c[q], q_c = a.co2[q];
        const double R_loc = thermo::R_of(q_v, q_c, a.R_bg);
        double T_curr, p_val;
        if (i == 0) {
            T_curr = T_prev;
            p_val = p_prev;
        } else {
            const double dz = a.dz[i];
            const double cp_loc = thermo::cp_of(q_v, q_c, T_prev, a.M_bg);
            const double T_ad = T_prev - (a.g / cp_loc) * dz;
            T_curr = smax(a.t_skin, T_ad);
            const double T_mean = 0.5 * (T_prev + T_curr);
            p_val = p_prev * exp(-a.g * dz / (R_loc * T_mean));
        }
        a.t[q] = T_curr * inv_t0;
        a.p_stat[q] = p_val;
        const double twf = smax(0.5, 1.0 - (a.cloud[q] + a.ice[q]));
        const double R_dloc = thermo::R_of(0.0, q_c, a.R_bg);
        a.r_dry[q] = p_val * 100.0 / (R_dloc * T_curr);
        a.r_humid[q] = p_val * 100.0 / (R_loc * T_curr * twf);
        if (i == 0) a.p_stat_landscape[(long long)j * d.pitch + k] = p_val;
        T_prev = T_curr;
        p_prev = p_val;
    }
}

// initWaterWapour (InitValues_Atm.cpp:843-926): the saturation profile's running minimum
// up the column over the dry-top floor
__global__ void __launch_bounds__(128) init_water_kernel(InitArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= d.km) return;
    double q_sat_min = 1.0;
    for (int i = 0; i < d.im; i++) {
        const long long q = idx3(d, i, j, k);
        const double q_s = thermo::saturation_mass_fraction_at(a.t[q] * a.t_0, a.p_stat[q], a.M_nw);
        if (q_s < q_sat_min) q_sat_min = q_s;
        a.c[q] = smax(q_sat_min, a.c_h2o_dry_top);
        a.cloud[q] = 0.0;
    }
}

// ThermoAtm::co2Atmosphere (ThermoAtm.h:873-918): CO2 well mixed in the dry air
__global__ void __launch_bounds__(256) co2_atmosphere_kernel(Dims d, const double* c, double* co2, double f_CO2,
                                                              double co2_scale)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.km) return;
    const long long q = (long long)blockIdx.y * d.pitch + k;
    co2[q] = (1.0 - c[q]) * f_CO2 * co2_scale;
}

__device__ __forceinline__ double cloud_q_sat(const InitArgs& a, double t_u, double p_u, double c, double co2)
{
    const double E_sat = (t_u >= a.t_0) ? thermo::saturation_pressure(t_u) : thermo::sublimation_pressure(t_u);
    return thermo::saturation_mass_fraction(E_sat, p_u, thermo::M_nonwater(c, co2, a.M_bg));
}

// initCloudIce pass 1 (InitValues_Atm.cpp:955-990): one warp per (i, j) row sums the
// vapour in excess of 0.74 q_sat, 32 strided partial sums combined in xor-butterfly order
__global__ void __launch_bounds__(256) cloud_rows_kernel(InitArgs a, double* row_sum)
{
    const Dims& d = a.d;
    const int lane = threadIdx.x & 31;
    const long long row = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= (long long)d.im * d.jm) return;
    const long long base = row * d.pitch;
    double s = 0.0;
    for (int k = lane; k < d.km; k += 32) {
        const long long q = base + k;
        const double t_u = a.t[q] * a.t_0;
        if (t_u >= kTCrit) continue;
        s += smax(0.0, a.c[q] - 0.74 * cloud_q_sat(a, t_u, a.p_stat[q], a.c[q], a.co2[q]));
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) s = s + __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) row_sum[row] = s;
}

// the level's rows added in order: cloud_max[i], floored at 1e-4 (:987-989)
__global__ void cloud_levels_kernel(InitArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.d.im) return;
    double s = 0.0;
    for (int j = 0; j < a.d.jm; j++) s += a.row_sum[(long long)i * a.d.jm + j];
    double cm = s / a.cloud_norm;
    if (cm <= 1e-4) cm = 1e-4;
    a.cloud_max[i] = cm;
}

// initCloudIce pass 2 (:1015-1079): large-scale (and convective) cloud, its ice and
// graupel share below the freezing point, nothing at or above the critical point
__global__ void __launch_bounds__(256) cloud_cells_kernel(InitArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.km) return;
    const int i = blockIdx.y / d.jm;
    const long long q = (long long)blockIdx.y * d.pitch + k;
    const double t_u = a.t[q] * a.t_0;
    const double p_u = a.p_stat[q];
    if (t_u >= kTCrit) {
        a.cloud[q] = 0.0; a.ice[q] = 0.0; a.gr[q] = 0.0;
        return;
    }
    const double q_sat = cloud_q_sat(a, t_u, p_u, a.c[q], a.co2[q]);
    const double x_norm = p_u * a.inv_p_crit;
    double H_crit = a.Hu_cr_max - a.Hu_curv * x_norm * (1.0 - x_norm);
    if (H_crit > 1.0) H_crit = 1.0;
    const double cmax = a.cloud_max[i];
    const double alfa_over_cmax = 1.5 / cmax;
    const double del_q_ls = smax(0.0, a.c[q] - H_crit * q_sat);
    const double cloud_ls = cmax * (1.0 - exp(-alfa_over_cmax * del_q_ls));
    double cloud_conv = 0.0;
    if (a.P_rain[q] > 0.0 && i < d.im - 1) {
        const double del_q_conv = smax(0.0, (a.P_rain[q + d.plane] - a.P_rain[q])
                                            / (a.two_step[i] * a.r_humid[q]) * a.dt_dim[i]);
        cloud_conv = cmax * (1.0 - exp(-alfa_over_cmax * del_q_conv));
    }
    const double cloud_val = cloud_ls + cloud_conv;
    double h_T = 0.0;
    if (t_u < a.t_0) {
        const double ratio = (t_u - a.t_0) / a.det_T_0;
        h_T = 1.0 - exp(-0.5 * ratio * ratio);
    }
    if (t_u <= a.t_00) {
        a.cloud[q] = 0.0; a.ice[q] = 0.0; a.gr[q] = 0.0;
    } else {
        a.cloud[q] = cloud_val;
        a.ice[q] = cloud_val * h_T;
        a.gr[q] = 0.1 * cloud_val * h_T;
    }
}

struct TurbInitArgs {
    Dims d;
    const double* v; const double* w;
    double* tke; double* dis; double* tken; double* disn; double* nue;
    double* vel_star;                    // 2-D [jm][pitch]
    const double* height;                // [im] float layer heights
    double u_0, abl_height, inv_u02, nd_omega, nd_eps, kL;   // kL = Karman * L_atm
    double sqrt_C_nue, c_pow_m025, c_pow_075, tke_wall_den, dis_wall;
    int k_epsilon, set_dis_wall;
};

// TurbulenceAtm::init up to its compute_sources (TurbulenceAtm.h:39-59): compute_vel_star
// (:88-99), init_fields' boundary-layer profiles of tke and omega/epsilon with their
// background floors (:193-265), apply_wall_bc (:109-147); one (j, k) column per thread
__global__ void __launch_bounds__(128) turb_init_kernel(TurbInitArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= d.km) return;
    const int i_surf = (1 < d.im - 1) ? 1 : d.im - 1;
    const long long s = idx3(d, i_surf, j, k);
    const double v_s = a.v[s], w_s = a.w[s];
    const double U_horiz = a.u_0 * sqrt(v_s * v_s + w_s * w_s);
    const double vs = smax(0.05, sqrt(0.002) * U_horiz);
    a.vel_star[(long long)j * d.pitch + k] = vs;
    if (j >= 1 && j < d.jm - 1 && k >= 1 && k < d.km - 1) {
        const double k_bg = 0.01 * vs * vs / a.sqrt_C_nue;
        const double om_bg = a.c_pow_m025 * sqrt(k_bg) / a.kL;
        const double eps_bg = a.c_pow_075 * pow(k_bg, 1.5) / a.kL;
        const double y_mount = a.height[0];
        for (int i = 1; i < d.im - 1; i++) {
            const long long q = idx3(d, i, j, k);
            const double z_i = a.height[i] - y_mount;
            const double z_safe = smax(z_i, 1.0e-6);
            const double z_frac = smin(z_i, a.abl_height) / a.abl_height;
            const double k_abl = vs * vs / a.sqrt_C_nue * pow(1.0 - z_frac, 2.0);
            const double k_phys = smax(k_abl, k_bg);
            double dis_nd;
            if (a.k_epsilon) {
                const double eps_phys = a.c_pow_075 * pow(k_phys, 1.5) / (0.42 * z_safe);
                dis_nd = smax(eps_phys, eps_bg) * a.nd_eps;
            } else {
                const double om_phys = a.c_pow_m025 * sqrt(k_phys) / (0.42 * z_safe);
                dis_nd = smax(om_phys, om_bg) * a.nd_omega;
            }
            const double tke = smax(0.0, k_phys * a.inv_u02);
            const double dis = smax(1.0e-10, dis_nd);
            a.tke[q] = tke; a.tken[q] = tke;
            a.dis[q] = dis; a.disn[q] = dis;
        }
    }
    const long long c0 = idx3(d, 0, j, k);
    a.tke[c0] = vs * vs / a.tke_wall_den;
    a.nue[c0] = 0.0;
    if (a.set_dis_wall) a.dis[c0] = a.dis_wall;
}

}  // namespace

// ThermoAtm::forces (ThermoAtm.h:518-614), the two arrays it shares with the right-hand
// side's outputs (CoriolisForce, BuoyancyForce) in the interior cells; the buoyancy
// reference is the level-mean temperature t_ref, or 1 where none exists yet (t_ref null:
// before the first RK4 step)
__global__ void __launch_bounds__(256) forces_kernel(Dims d, const GeoIJ* geo, const double* sin_w,
                                                     const double* u, const double* v, const double* w,
                                                     const double* t, const double* r_humid, const double* t_ref,
                                                     double* coriolis, double* buoyancy, double two_omega,
                                                     double nontrad_d, double u_0, double r_air, double g)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y, i = row / d.jm, j = row % d.jm;
    if (k < 1 || k >= d.km - 1 || i < 1 || i >= d.im - 1 || j < 1 || j >= d.jm - 1) return;
    const long long q = (long long)row * d.pitch + k;
    const double sinthe = sin_w[j], costhe = geo[row].costhe;
    const double w_ijk = w[q] * u_0;
    const double Cor_r = -nontrad_d * two_omega * sinthe * w_ijk;
    const double Cor_the = two_omega * costhe * w_ijk;
    const double Cor_phi = -two_omega * (costhe * v[q] + nontrad_d * sinthe * u[q]) * u_0;
    coriolis[q] = 1.0 * r_air * sqrt(Cor_r * Cor_r + Cor_the * Cor_the + Cor_phi * Cor_phi);
    buoyancy[q] = 1.0e-3 * 1.0 * r_humid[q] * g * (t[q] - (t_ref ? t_ref[i] : 1.0));
}

void launch_forces(athad_ctx* ctx, const double* t_ref)
{
    const Dims& d = ctx->L.d;
    const athad_params& p = ctx->p;
    forces_kernel<<<dim3((d.km + 255) / 256, d.im * d.jm), 256, 0, ctx->stream>>>(
        d, ctx->geo, ctx->sin_w, ctx->field[ATHAD_U], ctx->field[ATHAD_V], ctx->field[ATHAD_W],
        ctx->field[ATHAD_T], ctx->field[ATHAD_R_HUMID], t_ref, ctx->field[ATHAD_CORIOLIS_FORCE],
        ctx->field[ATHAD_BUOYANCY_FORCE], 2.0 * p.omega, p.coriolis_nontrad ? 1.0 : 0.0, p.u_0, p.r_air, p.g);
}

namespace {

// UtilsAtm::precipitationSum (UtilsAtm.h:51-65)
__global__ void __launch_bounds__(256) precipitation_sum_kernel(Dims d, const double* r, const double* sn,
                                                                const double* gp, const double* cv, double* out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.km) return;
    const long long q = (long long)blockIdx.y * d.pitch + k;
    out[q] = r[q] + sn[q] + gp[q] + cv[q];
}

__global__ void __launch_bounds__(256) copy_top_kernel(Dims d, const double* t, double* t_top)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.km) return;
    t_top[(long long)blockIdx.y * d.pitch + k] = t[idx3(d, d.im - 1, blockIdx.y, k)];
}

// ---- host tables ----------------------------------------------------------------------

// init_tropopause_layers (InitValues_Atm.cpp:330-401)
std::vector<double> tropopause_levels(int im, int jm, const athad_params& p, const athad_init_config& c)
{
    std::vector<double> lev(jm, 0.0);
    const int j_max = jm - 1, j_half = j_max / 2;
    const double x_max = c.tropopause_equator * std::sqrt(c.tropopause_equator / c.tropopause_pole - 1.0);
    const double idx_scale = (double)(im - 1) / p.zeta;
    for (int j = 0; j <= j_half; j++) {
        const double x = x_max * (double)(j_half - j) / (double)j_half;
        const double a = c.tropopause_equator;
        const double h = std::pow(a, 3.0) / (std::pow(a, 2.0) + std::pow(x, 2.0));   // AtomUtils::Agnesi
        double v = 0.0;
        if (h > 0.0 && p.L_atm > 0.0 && p.zeta > 0.0)
            v = std::min(std::max(std::round(idx_scale * std::log(1.0 + h / p.L_atm)), 0.0), (double)(im - 1));
        lev[j] = v;
        lev[j_max - j] = v;
    }
    return lev;
}

// VelocityInitializer::compute (VelocityInitializer.h:23-105): the prescribed cells,
// n_cells_hemisphere per hemisphere with the Hadley edge at 30 * cell_lat_scale degrees,
// as (i, j) tables of u, v, w (non-dimensional)
class VelocityProfile {
public:
    VelocityProfile(int im, int jm, const athad_params& p, const athad_init_config& c,
                    const std::vector<double>& height, const std::vector<double>& trop)
        : im_(im), jm_(jm), p_(p), c_(c), h_(height), trop_(trop),
          u_((size_t)im * jm, 0.0), v_((size_t)im * jm, 0.0), w_((size_t)im * jm, 0.0) {}

    // u, v, w tables, each im*jm, rows j contiguous per level i
    std::vector<double> build()
    {
        const int n = c_.n_cells_hemisphere;
        for (int k = 0; k <= n; k++) {                       // radial velocity on the edges
            const double phi = edge(k);
            const double coeff = radial_coeff(k, phi);
            radial_row(row_n(phi), coeff);
            if (row_s(phi) != row_n(phi)) radial_row(row_s(phi), coeff);
        }
        for (int k = 0; k <= n; k++) anchor(edge(k), edge_amp(k));
        for (int k = 0; k < n; k++) anchor(0.5 * (edge(k) + edge(k + 1)), centre_amp(k));
        chain(u_, anchors(false, false));
        chain(v_, anchors(true, false));
        chain(w_, anchors(true, true));
        const double inv_u_0 = 1.0 / p_.u_0;
        const int jeq = (jm_ - 1) / 2;
        std::vector<double> out((size_t)3 * im_ * jm_);
        for (int i = 0; i < im_; i++)
            for (int j = 0; j <= jeq; j++) {
                const size_t q = (size_t)i * jm_ + j, qr = (size_t)i * jm_ + (jm_ - 1 - j);
                const double u = u_[q] * inv_u_0, w = w_[q] * inv_u_0, v = v_[q] * inv_u_0;
                out[q] = u; out[(size_t)2 * im_ * jm_ + q] = w; out[(size_t)im_ * jm_ + q] = v;
                out[qr] = u; out[(size_t)2 * im_ * jm_ + qr] = w;
                out[(size_t)im_ * jm_ + qr] = (qr == q) ? v : -v;   // v is antisymmetric
            }
        return out;
    }

private:
    struct Amp { double v_trop, v_surf, w_trop, w_surf; bool has_w; };
    int im_, jm_;
    const athad_params& p_;
    const athad_init_config& c_;
    const std::vector<double>& h_;
    const std::vector<double>& trop_;
    std::vector<double> u_, v_, w_;

    double& at(std::vector<double>& a, int i, int j) { return a[(size_t)i * jm_ + j]; }
    double edge(int k) const
    {
        const int n = c_.n_cells_hemisphere;
        if (k <= 0) return 0.0;
        if (n <= 1) return 90.0;
        const double hadley = 30.0 * c_.cell_lat_scale;
        return hadley + (90.0 - hadley) * (double)(k - 1) / (double)(n - 1);
    }
    int row_n(double phi) const
    {
        const int j = (int)std::lround((90.0 - phi) / (180.0 / (double)(jm_ - 1)));
        return std::min(std::max(j, 0), jm_ - 1);
    }
    int row_s(double phi) const { return (jm_ - 1) - row_n(phi); }
    int level(int j) const { return (int)trop_[j]; }
    Amp edge_amp(int k) const
    {
        const int n = c_.n_cells_hemisphere;
        if (k == 0) return {0.0, 0.0, -3.0, -5.0, true};          // equator
        if (k == n) return {0.5, 0.0, 0.0, 0.0, true};            // pole
        if (k == 1) return {0.0, 0.5, 30.0, -1.0, true};          // subtropical edge
        return {-0.2, 0.0, 10.0, 6.0, true};                      // subpolar edges
    }
    Amp centre_amp(int k) const
    {
        const int n = c_.n_cells_hemisphere;
        if (k == 0) return {-3.0, 3.5, 5.0, -7.0, true};          // Hadley
        if (k == n - 1) return {0.5, 0.6, 0.0, 0.0, false};       // polar
        return {4.0, -1.5, 15.0, 10.0, true};                     // Ferrel
    }
    static double radial_coeff(int k, double phi)
    {
        double mag;
        if (phi == 0.0) mag = 0.02894;
        else if (phi == 30.0) mag = 0.02315;
        else if (phi == 60.0) mag = 0.01736;
        else if (phi == 90.0) mag = 0.011574;
        else mag = 0.02894 * (1.0 - phi / 150.0);
        return (k % 2 == 0) ? mag : -mag;
    }
    double amp_scale(bool is_v) const
    {
        const double s = c_.cell_lat_scale;
        if (c_.cell_amp_mode == 1) return s;
        if (c_.cell_amp_mode == 2) return is_v ? s : s * s;
        return 1.0;
    }
    void radial_row(int j, double coeff)                    // init_u
    {
        const int tl = level(j);
        const double top = h_[tl], half = top / 3.0;
        const double up = 3.0 / half, down = 1.0 / half;
        for (int i = 0; i < tl; i++) {
            const double h = h_[i];
            at(u_, i, j) = coeff * ((h < half) ? h * up : (top - h) * down);
        }
    }
    void tangential_row(std::vector<double>& a, bool is_v, int j, double c_trop, double c_sl)   // init_v_or_w
    {
        const int tl = level(j);
        const double inv_top = 1.0 / h_[tl];
        const double s = amp_scale(is_v);
        c_trop *= s;
        c_sl *= s;
        const double slope = (c_trop - c_sl) * inv_top;
        for (int i = 0; i < tl; i++) at(a, i, j) = slope * h_[i] + c_sl;
        if (tl >= im_ - 1) return;
        const double h_top = h_[im_ - 1];
        const double inv_range = 1.0 / (h_top - h_[tl]);
        for (int i = tl; i < im_; i++) at(a, i, j) = c_trop * (h_top - h_[i]) * inv_range;
    }
    void anchor(double phi, const Amp& a)
    {
        const int jn = row_n(phi), js = row_s(phi);
        tangential_row(v_, true, jn, a.v_trop, a.v_surf);
        if (js != jn) tangential_row(v_, true, js, a.v_trop, a.v_surf);
        if (!a.has_w) return;
        tangential_row(w_, false, jn, a.w_trop, a.w_surf);
        if (js != jn) tangential_row(w_, false, js, a.w_trop, a.w_surf);
    }
    std::vector<int> anchors(bool centres, bool skip_polar_centre) const
    {
        const int n = c_.n_cells_hemisphere;
        std::vector<double> phis;
        for (int k = 0; k <= n; k++) phis.push_back(edge(k));
        if (centres)
            for (int k = 0; k < n; k++)
                if (!(skip_polar_centre && k == n - 1)) phis.push_back(0.5 * (edge(k) + edge(k + 1)));
        std::vector<int> rows;
        for (double phi : phis) {
            rows.push_back(row_n(phi));
            if (row_s(phi) != row_n(phi)) rows.push_back(row_s(phi));
        }
        std::sort(rows.begin(), rows.end());
        rows.erase(std::unique(rows.begin(), rows.end()), rows.end());
        return rows;
    }
    void chain(std::vector<double>& a, const std::vector<int>& rows)   // form_diagonals between anchors
    {
        for (size_t q = 0; q + 1 < rows.size(); q++) {
            const int s = rows[q], e = rows[q + 1];
            if (e <= s) continue;
            const double inv_range = 1.0 / (double)(e - s);
            for (int i = 0; i < im_; i++) {
                const double a0 = at(a, i, s);
                const double slope = (at(a, i, e) - a0) * inv_range;
                for (int j = s; j < e; j++) at(a, i, j) = slope * (double)(j - s) + a0;
            }
        }
    }
};

}  // namespace

}  // namespace athad

void athad_default_init_config(athad_init_config* c)
{
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->struct_size = sizeof(athad_init_config);
    c->n_cells_hemisphere = 5;      // cli/config_cond.xml:65
    c->cell_amp_mode = 0;           // :64
    c->t_surf_equator = 513.15;     // :21
    c->t_surf_pole = 503.15;        // :22
    c->tropopause_equator = 207000.0;   // :62
    c->tropopause_pole = 195000.0;  // :61
    c->cell_lat_scale = 0.11;       // :63
    c->co2_scale = 1.0;             // :107
    c->vel_star_init = 0.4;         // UtilsAtm.h:388 (resetArrays)
    // m_comp's mass fractions (AtmMixture::resolve) of x = (H2O .5578, CO2 .4109, N2 .0313)
    const double x[8] = {0.5578, 0.4109, 0.0313, 0.0, 0.0, 0.0, 0.0, 0.0};
    const double m_H2O = x[0] * thermo::M_H2O, m_CO2 = x[1] * thermo::M_CO2;
    const double m_bg = x[2] * 0.028014 + x[3] * 0.016043 + x[4] * 0.017031
                      + x[5] * 0.002016 + x[6] * 0.028010 + x[7] * 0.064066;
    const double M_mean = m_H2O + m_CO2 + m_bg;
    c->q_CO2 = m_CO2 / M_mean;
    c->q_bg = m_bg / M_mean;
}

athad_status athad_forces(athad_ctx* ctx)
{
    if (!ctx) return ATHAD_ERR_INVALID;
    athad::launch_forces(ctx, ctx->level_mean_valid ? ctx->prof[ATHAD_PROF_T_REF_LEVEL] : nullptr);
    ATHAD_CHECK_LAUNCH(ctx, "forces");
    return ATHAD_OK;
}

athad_status athad_initial_state(athad_ctx* ctx, const athad_init_config* cfg)
{
    using namespace athad;
    if (!ctx) return ATHAD_ERR_INVALID;
    if (!cfg || cfg->struct_size != sizeof(athad_init_config))
        return fail(ctx, ATHAD_ERR_INVALID, "initial_state: bad athad_init_config");
    if (cfg->n_cells_hemisphere < 1 || cfg->n_cells_hemisphere > 30)
        return fail(ctx, ATHAD_ERR_INVALID, "initial_state: n_cells_hemisphere outside [1, 30]");
    if (!(cfg->tropopause_pole > 0.0) || !(cfg->tropopause_equator >= cfg->tropopause_pole))
        return fail(ctx, ATHAD_ERR_INVALID, "initial_state: tropopause heights need equator >= pole > 0");
    if (!(cfg->cell_lat_scale > 0.0) || !(cfg->co2_scale >= 0.0))
        return fail(ctx, ATHAD_ERR_INVALID, "initial_state: bad cell_lat_scale or co2_scale");
    const athad_params& p = ctx->p;
    const Dims& d = ctx->L.d;
    const int im = d.im, jm = d.jm, km = d.km;
    cudaStream_t st = ctx->stream;
    athad_status s = ATHAD_OK;
#define ATHAD_TRY(expr) do { s = (expr); if (s != ATHAD_OK) return s; } while (0)
    const dim3 rows_grid((km + 255) / 256, im * jm), cols_grid((km + 127) / 128, jm);

    // UtilsAtm::resetArrays (UtilsAtm.h:364-451): zero, except t, tn, t_eq, co2n and the
    // moist static energies = 1, HumidityRel = 100, vel_star = 0.4
    for (int f = 0; f < ATHAD_NFIELDS; f++)
        ATHAD_TRY(cuda_check(ctx, cudaMemsetAsync(ctx->field[f], 0, ctx->L.field_elems * sizeof(double), st), "reset"));
    for (int f : {ATHAD_T, ATHAD_TN, ATHAD_T_EQ, ATHAD_CO2N, ATHAD_MC_S, ATHAD_MC_S_U, ATHAD_MC_S_D})
        launch_fill(d, ctx->field[f], 1.0, st);
    launch_fill(d, ctx->field[ATHAD_HUMIDITY_REL], 100.0, st);
    for (int f = 0; f < ATHAD_NFIELDS2D; f++)
        ATHAD_TRY(cuda_check(ctx, cudaMemsetAsync(ctx->f2d[f], 0, ctx->L.f2d_elems * sizeof(double), st), "reset 2-D"));
    {
        Dims d2 = d;
        d2.fstride = (long long)ctx->L.f2d_elems;   // a 2-D field: jm rows of pitch
        launch_fill(d2, ctx->f2d[ATHAD_2D_VEL_STAR], cfg->vel_star_init, st);
    }
    for (int f = 0; f < ATHAD_NPROFILES; f++)
        ATHAD_TRY(cuda_check(ctx, cudaMemsetAsync(ctx->prof[f], 0, (size_t)im * sizeof(double), st), "reset profiles"));
    ATHAD_CHECK_LAUNCH(ctx, "initial_state reset");
    ctx->q_co2_ref = ctx->q_h2o_ref = ctx->q_h2o_fixed_ref = -1.0;   // co2Column(true), waterBudget(true) below
    ctx->air_levels.clear();
    ctx->h2o_levels.clear();
    ctx->level_mean_valid = false;

    // host tables: tropopause levels, velocity profiles, surface temperature, layer steps
    const std::vector<double>& h = ctx->height_h;
    const std::vector<double> trop = tropopause_levels(im, jm, p, *cfg);
    ATHAD_TRY(athad_set_tropopause_layers(ctx, trop.data(), jm));
    std::vector<double> tab = VelocityProfile(im, jm, p, *cfg, h, trop).build();
    const size_t n_uvw = tab.size();
    std::vector<double> Ts(jm), dz(im, 0.0), dt_dim(im), two_step(im);
    const double d_j_half = 0.5 * (jm - 1);
    for (int j = 0; j <= (jm - 1) / 2; j++) {   // the parabola x^2 - 2x (AtomUtils::parabola), mirrored
        const double r = (double)j / d_j_half;
        Ts[j] = (cfg->t_surf_pole - cfg->t_surf_equator) * (r * r - 2.0 * r) + cfg->t_surf_pole;
        Ts[jm - 1 - j] = Ts[j];
    }
    for (int i = 1; i < im; i++) dz[i] = (double)((float)h[i] - (float)h[i - 1]);
    for (int i = 0; i < im - 1; i++) {            // initCloudIce's per-level steps (:995-1006)
        const double step = (double)((float)h[i + 1] - (float)h[i]);
        dt_dim[i] = step / 1.6;
        two_step[i] = 2.0 * step;
    }
    dt_dim[im - 1] = dt_dim[im - 2];
    two_step[im - 1] = two_step[im - 2];
    // the tables go to the upload staging field, which nothing else reads during the call
    double* stage = ctx->upload_stage;
    double* d_tab = stage;
    double* d_Ts = stage + n_uvw;
    double* d_dz = d_Ts + jm;
    double* d_dt_dim = d_dz + im;
    double* d_two_step = d_dt_dim + im;
    if (n_uvw + (size_t)jm + 3 * (size_t)im > ctx->L.field_elems)
        return fail(ctx, ATHAD_ERR_INVALID, "initial_state: grid too small for the table staging");
    ATHAD_TRY(cuda_check(ctx, cudaMemcpyAsync(d_tab, tab.data(), n_uvw * sizeof(double), cudaMemcpyHostToDevice, st), "velocity tables"));
    ATHAD_TRY(cuda_check(ctx, cudaMemcpyAsync(d_Ts, Ts.data(), jm * sizeof(double), cudaMemcpyHostToDevice, st), "Ts"));
    ATHAD_TRY(cuda_check(ctx, cudaMemcpyAsync(d_dz, dz.data(), im * sizeof(double), cudaMemcpyHostToDevice, st), "dz"));
    ATHAD_TRY(cuda_check(ctx, cudaMemcpyAsync(d_dt_dim, dt_dim.data(), im * sizeof(double), cudaMemcpyHostToDevice, st), "dt_dim"));
    ATHAD_TRY(cuda_check(ctx, cudaMemcpyAsync(d_two_step, two_step.data(), im * sizeof(double), cudaMemcpyHostToDevice, st), "two_step"));

    // VelocityInitializer::compute; bcVelSurfSur (nothing without land); damp_wiggles of u, v, w
    init_velocity_kernel<<<rows_grid, 256, 0, st>>>(d, d_tab, ctx->field[ATHAD_U], ctx->field[ATHAD_V],
                                                    ctx->field[ATHAD_W]);
    ATHAD_CHECK_LAUNCH(ctx, "initial_state velocities");
    for (int f : {ATHAD_U, ATHAD_V, ATHAD_W}) ATHAD_TRY(athad_damp_wiggles(ctx, (athad_field)f));

    InitArgs a;
    std::memset(&a, 0, sizeof a);
    a.d = d;
    a.t = ctx->field[ATHAD_T]; a.p_stat = ctx->field[ATHAD_P_STAT]; a.r_dry = ctx->field[ATHAD_R_DRY];
    a.r_humid = ctx->field[ATHAD_R_HUMID]; a.c = ctx->field[ATHAD_C]; a.co2 = ctx->field[ATHAD_CO2];
    a.cloud = ctx->field[ATHAD_CLOUD]; a.ice = ctx->field[ATHAD_ICE]; a.gr = ctx->field[ATHAD_GR];
    a.P_rain = ctx->field[ATHAD_P_RAIN];
    a.p_stat_landscape = ctx->f2d[ATHAD_2D_P_STAT_LANDSCAPE];
    a.Ts = d_Ts; a.dz = d_dz; a.dt_dim = d_dt_dim; a.two_step = d_two_step;
    a.t_0 = p.t_0; a.r_air = p.r_air; a.R_mix = p.R_mix; a.R_bg = p.R_bg; a.M_bg = p.M_bg; a.g = p.g;
    a.t_skin = p.t_skin; a.c_h2o_dry_top = p.c_h2o_dry_top; a.t_00 = p.t_00;
    a.M_nw = thermo::M_nonwater(p.c_0, p.co2_0, p.M_bg);

    // initTemperatureData (InitValues_Atm.cpp:466-620); damp_wiggles(t); the lid snapshot
    init_temperature_kernel<<<cols_grid, 128, 0, st>>>(a);
    ATHAD_CHECK_LAUNCH(ctx, "initial_state temperature");
    ATHAD_TRY(athad_damp_wiggles(ctx, ATHAD_T));
    copy_top_kernel<<<dim3((km + 255) / 256, jm), 256, 0, st>>>(d, ctx->field[ATHAD_T], ctx->f2d[ATHAD_2D_T_TOP_INIT]);
    ATHAD_CHECK_LAUNCH(ctx, "initial_state lid");

    // initWaterWapour; two passes of co2Atmosphere and densities(true) (cAtmosphereModel.cpp:563-568)
    init_water_kernel<<<cols_grid, 128, 0, st>>>(a);
    ATHAD_CHECK_LAUNCH(ctx, "initial_state water");
    const double f_CO2 = (cfg->q_CO2 + cfg->q_bg > 0.0) ? cfg->q_CO2 / (cfg->q_CO2 + cfg->q_bg)
                                                        : p.co2_0 * cfg->co2_scale;
    for (int pass = 0; pass < 2; pass++) {
        co2_atmosphere_kernel<<<rows_grid, 256, 0, st>>>(d, ctx->field[ATHAD_C], ctx->field[ATHAD_CO2], f_CO2,
                                                         cfg->co2_scale);
        ATHAD_CHECK_LAUNCH(ctx, "initial_state co2");
        ATHAD_TRY(athad_densities(ctx, 1));
    }

    // initCloudIce (InitValues_Atm.cpp:930-1117): the Earth parabola of critical humidity
    // anchored to the surface pressure
    a.row_sum = ctx->row_sum;
    a.cloud_max = ctx->row_cnt;
    a.Hu_cr_max = 1.0;
    const double x_mid = (0.55 * p.p_0) / p.p_0;
    a.Hu_curv = (1.0 - 0.8) / (x_mid * (1.0 - x_mid));
    a.inv_p_crit = 1.0 / p.p_0;
    a.det_T_0 = p.t_0;
    a.cloud_norm = (double)((jm - 1) * (km - 1));
    cloud_rows_kernel<<<(unsigned)(((long long)im * jm + 7) / 8), 256, 0, st>>>(a, ctx->row_sum);
    cloud_levels_kernel<<<(im + 127) / 128, 128, 0, st>>>(a);
    cloud_cells_kernel<<<rows_grid, 256, 0, st>>>(a);
    ATHAD_CHECK_LAUNCH(ctx, "initial_state cloud");

    // SaturationAdjustment and damp_wiggles(ice, c, cloud) (cAtmosphereModel.cpp:574-577)
    ATHAD_TRY(athad_saturation_adjust(ctx));
    for (int f : {ATHAD_ICE, ATHAD_C, ATHAD_CLOUD}) ATHAD_TRY(athad_damp_wiggles(ctx, (athad_field)f));
    // the configured ice scheme (the CategoryIceScheme switch) and damp_wiggles(P_rain,
    // P_snow) (:581-596)
    ATHAD_TRY(athad_ice_scheme(ctx));
    for (int f : {ATHAD_P_RAIN, ATHAD_P_SNOW}) ATHAD_TRY(athad_damp_wiggles(ctx, (athad_field)f));
    // MoistConvection(iter_n = 0) and the smoothing of its outputs (:599-608)
    ATHAD_TRY(athad_moist_convection(ctx, 0));
    for (int f : {ATHAD_P_CONV, ATHAD_E_U, ATHAD_M_U, ATHAD_Q_V_U, ATHAD_Q_C_U, ATHAD_E_D, ATHAD_M_D, ATHAD_Q_V_D})
        ATHAD_TRY(athad_damp_wiggles(ctx, (athad_field)f));

    // TurbulenceAtm::init, ::run and the smoothing of the turbulence fields (:612-624)
    {
        TurbInitArgs t;
        std::memset(&t, 0, sizeof t);
        t.d = d;
        t.v = ctx->field[ATHAD_V]; t.w = ctx->field[ATHAD_W];
        t.tke = ctx->field[ATHAD_TKE]; t.dis = ctx->field[ATHAD_DIS];
        t.tken = ctx->field[ATHAD_TKEN]; t.disn = ctx->field[ATHAD_DISN]; t.nue = ctx->field[ATHAD_NUE];
        t.vel_star = ctx->f2d[ATHAD_2D_VEL_STAR];
        t.height = ctx->height;
        const double C_nue = 0.028;
        t.u_0 = p.u_0; t.abl_height = p.abl_height;
        t.inv_u02 = 1.0 / (p.u_0 * p.u_0);
        t.nd_omega = p.L_atm / p.u_0;
        t.nd_eps = p.L_atm / (p.u_0 * p.u_0 * p.u_0);
        t.kL = 0.42 * p.L_atm;
        t.sqrt_C_nue = std::sqrt(C_nue);
        t.c_pow_m025 = std::pow(C_nue, -0.25);
        t.c_pow_075 = std::pow(C_nue, 0.75);
        t.tke_wall_den = std::sqrt(C_nue) * p.u_0 * p.u_0;
        const double y1_safe = (ctx->layer_height1 < 1.0e-6) ? 1.0e-6 : ctx->layer_height1;
        t.k_epsilon = (p.turb_model == ATHAD_TURB_K_EPSILON);
        t.set_dis_wall = 1;
        if (p.turb_model == ATHAD_TURB_K_EPSILON) t.dis_wall = 0.0;
        else if (p.turb_model == ATHAD_TURB_K_OMEGA) t.dis_wall = 6.0 * 1.5e-5 / (0.075 * y1_safe * y1_safe) * t.nd_omega;
        else t.dis_wall = 60.0 * 1.5e-5 / (0.0333 * y1_safe * y1_safe) * t.nd_omega;
        turb_init_kernel<<<cols_grid, 128, 0, st>>>(t);
        ATHAD_CHECK_LAUNCH(ctx, "initial_state turbulence");
    }
    ATHAD_TRY(athad_turbulence_run(ctx));   // init's compute_sources and clamp_nue
    ATHAD_TRY(athad_turbulence_run(ctx));   // run()
    for (int f : {ATHAD_TKE, ATHAD_DIS, ATHAD_NUE, ATHAD_PROD, ATHAD_TKE_SOURCE, ATHAD_DIS_SOURCE})
        ATHAD_TRY(athad_damp_wiggles(ctx, (athad_field)f));

    // precipitationSum, co2Atmosphere, co2Column(true), waterBudget(true), densities(),
    // waterVapourEvaporation, latentSensibleHeat (:627-638)
    precipitation_sum_kernel<<<rows_grid, 256, 0, st>>>(d, ctx->field[ATHAD_P_RAIN], ctx->field[ATHAD_P_SNOW],
                                                        ctx->field[ATHAD_P_GRAUPEL], ctx->field[ATHAD_P_CONV],
                                                        ctx->field[ATHAD_PRECIPITATION]);
    co2_atmosphere_kernel<<<rows_grid, 256, 0, st>>>(d, ctx->field[ATHAD_C], ctx->field[ATHAD_CO2], f_CO2,
                                                     cfg->co2_scale);
    ATHAD_CHECK_LAUNCH(ctx, "initial_state precipitation, co2");
    athad_budget_report rep;
    ATHAD_TRY(athad_co2_column(ctx, &rep));
    ATHAD_TRY(athad_water_budget(ctx, &rep, nullptr));
    ATHAD_TRY(athad_densities(ctx, 0));
    launch_forces(ctx, nullptr);   // no level mean exists yet
    ATHAD_CHECK_LAUNCH(ctx, "initial_state forces");
    ATHAD_TRY(athad_water_vapour_evaporation(ctx));
    ATHAD_TRY(athad_latent_sensible_heat(ctx));

    // bcRadius, bcTheta, bcPhi, bcScalarSurfSur, bcSolidGround: no turbulence wall values
    // here (:651-656); the initial projection (:665); storeIntermediateData3D (:667); the
    // Held-Suarez target t_eq := t (:750-753)
    ATHAD_TRY(boundary_conditions(ctx, 0));
    ATHAD_TRY(athad_project_initial_velocity(ctx, 200, 0));
    ATHAD_TRY(athad_store_n_level(ctx));
    ATHAD_TRY(cuda_check(ctx, cudaMemcpyAsync(ctx->field[ATHAD_T_EQ], ctx->field[ATHAD_T],
                                              ctx->L.field_elems * sizeof(double), cudaMemcpyDeviceToDevice, st),
                         "t_eq"));
#undef ATHAD_TRY
    return ATHAD_OK;
}
