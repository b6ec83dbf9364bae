// k_turb.cu - TurbulenceAtm::run (TurbulenceAtm.h:62-79) of the ATHAD_COND atmosphere on
// sm_100a, flat terrain:
//
//   turb_vel_star_kernel   compute_vel_star (:88-99): friction velocity per (j, k) column
//                          from the wind of the first air cell, i = 1;
//   turb_sources_kernel    compute_sources (:323-476) with the closure of the configured
//                          model: compute_k_epsilon (:481-528), compute_k_omega (:533-650)
//                          or compute_k_omega_SST (:656-772): prod, nue, tke_source and
//                          dis_source of every interior cell;
//   turb_finish_kernel     the floors each cell applies to its own tke/dis (:352-353,
//                          :459-460) and clamp_nue (:271-295) over the whole grid.
//
// The reference sweeps in place, so a cell reads the already-floored tke/dis of the
// neighbours its loop order visited first.  Here every cell reads the state before the
// call and the floors follow in a second pass: the result does not depend on an order,
// and a mirror-symmetric state stays mirror-symmetric.  The two agree wherever the floors
// do not bind at a neighbour (they bind where the RK4 step left tke below the column's
// background k_bg).  Compiled without fused multiply-add: the operations round as the
// reference's do; exp, pow and tanh are CUDA's.
#include "kernels.cuh"

namespace athad {

namespace {

constexpr double kCNue = 0.028;       // TurbulenceAtm.h:158
constexpr double kDisMin = 1.0e-10;   // :161
constexpr double kNueAir = 1.5e-5;    // constructor default (:28)

__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double dclamp(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

// background tke floor of a column, :329-330
__device__ __forceinline__ double k_bg_of(const TurbArgs& a, double vs)
{
    return 0.01 * vs * vs / (sqrt(kCNue) * a.u_0 * a.u_0);
}

__global__ void __launch_bounds__(128) turb_vel_star_kernel(TurbArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= d.km) return;
    const int i_surf = (1 < d.im - 1) ? 1 : d.im - 1;
    const double v_s = a.v[idx3(d, i_surf, j, k)];
    const double w_s = a.w[idx3(d, i_surf, j, k)];
    const double U_horiz = a.u_0 * sqrt(v_s * v_s + w_s * w_s);
    a.vel_star[(long long)j * d.pitch + k] = dmax(0.05, sqrt(0.002) * U_horiz);
}

template <int MODEL>
__global__ void __launch_bounds__(128) turb_sources_kernel(TurbArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (i < 1 || i >= d.im - 1 || j < 1 || j >= d.jm - 1 || k < 1 || k >= d.km - 1) return;
    const long long c = idx3(d, i, j, k);
    const long long sI = d.plane, sJ = d.pitch;
    const TurbLevel L = a.lev[i];
    const double rm = L.rm, exp_rm = L.exp_rm;
    double sinthe = a.sin_w[j];
    if (sinthe == 0.0) sinthe = 1.0e-5;
    const double rmsinthe = rm * sinthe;
    const double inv_2dr = a.inv_2dr, inv_2dthe = a.inv_2dthe, inv_2dphi = a.inv_2dphi;
    const double inv_rm2dthe = inv_2dthe / L.rmet;
    const double inv_rmsinthe2dphi = inv_2dphi / (L.rmet * sinthe);
    const double* u = a.u;
    const double* v = a.v;
    const double* w = a.w;
    const double dudr = (u[c + sI] - u[c - sI]) * inv_2dr * exp_rm;
    const double dvdr = (v[c + sI] - v[c - sI]) * inv_2dr * exp_rm;
    const double dwdr = (w[c + sI] - w[c - sI]) * inv_2dr * exp_rm;
    const double dudthe = (u[c + sJ] - u[c - sJ]) * inv_rm2dthe;
    const double dvdthe = (v[c + sJ] - v[c - sJ]) * inv_rm2dthe;
    const double dwdthe = (w[c + sJ] - w[c - sJ]) * inv_rm2dthe;
    const double dudphi = (u[c + 1] - u[c - 1]) * inv_rmsinthe2dphi;
    const double dvdphi = (v[c + 1] - v[c - 1]) * inv_rmsinthe2dphi;
    const double dwdphi = (w[c + 1] - w[c - 1]) * inv_rmsinthe2dphi;

    const double* T = a.tke;
    const double* D = a.dis;
    const double tke = dmax(0.0, T[c]);          // the entry floors of the cell, :352-353
    const double dis = dmax(kDisMin, D[c]);
    const double dtkedr = (T[c + sI] - T[c - sI]) * inv_2dr * exp_rm;
    const double ddisdr = (D[c + sI] - D[c - sI]) * inv_2dr * exp_rm;

    const double nue_max = a.nue_max;
    double cnue;
    {
        const double dis_here = dmax(dis, kDisMin);
        const double tke_here = dmax(tke, 0.0);
        cnue = (MODEL == ATHAD_TURB_K_EPSILON) ? kCNue * tke_here * tke_here / dis_here : tke_here / dis_here;
        cnue = dmin(cnue, nue_max);
    }
    const double der = 0.66667 * (dudr + dvdthe + dwdphi);
    const double prod = dmax(0.0,
          (cnue * (2.0 * dudr - der) - 0.66667 * tke) * dudr
        + (cnue * (dudthe + dvdr)) * dudthe
        + (cnue * (dudphi + dwdr)) * dudphi
        + (cnue * (2.0 * dvdthe - der) - 0.66667 * tke) * dvdthe
        + (cnue * (dvdr + dudthe)) * dvdr
        + (cnue * (dvdphi + dwdthe)) * dvdphi
        + (cnue * (2.0 * dwdphi - der) - 0.66667 * tke) * dwdphi
        + (cnue * (dwdr + dudphi)) * dwdr
        + (cnue * (dwdthe + dvdphi)) * dwdthe);
    a.prod[c] = prod;
    const double W12 = dudthe - dvdr;
    const double W13 = dudphi - dwdr;
    const double W23 = dvdphi - dwdthe;
    const double Omega = sqrt(W12 * W12 + W13 * W13 + W23 * W23);

    double nue, tke_source, dis_source;
    if (MODEL == ATHAD_TURB_K_EPSILON) {
        const double y_phys = dmax(L.height - a.y_mount, a.L_atm);
        const double y_star = y_phys / a.L_atm;
        nue = kCNue * tke * tke / dmax(dis, kDisMin);
        const double d_plus = y_phys * a.vel_star[(long long)j * d.pitch + k] / kNueAir;
        const double f_nue = 1.0 - exp(-0.0115 * d_plus);
        const double Re_T = tke * tke * a.u_0 * a.L_atm / dmax(dis * kNueAir, kDisMin * kNueAir);
        const double f_2 = 1.0 - 0.4 / 1.8 * exp(-Re_T * Re_T / 36.0);
        nue *= f_nue;
        const double y_star2 = y_star * y_star;
        const double L_k = -2.0 * tke / y_star2;
        const double L_w = -2.0 * dis / y_star2 * exp(-d_plus / 2.0);
        const double P_k = prod, Y_k = dis;
        const double tke_safe = dmax(tke, kDisMin);
        const double P_w = 1.35 * dis / tke_safe * P_k;
        const double Y_w = 1.80 * f_2 * dis * dis / tke_safe;
        tke_source = P_k - Y_k + L_k / a.re_turb;
        dis_source = P_w - Y_w + L_w / a.re_turb;
    } else {
        // the theta and phi gradients of tke/dis the closures form with 1/rm (:593-596,
        // :722-725)
        const double dtkedthe_neu = (T[c + sJ] - T[c - sJ]) / (rm * 2.0 * a.dthe);
        const double ddisdthe_neu = (D[c + sJ] - D[c - sJ]) / (rm * 2.0 * a.dthe);
        const double dtkedphi_neu = (T[c + 1] - T[c - 1]) / (rmsinthe * 2.0 * a.dphi);
        const double ddisdphi_neu = (D[c + 1] - D[c - 1]) / (rmsinthe * 2.0 * a.dphi);
        const double cross = dtkedr * ddisdr + dtkedthe_neu * ddisdthe_neu + dtkedphi_neu * ddisdphi_neu;
        if (MODEL == ATHAD_TURB_K_OMEGA) {
            const double bet_star = 0.09, gam = 0.52, C_lim = 0.875, bet_0 = 0.0708;
            const double dudr_u = (u[c + sI] - u[c - sI]) / (2.0 * a.dr) / (rm + 1.0);
            const double dvdthe_u = (v[c + sJ] - v[c - sJ]) / (rm * 2.0 * a.dthe);
            const double dwdphi_u = (w[c + 1] - w[c - 1]) / (rmsinthe * 2.0 * a.dphi);
            const double dudthe_u = (u[c + sJ] - u[c - sJ]) / (rm * 2.0 * a.dthe);
            const double dudphi_u = (u[c + 1] - u[c - 1]) / (rmsinthe * 2.0 * a.dphi);
            const double dvdr_u = (v[c + sI] - v[c - sI]) / (2.0 * a.dr) / (rm + 1.0);
            const double dwdr_u = (w[c + sI] - w[c - sI]) / (2.0 * a.dr) / (rm + 1.0);
            const double dvdphi_u = (v[c + 1] - v[c - 1]) / (rmsinthe * 2.0 * a.dphi);
            const double dwdthe_u = (w[c + sJ] - w[c - sJ]) / (rm * 2.0 * a.dthe);
            const double S11 = dudr_u, S22 = dvdthe_u, S33 = dwdphi_u;
            const double S12 = 0.5 * (dudthe_u + dvdr_u);
            const double S13 = 0.5 * (dudphi_u + dwdr_u);
            const double S23 = 0.5 * (dvdphi_u + dwdthe_u);
            const double S_mag = sqrt(2.0 * (S11 * S11 + S22 * S22 + S33 * S33
                                           + 2.0 * (S12 * S12 + S13 * S13 + S23 * S23)));
            const double w_hat = dmax(dis, C_lim * S_mag / sqrt(bet_star));
            const double sig_d = (cross <= 0.0) ? 0.0 : 0.125;
            const double chi_w = fabs(Omega * Omega * S_mag / pow(bet_star * dmax(dis, 1.0e-20), 3.0));
            const double f_bet = (1.0 + 85.0 * chi_w) / (1.0 + 100.0 * chi_w);
            const double bet_wc = bet_0 * f_bet;
            nue = tke / dmax(w_hat, 1.0e-20);
            const double P_k = dmin(prod, 20.0 * bet_star * tke * dis);
            const double Y_k = bet_star * tke * dis;
            const double P_w = gam * dis / dmax(tke, 1.0e-20) * P_k;
            const double Y_w = bet_wc * dis * dis;
            const double D_w = sig_d / dmax(dis, 1.0e-20) * cross;
            tke_source = P_k - Y_k;
            dis_source = P_w - Y_w + D_w;
        } else {
            const double a1 = 0.31, bet_star = 0.09, bet1 = 0.0333, bet2 = 0.0368;
            const double gam1 = 0.413, gam2 = 0.2, sig_w2 = 1.168;
            const double nue_air_nd = kNueAir / (a.u_0 * a.L_atm);
            const double y_phys = dmax(L.height - a.y_mount, 1.0e-6);
            const double y_star = y_phys / a.L_atm;
            const double CD_kw = dmax(2.0 * sig_w2 / dmax(dis, 1.0e-20) * cross, 1.0e-20);
            const double dis_safe = dmax(dis, 1.0e-20);
            const double arg1 = dmin(
                dmax(sqrt(tke) / (bet_star * dis_safe * y_star),
                     500.0 * nue_air_nd / (y_star * y_star * dis_safe)),
                4.0 * sig_w2 * tke / (CD_kw * y_star * y_star));
            const double arg2 = dmax(
                2.0 * sqrt(tke) / (bet_star * dis_safe * y_star),
                500.0 * nue_air_nd / (y_star * y_star * dis_safe));
            const double F1 = tanh(pow(arg1, 4.0));
            const double F2 = tanh(pow(arg2, 2.0));
            nue = a1 * tke / dmax(a1 * dis_safe, Omega * F2);
            const double tke_safe = dmax(tke, 1.0e-20);
            const double P_k = dmin(prod, 20.0 * bet_star * tke_safe * dis_safe);
            const double Y_k = bet_star * tke_safe * dis_safe;
            const double P_w = (F1 * gam1 + (1.0 - F1) * gam2) * P_k * dis_safe / tke_safe;
            const double Y_w = (F1 * bet1 + (1.0 - F1) * bet2) * dis_safe * dis_safe;
            const double D_w = 2.0 * (1.0 - F1) * sig_w2 / dis_safe * cross;
            tke_source = P_k - Y_k;
            dis_source = P_w - Y_w + D_w;
        }
    }
    // the end of the cell, :455-472, with the floored values the second pass stores
    const double tke_fin = dmax(k_bg_of(a, a.vel_star[(long long)j * d.pitch + k]), tke);
    const double dis_fin = dmax(kDisMin, dis);
    a.nue[c] = dclamp(nue, 0.0, nue_max);
    const double dis_src_max = 20.0 * dis_fin * dis_fin;
    a.dis_source[c] = dclamp(dis_source, -dis_src_max, dis_src_max);
    const double tke_src_max = 20.0 * tke_fin * dis_fin;
    a.tke_source[c] = dclamp(tke_source, -tke_src_max, tke_src_max);
}

// the floors of tke/dis in the interior and clamp_nue everywhere
__global__ void __launch_bounds__(128) turb_finish_kernel(TurbArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= d.km || j >= d.jm) return;
    const long long c = idx3(d, i, j, k);
    if (i >= 1 && i < d.im - 1 && j >= 1 && j < d.jm - 1 && k >= 1 && k < d.km - 1) {
        const double k_bg = k_bg_of(a, a.vel_star[(long long)j * d.pitch + k]);
        a.tke[c] = dmax(k_bg, dmax(0.0, a.tke[c]));
        a.dis[c] = dmax(kDisMin, a.dis[c]);
    }
    a.nue[c] = dclamp(a.nue[c], 0.0, a.nue_max) * a.lev[i].nue_fac;
}

}  // namespace

void launch_turbulence_run(const TurbArgs& a, cudaStream_t st)
{
    const Dims& d = a.d;
    turb_vel_star_kernel<<<dim3((d.km + 127) / 128, d.jm), 128, 0, st>>>(a);
    const dim3 block(32, 4), grid((d.km + 31) / 32, (d.jm + 3) / 4, d.im);
    switch (a.turb_model) {
        case ATHAD_TURB_K_EPSILON: turb_sources_kernel<ATHAD_TURB_K_EPSILON><<<grid, block, 0, st>>>(a); break;
        case ATHAD_TURB_K_OMEGA: turb_sources_kernel<ATHAD_TURB_K_OMEGA><<<grid, block, 0, st>>>(a); break;
        default: turb_sources_kernel<ATHAD_TURB_K_OMEGA_SST><<<grid, block, 0, st>>>(a); break;
    }
    turb_finish_kernel<<<grid, block, 0, st>>>(a);
}

}  // namespace athad
