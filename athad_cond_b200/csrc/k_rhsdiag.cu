// k_rhsdiag.cu - the right-hand side's diagnostic outputs (RHS_Atm_Turb.cpp:447-491,
// 1031-1057) on sm_100a: the acting forces (Coriolis, buoyancy, pressure gradient), the
// heat diagnostics Q_Latent and Q_Sensible, and on momentum-budget steps the six terms each
// of rhs_v and rhs_w.  The reference writes them in every right-hand-side call; nothing in
// the model reads them back, so here they are formed only on the steps whose output is
// wanted (athad_step_scalars.write_diagnostics), by one launch after the last stage that
// reads that stage's input state - the state the reference's last call sees - and forms
// each term with the operations and order of the FP64 stage kernel (k_rk4.cu) and the
// reference.  Compiled without fused multiply-add, as k_rk4.cu.
#include "kernels.cuh"
#include "thermo.cuh"

namespace athad {

namespace {

template <typename TY>
struct StarD {
    double c, ip, im, jp, jm, kp, km;
};

template <typename TY>
__device__ __forceinline__ StarD<TY> star(const TY* __restrict__ F, long long c, long long sI, long long sJ)
{
    StarD<TY> s;
    s.c = (double)F[c];
    s.ip = (double)F[c + sI]; s.im = (double)F[c - sI];
    s.jp = (double)F[c + sJ]; s.jm = (double)F[c - sJ];
    s.kp = (double)F[c + 1];  s.km = (double)F[c - 1];
    return s;
}

__device__ __forceinline__ double minmod_d(double a, double b)
{
    return (a * b <= 0.0) ? 0.0 : (fabs(a) < fabs(b) ? a : b);
}

template <typename TY> __device__ __forceinline__ const TY* ycol(const RhsDiagArgs& a, int n);
template <> __device__ __forceinline__ const double* ycol<double>(const RhsDiagArgs& a, int n) { return a.Y64[n]; }
template <> __device__ __forceinline__ const float* ycol<float>(const RhsDiagArgs& a, int n) { return a.Y32[n]; }

template <typename TY>
__global__ void __launch_bounds__(128) rhs_diag_kernel(const RhsDiagArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int i = blockIdx.z;
    if (k < 1 || k >= d.km - 1 || j < 1 || j >= d.jm - 1 || i < 1 || i >= d.im - 1) return;
    const long long c = idx3(d, i, j, k), sI = d.plane, sJ = d.pitch;
    const GeoIJ& G = a.geo[i * d.jm + j];
    const double exp_rm = G.exp_rm, exp_2_rm = G.exp_2_rm, inv_rm = G.inv_rm, inv_rm2 = G.inv_rm2;
    const double inv_rmsinthe = G.inv_rmsinthe, inv_rm2sinthe = G.inv_rm2sinthe;
    const double inv_rm2sinthe2 = G.inv_rm2sinthe2, cos_rm2sin = G.costhe_inv_rm2sinthe;
    const double sinthe = G.sinthe, costhe = G.costhe;

    const double t_ijk = (double)ycol<TY>(a, 0)[c], u_ijk = (double)ycol<TY>(a, 1)[c], v_ijk = (double)ycol<TY>(a, 2)[c];
    const double w_ijk = (double)ycol<TY>(a, 3)[c], c_ijk = (double)ycol<TY>(a, 4)[c];
    const double u_exp = u_ijk * exp_rm, v_invrm = v_ijk * inv_rm, w_invrs = w_ijk * inv_rmsinthe;
    const double dpdr = (a.p_dyn[c + sI] - a.p_dyn[c - sI]) * a.inv_2dr;
    const double dpdthe = (a.p_dyn[c + sJ] - a.p_dyn[c - sJ]) * a.inv_2dthe;
    const double dpdphi = (a.p_dyn[c + 1] - a.p_dyn[c - 1]) * a.inv_2dphi;
    const double nontrad = a.nontrad ? 1.0 : 0.0;
    const double coriolis_rad = nontrad * 2.0 * sinthe * w_ijk;
    const double coriolis_the = 2.0 * costhe * w_ijk;
    const double coriolis_phi = -2.0 * (costhe * v_ijk + nontrad * sinthe * u_ijk);

    if (a.flags & 1) {
        // acting forces (:447-456)
        a.out[0][c] = 1.0 * a.coeff_Coriolis
            * sqrt((coriolis_rad * coriolis_rad + coriolis_the * coriolis_the + coriolis_phi * coriolis_phi) / 3.0);
        a.out[1][c] = 1.0 * a.coeff_buoy * (t_ijk - a.t_ref[i]);
        const double pt = dpdthe * inv_rm, pp = dpdphi * inv_rmsinthe;
        a.out[2][c] = -a.coeff_u_p * sqrt((dpdr * dpdr + pt * pt + pp * pp) / 3.0);
        // latent heat of the advected condensate (:458-488): the thresholds are saturation
        // mass fractions at p_hydro = 0 (never written), i.e. 0 below the critical point
        // and 1 above it (no saturation) for rain, always 0 for ice
        const double t_u = t_ijk * a.t_0;
        const double q_rain = thermo::saturation_mass_fraction(thermo::saturation_pressure(t_u), 0.0, 0.0);
        const double q_ice = thermo::saturation_mass_fraction(thermo::sublimation_pressure(t_u), 0.0, 0.0);
        const StarD<TY> CL = star(ycol<TY>(a, 5), c, sI, sJ);
        const StarD<TY> IC = star(ycol<TY>(a, 6), c, sI, sJ);
        const double q_lat = (c_ijk >= 0.85 * q_rain)
            ? u_ijk * ((CL.ip - CL.im) * a.inv_2dr) + v_ijk * inv_rm * ((CL.jp - CL.jm) * a.inv_2dthe)
              + w_ijk * inv_rmsinthe * ((CL.kp - CL.km) * a.inv_2dphi) : 0.0;
        const double q_lat_ice = (c_ijk >= 0.85 * q_ice)
            ? u_ijk * ((IC.ip - IC.im) * a.inv_2dr) + v_ijk * inv_rm * ((IC.jp - IC.jm) * a.inv_2dthe)
              + w_ijk * inv_rmsinthe * ((IC.kp - IC.km) * a.inv_2dphi) : 0.0;
        a.out[3][c] = a.coeff_L * (q_lat + q_lat_ice);
        // sensible heat (:490-491), the meridional second difference in mirror-exact form
        const StarD<TY> T = star(ycol<TY>(a, 0), c, sI, sJ);
        const double d2tdr2 = (T.ip - 2.0 * T.c + T.im) * a.inv_dr2;
        const double dtdr = (T.ip - T.im) * a.inv_2dr;
        const double d2tdthe2 = ((T.jp + T.jm) - 2.0 * T.c) * a.inv_dthe2;
        const double dtdthe = (T.jp - T.jm) * a.inv_2dthe;
        const double d2tdphi2 = (T.kp - 2.0 * T.c + T.km) * a.inv_dphi2;
        a.out[4][c] = a.coeff_S * (d2tdr2 + dtdr * 2.0 * inv_rm + d2tdthe2 * inv_rm2
            + dtdthe * cos_rm2sin + d2tdphi2 * inv_rm2sinthe2);
    }
    if (a.flags & 2) {
        // the terms of rhs_v and rhs_w (:1031-1057)
        const double nue_ijk = a.nue[c];
        const double diffusion_vel_re = (a.inv_re + nue_ijk) * a.diffusion_ramp;
        double drag_profile = 1.0 - (double)i / 5.0;
        if (drag_profile < 0.0) drag_profile = 0.0;
        const double surf_drag = a.drag_pref * drag_profile;
        const StarD<TY> U = star(ycol<TY>(a, 1), c, sI, sJ);
        const StarD<TY> V = star(ycol<TY>(a, 2), c, sI, sJ);
        const StarD<TY> W = star(ycol<TY>(a, 3), c, sI, sJ);
        const double inv_dr = 2.0 * a.inv_2dr, inv_dthe = 2.0 * a.inv_2dthe, inv_dphi = 2.0 * a.inv_2dphi;
        const double dudthe = (U.jp - U.jm) * a.inv_2dthe, dudphi = (U.kp - U.km) * a.inv_2dphi;
        const double dvdphi = (V.kp - V.km) * a.inv_2dphi, dwdphi = (W.kp - W.km) * a.inv_2dphi;
        const double v_metric = G.v_metric, two_over_rm_exp = G.two_over_rm_exp;
        const double diffusion_v = ((V.ip - 2.0 * V.c + V.im) * a.inv_dr2 * exp_2_rm
            + (V.ip - V.im) * a.inv_2dr * two_over_rm_exp
            + ((V.jp + V.jm) - 2.0 * V.c) * a.inv_dthe2 * inv_rm2
            + (V.jp - V.jm) * a.inv_2dthe * cos_rm2sin
            - v_metric * v_ijk + (V.kp - 2.0 * V.c + V.km) * a.inv_dphi2 * inv_rm2sinthe2
            + 2.0 * dudthe * inv_rm2
            - dwdphi * 2.0 * costhe * inv_rm2sinthe2) * diffusion_vel_re;
        const double diffusion_w = ((W.ip - 2.0 * W.c + W.im) * a.inv_dr2 * exp_2_rm
            + (W.ip - W.im) * a.inv_2dr * two_over_rm_exp
            + ((W.jp + W.jm) - 2.0 * W.c) * a.inv_dthe2 * inv_rm2
            + (W.jp - W.jm) * a.inv_2dthe * cos_rm2sin
            - v_metric * w_ijk + (W.kp - 2.0 * W.c + W.km) * a.inv_dphi2 * inv_rm2sinthe2
            + 2.0 * dudphi * inv_rm2sinthe
            + dvdphi * 2.0 * costhe * inv_rm2sinthe2) * diffusion_vel_re;
        const double vr = minmod_d(V.c - V.im, V.ip - V.c) * inv_dr;
        const double vt = minmod_d(V.c - V.jm, V.jp - V.c) * inv_dthe;
        const double vp = minmod_d(V.c - V.km, V.kp - V.c) * inv_dphi;
        const double wr = minmod_d(W.c - W.im, W.ip - W.c) * inv_dr;
        const double wt = minmod_d(W.c - W.jm, W.jp - W.c) * inv_dthe;
        const double wp = minmod_d(W.c - W.km, W.kp - W.c) * inv_dphi;
        a.out[5][c] = -(dpdthe * inv_rm);
        a.out[6][c] = 1.0 * a.force_nd * coriolis_the;
        a.out[7][c] = -(u_exp * vr);
        a.out[8][c] = -(v_invrm * vt + w_invrs * vp);
        a.out[9][c] = diffusion_v;
        a.out[10][c] = a.coeff_MC_vel * a.MC_v[c] - surf_drag * v_ijk;
        a.out[11][c] = -(dpdphi * inv_rmsinthe);
        a.out[12][c] = 1.0 * a.force_nd * coriolis_phi;
        a.out[13][c] = -(u_exp * wr);
        a.out[14][c] = -(v_invrm * wt + w_invrs * wp);
        a.out[15][c] = diffusion_w;
        a.out[16][c] = a.coeff_MC_vel * a.MC_w[c] - surf_drag * w_ijk;
    }
}

}  // namespace

void launch_rhs_diagnostics(const RhsDiagArgs& a, cudaStream_t st)
{
    const dim3 grid((a.d.km + 127) / 128, a.d.jm, a.d.im);
    if (a.Y32[0]) rhs_diag_kernel<float><<<grid, 128, 0, st>>>(a);
    else rhs_diag_kernel<double><<<grid, 128, 0, st>>>(a);
}

}  // namespace athad
