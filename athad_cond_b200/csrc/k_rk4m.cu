// k_rk4m.cu - the mixed-precision RK4 step (athad_params.precision = MIXED) on sm_100a.
//
// Same time step as k_rk4.cu (RungeKutta_Atm_Turb.cpp:44-273 with the right-hand side of
// RHS_Atm_Turb.cpp:31-1080, flat terrain, Jacobi stages), with this split of precision:
//   * FP32: the right-hand-side arithmetic, the three intermediate stage states, the RK4
//     accumulator K = k1 + 2k2 + 2k3, a FP32 copy of the time level n for stages 2-3, and
//     the per-cell forcing, packed once per step by stage 1 (below);
//   * FP64: the prognostic fields themselves (time level n and the result), the final
//     combination y = y_n + dt/6 (K + k4) of stage 4, the stage-1 state y_n + dt/2 k1,
//     the level-mean temperature and the mean-density profile.
// The model's other modules keep reading and writing the FP64 fields; only the RK4
// step's private buffers are FP32.
//
// Forcing packing: the reference's RHS reads 15 per-cell forcing fields (p_dyn, nue, t_eq,
// p_stat, r_humid, S_c..S_v, MC_t..MC_w) in every stage.  Stage 1 reads them in FP64 and
// writes 11 FP32 fields that stages 2-4 read instead: p_dyn (stencil), nue, t_eq, the
// Held-Suarez relaxation rate k_T L/u_0, and the combined source terms of t, c, cloud, ice,
// gr, v and w, each formed in FP64 from the same operands as the reference's terms.
//
// Memory traffic per grid point and step (algorithmic, 4-byte FP32 and 8-byte FP64
// fields): stage 1 reads 11 state + 11 level-n + 15 forcing FP64 and writes 11 stage +
// 11 K + 11 level-n + 11 forcing FP32 = 472 B; stages 2-3 read 11 stage + 11 level-n + 11 K
// + 11 forcing FP32 and write 11 stage + 11 K FP32 = 264 B each; stage 4 reads 11 stage +
// 11 K + 11 forcing FP32 and 11 level-n FP64 and writes 11 FP64 results + 3 FP64 aux =
// 332 B; with the level mean (8 B), 1340 B against 2096 B for the FP64 step.
//
// Mirror symmetry: the same expression structure as the FP64 kernel (second differences
// sum the two neighbours first; mirror-exact FP32 tables rounded from the FP64 ones);
// negation commutes with every IEEE operation including fused multiply-add, so a mirrored
// state still gives a bit-for-bit mirrored result.
#include "kernels.cuh"

namespace athad {

namespace {

__device__ __forceinline__ float fmaxs(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float fmins(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float fclamps(float v, float lo, float hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }
__device__ __forceinline__ float fminmod(float a, float b)
{
    return (a * b <= 0.0f) ? 0.0f : (fabsf(a) < fabsf(b) ? a : b);
}

// Single-use operands of a stage can be loaded with the streaming hint so they do not
// displace the stencil fields' lines from L1: ATHAD_RK4M_STREAM bit 1 the time level n, bit 2
// the packed forcing, bit 4 the accumulator.  Off: all three on made the mixed step 2 %
// slower at 41x181x361 (1.033 -> 1.055 ms; the FP64 step gains and uses it, k_rk4.cu).
#ifndef ATHAD_RK4M_STREAM
#define ATHAD_RK4M_STREAM 0
#endif
template <int BIT, class T>
__device__ __forceinline__ T ld_single(const T* p)
{
    if (ATHAD_RK4M_STREAM & BIT) return __ldcs(p);
    return __ldg(p);
}
// the accumulator, which the launch also writes (same thread, same cell): a coherent load
template <class T>
__device__ __forceinline__ T ld_acc(const T* p)
{
    if (ATHAD_RK4M_STREAM & 4) return __ldcs(p);
    return *p;
}

struct StarF {
    float c, ip, im, jp, jm, kp, km;
};

template <int STAGE>
__device__ __forceinline__ float ldY(const RK4MArgs& a, int n, long long c)
{
    if (STAGE == 1) return (float)__ldg(a.Y[n] + c);
    return __ldg(a.Yin[n] + c);
}

template <int STAGE>
__device__ __forceinline__ StarF load_star(const RK4MArgs& a, int n, long long c, long long sI, long long sJ)
{
    StarF s;
    s.c = ldY<STAGE>(a, n, c);
    s.ip = ldY<STAGE>(a, n, c + sI); s.im = ldY<STAGE>(a, n, c - sI);
    s.jp = ldY<STAGE>(a, n, c + sJ); s.jm = ldY<STAGE>(a, n, c - sJ);
    s.kp = ldY<STAGE>(a, n, c + 1);  s.km = ldY<STAGE>(a, n, c - 1);
    return s;
}

// the pressure perturbation: FP64 field in stage 1, its packed FP32 copy afterwards
template <int STAGE>
__device__ __forceinline__ float ldP(const RK4MArgs& a, long long c)
{
    if (STAGE == 1) return (float)__ldg(a.p_dyn + c);
    return __ldg(a.F[ATHAD_MF_P] + c);
}

__device__ __forceinline__ float d1r(const StarF& s, const RK4MArgs& a) { return (s.ip - s.im) * a.inv_2dr; }
__device__ __forceinline__ float d1t(const StarF& s, const RK4MArgs& a) { return (s.jp - s.jm) * a.inv_2dthe; }
__device__ __forceinline__ float d1p(const StarF& s, const RK4MArgs& a) { return (s.kp - s.km) * a.inv_2dphi; }
__device__ __forceinline__ float d2r(const StarF& s, const RK4MArgs& a) { return (s.ip - 2.0f * s.c + s.im) * a.inv_dr2; }
__device__ __forceinline__ float d2t(const StarF& s, const RK4MArgs& a) { return ((s.jp + s.jm) - 2.0f * s.c) * a.inv_dthe2; }
__device__ __forceinline__ float d2p(const StarF& s, const RK4MArgs& a) { return (s.kp - 2.0f * s.c + s.km) * a.inv_dphi2; }
__device__ __forceinline__ float ar(const StarF& s, const RK4MArgs& a) { return fminmod(s.c - s.im, s.ip - s.c) * a.inv_dr; }
__device__ __forceinline__ float at(const StarF& s, const RK4MArgs& a) { return fminmod(s.c - s.jm, s.jp - s.c) * a.inv_dthe; }
__device__ __forceinline__ float ap(const StarF& s, const RK4MArgs& a) { return fminmod(s.c - s.km, s.kp - s.c) * a.inv_dphi; }

// Stage update of field n (0 t, 1 u, 2 v, 3 w, 4 c, 5 cloud, 6 ice, 7 gr, 8 co2, 9 tke,
// 10 dis) with the clamps of RungeKutta_Atm_Turb.cpp:176-263.
template <int STAGE>
__device__ __forceinline__ void stage_update(const RK4MArgs& a, int n, long long c, float kn)
{
    if (STAGE == 1) {
        const double yn = ld_single<1>(a.Yn[n] + c);
        a.Yn32[n][c] = (float)yn;
        a.K[n][c] = kn;
        double y = yn + (double)kn * a.half_dt;
        if (n >= 4 && n <= 7) y = smax(0.0, y);
        else if (n == 9) y = safe_clamp(y, 0.0, (double)a.tke_max_nd);
        else if (n == 10) y = smax(1.0e-10, y);
        a.Yout[n][c] = (float)y;
    } else if (STAGE < 4) {
        const float yn = ld_single<1>(a.Yn32[n] + c);
        a.K[n][c] = ld_acc(a.K[n] + c) + 2.0f * kn;
        float y = yn + kn * ((STAGE == 3) ? a.dt_f : a.half_dt_f);
        if (n >= 4 && n <= 7) y = fmaxs(0.0f, y);
        else if (n == 9) y = isfinite(y) ? fclamps(y, 0.0f, a.tke_max_nd) : 0.0f;
        else if (n == 10) y = fmaxs(1.0e-10f, y);
        a.Yout[n][c] = y;
    } else {
        const double yn = ld_single<1>(a.Yn[n] + c);
        const float kk = ld_acc(a.K[n] + c) + kn;
        double y = yn + (double)kk * a.dt_sixth;
        if (n >= 4 && n <= 7) y = smax(0.0, y);
        else if (n == 9) y = safe_clamp(y, 0.0, (double)a.tke_max_nd);
        else if (n == 10) y = smax(1.0e-10, y);
        a.Y[n][c] = y;
        if (a.store_n) a.Yn_store[n][c] = y;   // storeIntermediateData3D fused
    }
}

// forcing value: computed from the FP64 fields (and stored) in stage 1, read afterwards
template <int STAGE>
__device__ __forceinline__ float forcing(const RK4MArgs& a, int f, long long c, double value_if_stage1)
{
    if (STAGE == 1) {
        const float v = (float)value_if_stage1;
        a.F[f][c] = v;
        return v;
    }
    return ld_single<2>(a.F[f] + c);
}

}  // namespace

// the tracer loop of the right-hand side (c, cloud, ice, gr, co2): unrolled, the five
// stencil loads of one tracer can be issued before the previous tracer's arithmetic
#ifndef ATHAD_RK4M_TRACER_UNROLL
#define ATHAD_RK4M_TRACER_UNROLL 5   // 41x181x361: 1.21 ms per step with 1, 1.02 ms with 5
                                     // (both at 12 CTAs per SM)
#endif
constexpr int kTracerUnroll = ATHAD_RK4M_TRACER_UNROLL;

// One cell of one stage.  Shared by the single-grid kernel and the batched persistent
// kernel (k_batch.cu), which reads each member's arguments from shared memory.
template <int STAGE>
__device__ __forceinline__ void rk4m_cell(const RK4MArgs& a, int i, int j, int k)
{
    const Dims& d = a.d;
    const long long c = idx3(d, i, j, k);
    const bool interior = (i > 0 && i < d.im - 1 && j > 0 && j < d.jm - 1 && k > 0 && k < d.km - 1);
    if (!interior) {
        if (STAGE == 1) {   // boundary values into both stage buffers; p_dyn for the stencil
#pragma unroll
            for (int n = 0; n < 11; n++) {
                const float v = (float)__ldg(a.Y[n] + c);
                a.Yout[n][c] = v;
                a.Ybnd[n][c] = v;
            }
            a.F[ATHAD_MF_P][c] = (float)__ldg(a.p_dyn + c);
        }
        if (STAGE == 4 && a.store_n) {   // the time-level copy of the cells RK4 leaves alone
#pragma unroll
            for (int n = 0; n < 11; n++) a.Yn_store[n][c] = __ldg(a.Y[n] + c);
        }
        return;
    }
    const long long sI = d.plane, sJ = d.pitch;
    const GeoF* G = a.geo + (i * d.jm + j);
    const float exp_rm = G->exp_rm, inv_rm = G->inv_rm, inv_rmsinthe = G->inv_rmsinthe;

    const float u_ijk = ldY<STAGE>(a, 1, c), v_ijk = ldY<STAGE>(a, 2, c), w_ijk = ldY<STAGE>(a, 3, c);
    const float nue_ijk = forcing<STAGE>(a, ATHAD_MF_NUE, c, STAGE == 1 ? __ldg(a.nue + c) : 0.0);
    const float u_exp = u_ijk * exp_rm, v_invrm = v_ijk * inv_rm, w_invrs = w_ijk * inv_rmsinthe;
    const float diffusion_vel_re = (a.inv_re + nue_ijk) * a.diffusion_ramp;

    // ---- turbulence production (RHS_Atm_Turb.cpp:528-561) ----
    float prod;
    {
        const StarF U = load_star<STAGE>(a, 1, c, sI, sJ);
        const StarF V = load_star<STAGE>(a, 2, c, sI, sJ);
        const StarF W = load_star<STAGE>(a, 3, c, sI, sJ);
        const float dudr_s = d1r(U, a) * exp_rm, dvdr_s = d1r(V, a) * exp_rm, dwdr_s = d1r(W, a) * exp_rm;
        const float dudthe_s = d1t(U, a) * inv_rm, dvdthe_s = d1t(V, a) * inv_rm, dwdthe_s = d1t(W, a) * inv_rm;
        const float dudphi_s = d1p(U, a) * inv_rmsinthe, dvdphi_s = d1p(V, a) * inv_rmsinthe,
                    dwdphi_s = d1p(W, a) * inv_rmsinthe;
        const float tke_ijk = ldY<STAGE>(a, 9, c), dis_ijk = ldY<STAGE>(a, 10, c);
        const float dis_here = fmaxs(dis_ijk, 1.0e-10f);
        const float tke_here = fmaxs(tke_ijk, 0.0f);
        float cnue = (a.turb_model == ATHAD_TURB_K_EPSILON) ? 0.028f * tke_here * tke_here / dis_here
                                                           : tke_here / dis_here;
        cnue = fmins(cnue, a.nue_max);
        const float der = 0.66667f * (dudr_s + dvdthe_s + dwdphi_s);
        prod = fmaxs(0.0f,
              (cnue * (2.0f * dudr_s - der) - 0.66667f * tke_ijk) * dudr_s
            + (cnue * (dudthe_s + dvdr_s)) * dudthe_s
            + (cnue * (dudphi_s + dwdr_s)) * dudphi_s
            + (cnue * (2.0f * dvdthe_s - der) - 0.66667f * tke_ijk) * dvdthe_s
            + (cnue * (dvdr_s + dudthe_s)) * dvdr_s
            + (cnue * (dvdphi_s + dwdthe_s)) * dvdphi_s
            + (cnue * (2.0f * dwdphi_s - der) - 0.66667f * tke_ijk) * dwdphi_s
            + (cnue * (dwdr_s + dudphi_s)) * dwdr_s
            + (cnue * (dwdthe_s + dvdphi_s)) * dwdthe_s);
    }

    // ---- tke and omega/epsilon (RHS_Atm_Turb.cpp:563-721, 835-836, 936-942, 1074-1075) ----
    {
        const float exp_2_rm = G->exp_2_rm, inv_rm2 = G->inv_rm2, inv_rm2sinthe2 = G->inv_rm2sinthe2;
        const float cos_rm2sin = G->costhe_inv_rm2sinthe, two_over_rm_exp = G->two_over_rm_exp;
        const StarF TK = load_star<STAGE>(a, 9, c, sI, sJ);
        const StarF DI = load_star<STAGE>(a, 10, c, sI, sJ);
        const float tke_ijk = TK.c, dis_ijk = DI.c;
        const float dtkedr = d1r(TK, a), dtkedthe = d1t(TK, a), dtkedphi = d1p(TK, a);
        const float ddisdr = d1r(DI, a), ddisdthe = d1t(DI, a), ddisdphi = d1p(DI, a);
        const float tke_s = fmaxs(tke_ijk, 1.0e-10f), dis_s = fmaxs(dis_ijk, 1.0e-10f);
        const float dis_src_max = 20.0f * dis_s * dis_s, tke_src_max = 20.0f * tke_s * dis_s;
        const float cross = dtkedr * ddisdr + dtkedthe * inv_rm * ddisdthe * inv_rm
                          + dtkedphi * inv_rmsinthe * ddisdphi * inv_rmsinthe;
        float diffusion_tke_re, diffusion_dis_re, tke_source, dis_source;
        if (a.turb_model == ATHAD_TURB_K_EPSILON) {
            diffusion_tke_re = a.inv_re + nue_ijk / 1.0f;
            diffusion_dis_re = a.inv_re + nue_ijk / 1.3f;
            const float P_k = prod, Y_k = dis_s;
            const float P_w = 1.35f * (dis_s / tke_s) * P_k;
            const float Y_w = 1.80f * dis_s * dis_s / tke_s;
            tke_source = fclamps(P_k - Y_k, -tke_src_max, tke_src_max);
            dis_source = fclamps(P_w - Y_w, -dis_src_max, dis_src_max);
        } else if (a.turb_model == ATHAD_TURB_K_OMEGA) {
            diffusion_tke_re = a.inv_re + 0.6f * nue_ijk;
            diffusion_dis_re = a.inv_re + 0.5f * nue_ijk;
            const float P_k = fmins(prod, 20.0f * 0.09f * tke_s * dis_s);
            const float Y_k = 0.09f * tke_s * dis_s;
            const float P_w = 0.52f * (dis_s / tke_s) * P_k;
            const float Y_w = 0.0708f * dis_s * dis_s;
            const float sig_d = (cross <= 0.0f) ? 0.0f : 0.125f;
            const float D_w = sig_d * cross / dis_s;
            tke_source = fclamps(P_k - Y_k, -tke_src_max, tke_src_max);
            dis_source = fclamps(P_w - Y_w + D_w, -dis_src_max, dis_src_max);
        } else {   // k-omega SST; wall distance as the FP64 kernel
            const float bet_star = 0.09f, sig_w2 = 1.168f;
            float d_j = (float)j;
            if (a.wall_mode == ATHAD_WALL_MIRROR) { const int jr = d.jm - 1 - j; if (jr < j) d_j = (float)jr; }
            float d_close = (float)i;
            if (d_j <= d_close) d_close = d_j;
            if ((float)k <= d_close) d_close = (float)k;
            const float CD_kw = fmaxs((2.0f * sig_w2) / dis_ijk * cross, 1.0e-20f);
            const float arg1 = fmins(fmaxs(
                sqrtf(tke_ijk) / (bet_star * dis_ijk * d_close),
                (500.0f * a.nue_air_nd) / (d_close * d_close * dis_ijk)),
                (4.0f * sig_w2 * tke_ijk) / (CD_kw * d_close * d_close));
            const float a2 = arg1 * arg1;
            const float F1 = tanhf(a2 * a2);
            const float bk = F1 * 1.176f + (1.0f - F1) * 1.0f;
            const float bw = F1 * 2.0f + (1.0f - F1) * sig_w2;
            diffusion_tke_re = a.inv_re + nue_ijk / bk;
            diffusion_dis_re = a.inv_re + nue_ijk / bw;
            const float P_k = fmins(prod, 20.0f * bet_star * tke_s * dis_s);
            const float Y_k = bet_star * tke_s * dis_s;
            const float P_w = (F1 * 0.413f + (1.0f - F1) * 0.2f) * P_k * dis_s / tke_s;
            const float Y_w = (F1 * 0.0333f + (1.0f - F1) * 0.0368f) * dis_s * dis_s;
            const float D_w = 2.0f * (1.0f - F1) * sig_w2 / dis_s * cross;
            tke_source = fclamps(P_k - Y_k, -tke_src_max, tke_src_max);
            dis_source = fclamps(P_w - Y_w + D_w, -dis_src_max, dis_src_max);
        }
        diffusion_tke_re *= a.diffusion_ramp;
        diffusion_dis_re *= a.diffusion_ramp;
        const float tr_tke = u_exp * dtkedr + v_invrm * dtkedthe + w_invrs * dtkedphi;
        const float tr_dis = u_exp * ddisdr + v_invrm * ddisdthe + w_invrs * ddisdphi;
        const float diffusion_tke = (d2r(TK, a) * exp_2_rm + dtkedr * two_over_rm_exp
            + d2t(TK, a) * inv_rm2 + dtkedthe * cos_rm2sin + d2p(TK, a) * inv_rm2sinthe2) * diffusion_tke_re;
        const float diffusion_dis = (d2r(DI, a) * exp_2_rm + ddisdr * two_over_rm_exp
            + d2t(DI, a) * inv_rm2 + ddisdthe * cos_rm2sin + d2p(DI, a) * inv_rm2sinthe2) * diffusion_dis_re;
        stage_update<STAGE>(a, 9, c, -tr_tke + diffusion_tke + tke_source);
        stage_update<STAGE>(a, 10, c, -tr_dis + diffusion_dis + dis_source);
        if (STAGE == 4 && a.write_diag) {
            a.prod[c] = prod;
            a.tke_source[c] = tke_source;
            a.dis_source[c] = dis_source;
        }
    }

    // ---- momentum (RHS_Atm_Turb.cpp:816-828, 870-884, 1001-1057, 1077-1079) ----
    {
        const float exp_2_rm = G->exp_2_rm, inv_rm2 = G->inv_rm2, inv_rm2sinthe2 = G->inv_rm2sinthe2;
        const float inv_rm2sinthe = G->inv_rm2sinthe;
        const float cos_rm2sin = G->costhe_inv_rm2sinthe, two_over_rm_exp = G->two_over_rm_exp;
        const float sinthe = G->sinthe, costhe = G->costhe, v_metric = G->v_metric;
        const float dpdr = (ldP<STAGE>(a, c + sI) - ldP<STAGE>(a, c - sI)) * a.inv_2dr;
        const float dpdthe = (ldP<STAGE>(a, c + sJ) - ldP<STAGE>(a, c - sJ)) * a.inv_2dthe;
        const float dpdphi = (ldP<STAGE>(a, c + 1) - ldP<STAGE>(a, c - 1)) * a.inv_2dphi;
        if (STAGE == 1) a.F[ATHAD_MF_P][c] = (float)__ldg(a.p_dyn + c);
        const float dpdr_exp = dpdr * exp_rm, dpdthe_invrm = dpdthe * inv_rm, dpdphi_invrs = dpdphi * inv_rmsinthe;
        const float nontrad = a.nontrad ? 1.0f : 0.0f;
        const float cotanthe = a.curvature ? costhe / sinthe : 0.0f;
        float drag_profile = 1.0f - (float)i / 5.0f;
        if (drag_profile < 0.0f) drag_profile = 0.0f;
        const float surf_drag = a.drag_pref * drag_profile;
        float dudthe, dudphi, dvdphi;
        {   // u
            const StarF U = load_star<STAGE>(a, 1, c, sI, sJ);
            dudthe = d1t(U, a);
            dudphi = d1p(U, a);
            float tr_u = u_exp * ar(U, a) + v_invrm * at(U, a) + w_invrs * ap(U, a);
            if (a.curvature) tr_u += -(v_ijk * v_ijk + w_ijk * w_ijk) * inv_rm;
            const float diffusion_u = (d2r(U, a) * exp_2_rm + 2.0f * u_ijk * inv_rm2
                + d2t(U, a) * inv_rm2 + 4.0f * d1r(U, a) * inv_rm * exp_rm
                + dudthe * cos_rm2sin + d2p(U, a) * inv_rm2sinthe2) * diffusion_vel_re;
            const float t_ijk = ldY<STAGE>(a, 0, c);
            const float coriolis_rad = nontrad * 2.0f * sinthe * w_ijk;
            const float rhs_u = -dpdr_exp - tr_u + diffusion_u
                + a.buoy_pref * (t_ijk - (float)__ldg(a.t_ref + i))
                + a.force_nd * coriolis_rad;
            stage_update<STAGE>(a, 1, c, rhs_u);
            if (STAGE == 4) a.aux_u[c] = (double)rhs_u + (double)dpdr_exp;
        }
        {   // v
            const StarF V = load_star<STAGE>(a, 2, c, sI, sJ);
            dvdphi = d1p(V, a);
            float tr_v = u_exp * ar(V, a) + v_invrm * at(V, a) + w_invrs * ap(V, a);
            if (a.curvature) tr_v += (u_ijk * v_ijk - w_ijk * w_ijk * cotanthe) * inv_rm;
            const float part_v = d2r(V, a) * exp_2_rm + d1r(V, a) * two_over_rm_exp
                + d2t(V, a) * inv_rm2 + d1t(V, a) * cos_rm2sin
                - v_metric * v_ijk + d2p(V, a) * inv_rm2sinthe2
                + 2.0f * dudthe * inv_rm2;
            const float dwdphi = (ldY<STAGE>(a, 3, c + 1) - ldY<STAGE>(a, 3, c - 1)) * a.inv_2dphi;
            const float diffusion_v = (part_v - dwdphi * 2.0f * costhe * inv_rm2sinthe2) * diffusion_vel_re;
            const float coriolis_the = 2.0f * costhe * w_ijk;
            const float mcv = forcing<STAGE>(a, ATHAD_MF_MV, c,
                                             STAGE == 1 ? a.coeff_MC_vel * __ldg(a.MC_v + c) : 0.0);
            const float rhs_v = -dpdthe_invrm - tr_v + diffusion_v
                + a.force_nd * coriolis_the + mcv - surf_drag * v_ijk;
            stage_update<STAGE>(a, 2, c, rhs_v);
            if (STAGE == 4) a.aux_v[c] = (double)rhs_v + (double)dpdthe_invrm;
        }
        {   // w
            const StarF W = load_star<STAGE>(a, 3, c, sI, sJ);
            float tr_w = u_exp * ar(W, a) + v_invrm * at(W, a) + w_invrs * ap(W, a);
            if (a.curvature) tr_w += (w_ijk * u_ijk + v_ijk * w_ijk * cotanthe) * inv_rm;
            const float diffusion_w = (d2r(W, a) * exp_2_rm + d1r(W, a) * two_over_rm_exp
                + d2t(W, a) * inv_rm2 + d1t(W, a) * cos_rm2sin
                - v_metric * w_ijk + d2p(W, a) * inv_rm2sinthe2
                + 2.0f * dudphi * inv_rm2sinthe
                + dvdphi * 2.0f * costhe * inv_rm2sinthe2) * diffusion_vel_re;
            const float coriolis_phi = -2.0f * (costhe * v_ijk + nontrad * sinthe * u_ijk);
            const float mcw = forcing<STAGE>(a, ATHAD_MF_MW, c,
                                             STAGE == 1 ? a.coeff_MC_vel * __ldg(a.MC_w + c) : 0.0);
            const float rhs_w = -dpdphi_invrs - tr_w + diffusion_w
                + a.force_nd * coriolis_phi + mcw - surf_drag * w_ijk;
            stage_update<STAGE>(a, 3, c, rhs_w);
            if (STAGE == 4) a.aux_w[c] = (double)rhs_w + (double)dpdphi_invrs;
        }
        // ---- temperature (RHS_Atm_Turb.cpp:752, 829, 866-868, 963-992) ----
        {
            const StarF T = load_star<STAGE>(a, 0, c, sI, sJ);
            const float t_ijk = T.c;
            const float pressure_t = a.coeff_energy_p * (u_exp * dpdr + v_invrm * dpdthe + w_invrs * dpdphi);
            const float tr_t = u_exp * ar(T, a) + v_invrm * at(T, a) + w_invrs * ap(T, a);
            const float diffusion_t_re = (a.inv_re + nue_ijk) * a.inv_pr_turb * a.diffusion_ramp;
            const float diffusion_t = (d2r(T, a) * exp_2_rm + d1r(T, a) * two_over_rm_exp
                + d2t(T, a) * inv_rm2 + d1t(T, a) * cos_rm2sin + d2p(T, a) * inv_rm2sinthe2) * diffusion_t_re;
            double q_t = 0.0, kT = 0.0, teq = 0.0;
            if (STAGE == 1) {
                const double r_h = __ldg(a.r_humid + c);
                q_t = a.coeff_MC_t * __ldg(a.MC_t + c)
                    + a.coeff_energy * (__ldg(a.S_c + c) + __ldg(a.S_r + c)) * a.lv * r_h
                    + a.coeff_energy * (__ldg(a.S_i + c) + __ldg(a.S_s + c) + __ldg(a.S_g + c)) * a.ls * r_h;
                const double k_a = 1.0 / (4.0 * 86400.0), k_s = 1.0 / (0.4 * 86400.0), sigma_b = 0.7;
                const double p_surf = __ldg(a.p_stat + idx3(d, 0, j, k));
                const double sigma = (p_surf > 0.0) ? __ldg(a.p_stat + c) / p_surf : 0.0;
                double bl = (sigma - sigma_b) / (1.0 - sigma_b);
                if (bl < 0.0) bl = 0.0;
                kT = (k_a + (k_s - k_a) * bl * (double)G->cos4lat) * a.L_atm_over_u0;
                teq = __ldg(a.t_eq + c);
            }
            const float qt = forcing<STAGE>(a, ATHAD_MF_QT, c, q_t);
            const float kTf = forcing<STAGE>(a, ATHAD_MF_KT, c, kT);
            const float teqf = forcing<STAGE>(a, ATHAD_MF_TEQ, c, teq);
            const float rhs_t = pressure_t - tr_t + diffusion_t + qt - kTf * (t_ijk - teqf);
            stage_update<STAGE>(a, 0, c, rhs_t);
        }
    }
    // ---- moisture and tracers (RHS_Atm_Turb.cpp:830-834, 911-934, 1059-1072) ----
    {
        const float exp_2_rm = G->exp_2_rm, inv_rm2 = G->inv_rm2, inv_rm2sinthe2 = G->inv_rm2sinthe2;
        const float cos_rm2sin = G->costhe_inv_rm2sinthe, two_over_rm_exp = G->two_over_rm_exp;
        const float dlnrho_dr_i = a.tracer_diff_flux ? (float)__ldg(a.dlnrho + i) * exp_2_rm : 0.0f;
        double r_h = 0.0;
        if (STAGE == 1) r_h = __ldg(a.r_humid + c);
#pragma unroll kTracerUnroll
        for (int n = 4; n <= 8; n++) {
            const StarF Q = load_star<STAGE>(a, n, c, sI, sJ);
            const float coef = (n == 8) ? a.diff_co2_re_inv : a.diff_prec_re_inv;
            const float tr = (n <= 6) ? (u_exp * ar(Q, a) + v_invrm * at(Q, a) + w_invrs * ap(Q, a))
                                      : (u_exp * d1r(Q, a) + v_invrm * d1t(Q, a) + w_invrs * d1p(Q, a));
            const float q1r = d1r(Q, a);
            const float dif = (d2r(Q, a) * exp_2_rm + q1r * two_over_rm_exp
                + d2t(Q, a) * inv_rm2 + d1t(Q, a) * cos_rm2sin
                + d2p(Q, a) * inv_rm2sinthe2
                + q1r * dlnrho_dr_i) * coef;
            float src = 0.0f;
            if (n <= 7) {
                double s1 = 0.0;
                if (STAGE == 1) {
                    if (n == 4)      s1 = __ldg(a.S_v + c) * r_h + a.coeff_MC_q * __ldg(a.MC_q + c);
                    else if (n == 5) s1 = __ldg(a.S_c + c) * r_h;
                    else if (n == 6) s1 = __ldg(a.S_i + c) * r_h;
                    else             s1 = __ldg(a.S_g + c) * r_h;
                }
                src = forcing<STAGE>(a, ATHAD_MF_QC + (n - 4), c, s1);
            }
            stage_update<STAGE>(a, n, c, -tr + dif + src);
        }
    }
}

#ifndef ATHAD_RK4M_MIN_BLOCKS
#define ATHAD_RK4M_MIN_BLOCKS 9    // 56 registers per thread, 9 CTAs of 128 threads per SM
                                   // (41x181x361, tracer loop unrolled: 12 CTAs 1.21 ms,
                                   // 11 1.11 ms, 10 1.02 ms, 9 0.96 ms, 8 1.04 ms)
#endif

#ifndef ATHAD_RK4M_BX
#define ATHAD_RK4M_BX 128        // CTA: BX longitudes x BY rows of one level (128 x 1 was 1 %
#endif                           // faster than 32 x 4, 64 x 2, 64 x 4, 32 x 8 at 41x181x361)
#ifndef ATHAD_RK4M_BY
#define ATHAD_RK4M_BY 1
#endif

#ifndef ATHAD_RK4M_MIN_BLOCKS_S1
#define ATHAD_RK4M_MIN_BLOCKS_S1 ATHAD_RK4M_MIN_BLOCKS   // stage 1 (forcing packing, FP64 reads)
#endif
#ifndef ATHAD_RK4M_MIN_BLOCKS_S4
#define ATHAD_RK4M_MIN_BLOCKS_S4 ATHAD_RK4M_MIN_BLOCKS   // stage 4 (FP64 combination, time level)
#endif

template <int STAGE>
__global__ void __launch_bounds__(ATHAD_RK4M_BX * ATHAD_RK4M_BY,
    (STAGE == 1 ? ATHAD_RK4M_MIN_BLOCKS_S1 : STAGE == 4 ? ATHAD_RK4M_MIN_BLOCKS_S4 : ATHAD_RK4M_MIN_BLOCKS)
    * 128 / (ATHAD_RK4M_BX * ATHAD_RK4M_BY))
rk4m_stage_kernel(const RK4MArgs a)
{
    pdl_trigger();
    pdl_wait();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (k >= a.d.km || j >= a.d.jm) return;
    // the even stages walk the radial planes from the top down, so that each stage starts
    // on the planes its predecessor wrote last (1.036 -> 1.030 ms per step at 41x181x361;
    // a stage's cells are independent, so the order changes no result)
#if ATHAD_RK4_SERPENTINE
    const int i = (STAGE % 2 == 0) ? a.d.im - 1 - (int)blockIdx.z : (int)blockIdx.z;
#else
    const int i = blockIdx.z;
#endif
    rk4m_cell<STAGE>(a, i, j, k);
}

void launch_rk4m_stage(int stage, const RK4MArgs& a, cudaStream_t st)
{
    const dim3 block(ATHAD_RK4M_BX, ATHAD_RK4M_BY, 1);
    const dim3 grid((a.d.km + ATHAD_RK4M_BX - 1) / ATHAD_RK4M_BX, (a.d.jm + ATHAD_RK4M_BY - 1) / ATHAD_RK4M_BY, a.d.im);
    switch (stage) {
        case 1: launch_dependent(rk4m_stage_kernel<1>, grid, block, 0, st, a); break;
        case 2: launch_dependent(rk4m_stage_kernel<2>, grid, block, 0, st, a); break;
        case 3: launch_dependent(rk4m_stage_kernel<3>, grid, block, 0, st, a); break;
        default: launch_dependent(rk4m_stage_kernel<4>, grid, block, 0, st, a); break;
    }
}


// ---------------------------------------------------------------------------------------
// Batched form: the members of an ensemble advance together, one persistent launch per
// stage.  The tiles of all members (BX longitudes x BY rows of one level) are numbered
// member after member; CTA b takes the contiguous range [b*per, (b+1)*per), so it changes
// member at most a few times.  On a change it copies that member's arguments into shared
// memory, sets the stage buffers of this stage and the member's step scalars, and runs the
// same per-cell code as the single-grid kernel.
template <int STAGE>
__device__ __forceinline__ void load_member_args(RK4MArgs& sa, const BatchTables& T, int m)
{
    const long long* src = reinterpret_cast<const long long*>(T.args + m);
    long long* dst = reinterpret_cast<long long*>(&sa);
    const int nthreads = blockDim.x * blockDim.y;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    __syncthreads();   // every warp is done with the previous member's arguments
    for (int w = tid; w < (int)(sizeof(RK4MArgs) / sizeof(long long)); w += nthreads) dst[w] = src[w];
    __syncthreads();
    if (tid < 11) {   // the table holds buffer A in Yout and buffer B in Ybnd
        float* A = sa.Yout[tid];
        float* B = sa.Ybnd[tid];
        sa.Yin[tid] = (STAGE == 3) ? B : A;
        sa.Yout[tid] = (STAGE == 1 || STAGE == 3) ? A : B;
        sa.Ybnd[tid] = B;
    } else if (tid == 32) {
        const BatchStep& st = T.step[m];
        sa.half_dt_f = st.half_dt_f; sa.dt_f = st.dt_f; sa.diffusion_ramp = st.diffusion_ramp;
        sa.drag_pref = st.drag_pref;
        const double x = (double)st.iter / (double)st.ramp_iters;
        const double ramp = (x < 1.0) ? x : 1.0;
        sa.buoy_pref = (float)(ramp * st.g * st.dt / st.u_0);
        sa.half_dt = st.half_dt; sa.dt_sixth = st.dt_sixth; sa.write_diag = st.write_diag;
    }
    __syncthreads();
}

template <int STAGE, int BX, int BY, int MINB>
__global__ void __launch_bounds__(BX * BY, MINB) rk4m_batch_kernel(const BatchTables T)
{
    __shared__ __align__(16) RK4MArgs sa;
    const int per = (T.total_tiles + gridDim.x - 1) / gridDim.x;
    const int t0 = blockIdx.x * per;
    const int t1 = min(T.total_tiles, t0 + per);
    if (t0 >= t1) return;
    // member owning tile t0: the last m with tile_start[m] <= t0 (binary search, uniform)
    int lo = 0, hi = T.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(T.tile_start + mid) <= t0) lo = mid; else hi = mid - 1;
    }
    int m = lo;
    load_member_args<STAGE>(sa, T, m);
    int tstart = __ldg(T.tile_start + m), tend = __ldg(T.tile_start + m + 1);
    int active = __ldg(&T.step[m].active);
    int nkx = (sa.d.km + BX - 1) / BX, nkj = nkx * ((sa.d.jm + BY - 1) / BY);
    for (int t = t0; t < t1; t++) {
        if (t >= tend) {
            while (__ldg(T.tile_start + m + 1) <= t) m++;
            load_member_args<STAGE>(sa, T, m);
            tstart = __ldg(T.tile_start + m); tend = __ldg(T.tile_start + m + 1);
            active = __ldg(&T.step[m].active);
            nkx = (sa.d.km + BX - 1) / BX; nkj = nkx * ((sa.d.jm + BY - 1) / BY);
        }
        if (!active) continue;
        const int local = t - tstart;
        const int i = local / nkj;
        const int rem = local - i * nkj;
        const int jt = rem / nkx;
        const int k = (rem - jt * nkx) * BX + threadIdx.x;
        const int j = jt * BY + threadIdx.y;
        if (k < sa.d.km && j < sa.d.jm) rk4m_cell<STAGE>(sa, i, j, k);
    }
}

// Tile shapes the autotuner chooses from: (longitudes, rows, CTAs per SM the register
// budget is sized for).
#define ATHAD_BATCH_SHAPES(X) X(0, 32, 4, 12) X(1, 32, 4, 8) X(2, 64, 2, 8) X(3, 32, 8, 4) X(4, 128, 1, 8) \
    X(5, 32, 4, 10)

template <int BX, int BY, int MINB>
static void launch_batch_shape(int stage, const BatchTables& T, int grid, cudaStream_t st)
{
    const dim3 block(BX, BY, 1);
    switch (stage) {
        case 1: rk4m_batch_kernel<1, BX, BY, MINB><<<grid, block, 0, st>>>(T); break;
        case 2: rk4m_batch_kernel<2, BX, BY, MINB><<<grid, block, 0, st>>>(T); break;
        case 3: rk4m_batch_kernel<3, BX, BY, MINB><<<grid, block, 0, st>>>(T); break;
        default: rk4m_batch_kernel<4, BX, BY, MINB><<<grid, block, 0, st>>>(T); break;
    }
}

template <int BX, int BY, int MINB>
static int batch_shape_grid()
{
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rk4m_batch_kernel<2, BX, BY, MINB>, BX * BY, 0);
    if (per_sm < 1) per_sm = 1;
    return sms * per_sm;
}

int batch_shape_count() { return 6; }

BatchShape batch_shape_info(int shape)
{
    BatchShape r{0, 0, 0};
#define ATHAD_SHAPE_INFO(ID, BX, BY, MINB) if (shape == ID) { r.bx = BX; r.by = BY; r.min_blocks = MINB; }
    ATHAD_BATCH_SHAPES(ATHAD_SHAPE_INFO)
#undef ATHAD_SHAPE_INFO
    return r;
}

int batch_shape_grid(int shape)
{
#define ATHAD_SHAPE_GRID(ID, BX, BY, MINB) if (shape == ID) return batch_shape_grid<BX, BY, MINB>();
    ATHAD_BATCH_SHAPES(ATHAD_SHAPE_GRID)
#undef ATHAD_SHAPE_GRID
    return 0;
}

void launch_rk4m_batch_stage(int stage, int shape, const BatchTables& T, int grid, cudaStream_t st)
{
#define ATHAD_SHAPE_LAUNCH(ID, BX, BY, MINB) if (shape == ID) { launch_batch_shape<BX, BY, MINB>(stage, T, grid, st); return; }
    ATHAD_BATCH_SHAPES(ATHAD_SHAPE_LAUNCH)
#undef ATHAD_SHAPE_LAUNCH
}

// computeLevelMeanTemperature of every member in one launch: one CTA per (member, level),
// the same row sums and mirror pairing as level_mean_kernel.
__global__ void __launch_bounds__(256) batch_level_mean_kernel(const LevelMeanMember* __restrict__ M, int n,
                                                               const BatchStep* __restrict__ step)
{
    extern __shared__ double rows[];
    const int g = blockIdx.x;
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (M[mid].level0 <= g) lo = mid; else hi = mid - 1;
    }
    const LevelMeanMember& mm = M[lo];
    if (!step[lo].active) return;
    const Dims d = mm.d;
    const int i = g - mm.level0;
    if (i >= d.im) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int j = warp; j < d.jm; j += nwarp) {
        const double* row = mm.t + idx3(d, i, j, 0);
        double s = 0.0;
        for (int k = lane; k < d.km; k += 32) s += __ldg(row + k);
        for (int off = 16; off >= 1; off >>= 1) s = s + __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) rows[j] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // explicit roundings: this file compiles with fused multiply-add, the single-grid
        // level mean without, and both must give the same bits
        double sum = 0.0, wsum = 0.0;
        const int half = d.jm / 2;
        for (int j = 0; j < half; j++) {
            sum = __dadd_rn(sum, __dmul_rn(mm.sin_w[j], __dadd_rn(rows[j], rows[d.jm - 1 - j])));
            wsum = __dadd_rn(wsum, __dmul_rn(__dmul_rn(2.0, mm.sin_w[j]), (double)d.km));
        }
        if (d.jm & 1) {
            sum = __dadd_rn(sum, __dmul_rn(mm.sin_w[half], rows[half]));
            wsum = __dadd_rn(wsum, __dmul_rn(mm.sin_w[half], (double)d.km));
        }
        mm.out[i] = (wsum > 0.0) ? sum / wsum : 1.0;
    }
}

void launch_batch_level_mean(const LevelMeanMember* M, int n, int total_levels, int max_jm,
                             const BatchStep* step, cudaStream_t st)
{
    batch_level_mean_kernel<<<total_levels, 256, sizeof(double) * max_jm, st>>>(M, n, step);
}

}  // namespace athad
