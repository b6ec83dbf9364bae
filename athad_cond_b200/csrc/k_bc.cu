// k_bc.cu - the per-iteration boundary conditions of the atmosphere on sm_100a
// (athad_boundary_conditions): BC_Atm::bcRadius, TurbulenceAtm::apply_wall_bc,
// BC_Atm::bcTheta, BC_Atm::bcPhi, BC_Atm::bcScalarSurfSur and BC_Atm::bcSolidGround, in the
// order of their call site (cAtmosphereModel.cpp:1439-1446), for flat terrain (every cell is
// air, so of the last two only bcSolidGround's value limits over every cell change anything).
//
// Three launches, one per direction, because each reads the boundary cells the previous
// one wrote (the corners): radial columns (one thread per (j, k)), polar rows (one thread
// per (i, k)), seam rows (one thread per (i, j)); then the value limits, cell by cell.  Every formula is a copy or a short sum
// evaluated in the reference's order; the file is compiled without fused multiply-add, so
// the results are bit-identical to the reference's.
//
// Fields: those of the reference's lists that the context holds (the right-hand side's
// CoriolisForce and BuoyancyForce, the heat diagnostics Q_Latent and Q_Sensible and the
// radiation flux included).  The reference's other arrays in the same lists, the outputs of
// ThermoAtm::forces and precipitableWater, are not held.  c43 and c13 are `const int` members
// initialised from 4.0/3.0 and 1.0/3.0 (cAtmosphereModel.h:158), i.e. 1 and 0.
#include "kernels.cuh"

namespace athad {

namespace {

__constant__ int kBothCubic[] = {                       // BC_Atm.h:567-574, Pattern A
    ATHAD_S_C_C, ATHAD_S_V, ATHAD_S_C, ATHAD_S_I, ATHAD_S_R, ATHAD_S_S, ATHAD_S_G,
    ATHAD_Q_V_U, ATHAD_Q_C_U, ATHAD_U_U, ATHAD_V_U, ATHAD_W_U,
    ATHAD_MC_S, ATHAD_MC_S_U, ATHAD_MC_S_D, ATHAD_M_U, ATHAD_M_D, ATHAD_Q_LATENT, ATHAD_Q_SENSIBLE,
    ATHAD_CORIOLIS_FORCE, ATHAD_BUOYANCY_FORCE};
__constant__ int kVnBot[] = {ATHAD_U, ATHAD_V, ATHAD_W, ATHAD_P_CONV};   // :586-590, Pattern B
__constant__ int kCubicBotVnTop[] = {                   // :599-603, Pattern C
    ATHAD_CLOUD, ATHAD_ICE, ATHAD_GR, ATHAD_CO2,
    ATHAD_C_U, ATHAD_E_DD, ATHAD_E_L, ATHAD_E_P, ATHAD_G_P,
    ATHAD_TKE, ATHAD_DIS, ATHAD_NUE, ATHAD_PROD, ATHAD_TKE_SOURCE, ATHAD_DIS_SOURCE};
__constant__ int kHydro[] = {ATHAD_P_STAT, ATHAD_R_HUMID, ATHAD_R_DRY};  // :656-665, Pattern D
__constant__ int kTheta[] = {                           // :760-776
    ATHAD_T, ATHAD_RADIATION, ATHAD_P_STAT, ATHAD_R_HUMID, ATHAD_R_DRY, ATHAD_U, ATHAD_V, ATHAD_W, ATHAD_C,
    ATHAD_CLOUD, ATHAD_ICE, ATHAD_GR, ATHAD_CO2, ATHAD_TKE, ATHAD_DIS, ATHAD_NUE, ATHAD_PROD,
    ATHAD_TKE_SOURCE, ATHAD_DIS_SOURCE,
    ATHAD_S_C_C, ATHAD_S_V, ATHAD_S_C, ATHAD_S_I, ATHAD_S_R, ATHAD_S_S, ATHAD_S_G,
    ATHAD_Q_V_U, ATHAD_Q_C_U, ATHAD_U_U, ATHAD_V_U, ATHAD_W_U, ATHAD_MC_S, ATHAD_MC_S_U,
    ATHAD_MC_S_D, ATHAD_C_U, ATHAD_E_DD, ATHAD_E_L, ATHAD_E_P, ATHAD_G_P, ATHAD_Q_LATENT,
    ATHAD_Q_SENSIBLE, ATHAD_CORIOLIS_FORCE, ATHAD_BUOYANCY_FORCE};
__constant__ int kPhiAvg[] = {                          // :806-817
    ATHAD_T, ATHAD_RADIATION, ATHAD_P_STAT, ATHAD_R_HUMID, ATHAD_R_DRY, ATHAD_U, ATHAD_V, ATHAD_W, ATHAD_C,
    ATHAD_CLOUD, ATHAD_ICE, ATHAD_GR, ATHAD_CO2,
    ATHAD_S_C_C, ATHAD_S_V, ATHAD_S_C, ATHAD_S_I, ATHAD_S_R, ATHAD_S_S, ATHAD_S_G,
    ATHAD_Q_V_U, ATHAD_Q_C_U, ATHAD_U_U, ATHAD_V_U, ATHAD_W_U, ATHAD_MC_S, ATHAD_MC_S_U,
    ATHAD_MC_S_D, ATHAD_C_U, ATHAD_E_DD, ATHAD_E_L, ATHAD_E_P, ATHAD_G_P, ATHAD_Q_LATENT,
    ATHAD_Q_SENSIBLE, ATHAD_CORIOLIS_FORCE, ATHAD_BUOYANCY_FORCE};
__constant__ int kPhiExtrap[] = {ATHAD_TKE, ATHAD_DIS, ATHAD_NUE, ATHAD_PROD, ATHAD_TKE_SOURCE,
                                 ATHAD_DIS_SOURCE};    // :822-825

template <int N>
constexpr int count(const int (&)[N]) { return N; }

// bcRadius (BC_Atm.h:556-746) and apply_wall_bc (TurbulenceAtm.h:109-147), one radial
// column per thread
__global__ void __launch_bounds__(128) bc_radius_kernel(BcArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= d.km) return;
    const int iml = d.im - 1;
    const long long s = d.plane;
    const long long c0 = idx3(d, 0, j, k), cl = idx3(d, iml, j, k);
    double* const* F = a.F;
    F[ATHAD_T][cl] = a.t_top_init[(long long)j * d.pitch + k];                         // :613-614
    for (int q = 0; q < count(kBothCubic); q++) {                                      // :629-633
        double* x = F[kBothCubic[q]];
        x[c0] = x[c0 + 3 * s] - 3.0 * x[c0 + 2 * s] + 3.0 * x[c0 + s];
        x[cl] = x[cl - 3 * s] - 3.0 * x[cl - 2 * s] + 3.0 * x[cl - s];
    }
    for (int q = 0; q < count(kHydro); q++) {                                          // :656-665
        double* x = F[kHydro[q]];
        x[c0] = x[c0 + 3 * s] - 3.0 * x[c0 + 2 * s] + 3.0 * x[c0 + s];
        const double x1 = x[cl - s], x2 = x[cl - 2 * s];
        x[cl] = (x1 > 0.0 && x2 > 0.0) ? (x1 * x1 / x2) : x1;
    }
    for (int q = 0; q < count(kVnBot); q++) {                                          // :671-675
        double* x = F[kVnBot[q]];
        x[c0] = 1.0 * x[c0 + s] - 0.0 * x[c0 + 2 * s];
        x[cl] = x[cl - s];
    }
    const int taper[4] = {ATHAD_V, ATHAD_W, ATHAD_VN, ATHAD_WN};                       // :685-690
    for (int q = 0; q < 4; q++) {
        double* x = F[taper[q]];
        x[cl] = 0.0;
        x[cl - s] *= (1.0 / 3.0);
        x[cl - 2 * s] *= (2.0 / 3.0);
    }
    F[ATHAD_U][cl] = 0.0; F[ATHAD_UN][cl] = 0.0;                                      // :704-705
    F[ATHAD_U][c0] = 0.0; F[ATHAD_UN][c0] = 0.0;                                      // :723-724
    for (int q = 0; q < count(kCubicBotVnTop); q++) {                                  // :727-731
        double* x = F[kCubicBotVnTop[q]];
        x[c0] = x[c0 + 3 * s] - 3.0 * x[c0 + 2 * s] + 3.0 * x[c0 + s];
        x[cl] = 1.0 * x[cl - s] - 0.0 * x[cl - 2 * s];
    }
    if (F[ATHAD_Q_V_U][c0] < 0.0) F[ATHAD_Q_V_U][c0] = 0.0;                            // :734-735
    if (F[ATHAD_Q_C_U][c0] < 0.0) F[ATHAD_Q_C_U][c0] = 0.0;
    // apply_wall_bc: the wall values of tke, nue and dis
    if (!a.wall_bc) return;
    const double vs = a.vel_star[(long long)j * d.pitch + k];
    F[ATHAD_TKE][c0] = vs * vs / a.tke_wall_den;
    F[ATHAD_NUE][c0] = 0.0;
    if (a.set_dis_wall) F[ATHAD_DIS][c0] = a.dis_wall;
}

// bcTheta (BC_Atm.h:750-796): pole copies, one (i, k) per thread
__global__ void __launch_bounds__(128) bc_theta_kernel(BcArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (k >= d.km) return;
    const long long n0 = idx3(d, i, 0, k), nl = idx3(d, i, d.jm - 1, k);
    for (int q = 0; q < count(kTheta); q++) {
        double* x = a.F[kTheta[q]];
        x[n0] = x[n0 + d.pitch];
        x[nl] = x[nl - d.pitch];
    }
}

// one 1-2-1 pass over the three seam cells {km-2, 0 = km-1, 1} of a row (BC_Atm.h:869-906)
__device__ __forceinline__ void smooth_seam(double* x, int km)
{
    const double c = 0.25;
    const double f_km2 = x[km - 2], f_0 = x[0], f_1 = x[1];
    const double w_km2 = x[km - 3], e_km2 = f_0;
    const double w_0 = f_km2, e_0 = f_1;
    const double w_1 = f_0, e_1 = x[2];
    x[km - 2] = f_km2 + c * (w_km2 - 2.0 * f_km2 + e_km2);
    const double m = f_0 + c * (w_0 - 2.0 * f_0 + e_0);
    x[0] = m;
    x[km - 1] = m;
    x[1] = f_1 + c * (w_1 - 2.0 * f_1 + e_1);
}

// bcPhi (BC_Atm.h:803-918), one (i, j) row per thread: seam average, zero-gradient, then
// the two smoothing passes of the velocities (each row's passes read only that row, so
// running them right after the row's own averaging is the reference's order)
__global__ void __launch_bounds__(128) bc_phi_kernel(BcArgs a)
{
    const Dims& d = a.d;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= d.jm) return;
    const long long r = idx3(d, i, j, 0);
    const int km = d.km;
    for (int q = 0; q < count(kPhiAvg); q++) {
        double* x = a.F[kPhiAvg[q]] + r;
        const double v0 = 1.0 * x[1] - 0.0 * x[2];
        const double vend = 1.0 * x[km - 2] - 0.0 * x[km - 3];
        const double m = (v0 + vend) * 0.5;
        x[0] = m;
        x[km - 1] = m;
    }
    for (int q = 0; q < count(kPhiExtrap); q++) {
        double* x = a.F[kPhiExtrap[q]] + r;
        x[0] = 1.0 * x[1] - 0.0 * x[2];
        x[km - 1] = 1.0 * x[km - 2] - 0.0 * x[km - 3];
    }
    for (int pass = 0; pass < 2; pass++) {
        smooth_seam(a.F[ATHAD_U] + r, km);  smooth_seam(a.F[ATHAD_UN] + r, km);
        smooth_seam(a.F[ATHAD_V] + r, km);  smooth_seam(a.F[ATHAD_VN] + r, km);
        smooth_seam(a.F[ATHAD_W] + r, km);  smooth_seam(a.F[ATHAD_WN] + r, km);
    }
}

// bcScalarSurfSur and bcSolidGround (BC_Atm.h:1026-1123, 23-547) with flat terrain: their
// land branches and the surface copies x[0] := x[i_mount = 0] change nothing, which leaves
// bcSolidGround's value limits over every cell (:470-545), one (i, j) row per block row
// a limit stores only where it changes the value (bit for bit: -0.0 stays -0.0), so the
// common case reads the fields and writes nothing
__device__ __forceinline__ void store_if_changed(double* p, double old_v, double new_v)
{
    if (__double_as_longlong(old_v) != __double_as_longlong(new_v)) *p = new_v;
}

__global__ void __launch_bounds__(128) bc_limits_kernel(BcArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.km) return;
    const long long c = (long long)blockIdx.y * d.pitch + k;
    double* const* F = a.F;
    const int sign[3] = {ATHAD_C, ATHAD_CLOUD, ATHAD_ICE};
#pragma unroll
    for (int q = 0; q < 3; q++)
        if (F[sign[q]][c] < 0.0) F[sign[q]][c] = 0.0;
    const double prod_max = 1.0e4, dis_max = 1.0e6;
    {   // tke and dis: non-negative, then clamped (a negative value becomes 0 first, which
        // the clamp keeps, or 1e-10 for dis)
        double v = F[ATHAD_TKE][c];
        const double v0 = v;
        if (v < 0.0) v = 0.0;
        store_if_changed(F[ATHAD_TKE] + c, v0, safe_clamp(v, 0.0, a.tke_max_nd));
        v = F[ATHAD_DIS][c];
        const double w0 = v;
        if (v < 0.0) v = 0.0;
        store_if_changed(F[ATHAD_DIS] + c, w0, safe_clamp(v, 1.0e-10, dis_max));
    }
    struct Lim { int f; double lo, hi; };
    const Lim lim[6] = {{ATHAD_TKEN, 0.0, a.tke_max_nd}, {ATHAD_DISN, 1.0e-10, dis_max},
                        {ATHAD_NUE, 0.0, a.nue_max}, {ATHAD_PROD, 0.0, prod_max},
                        {ATHAD_TKE_SOURCE, -prod_max, prod_max}, {ATHAD_DIS_SOURCE, -prod_max, prod_max}};
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const double v = F[lim[q].f][c];
        store_if_changed(F[lim[q].f] + c, v, safe_clamp(v, lim[q].lo, lim[q].hi));
    }
    const int vel[6] = {ATHAD_U, ATHAD_UN, ATHAD_V, ATHAD_VN, ATHAD_W, ATHAD_WN};
    const double vm = a.vel_max_nd;
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const double v = F[vel[q]][c];
        store_if_changed(F[vel[q]] + c, v, !is_finite_bits(v) ? 0.0 : (v < -vm) ? -vm : (v > vm) ? vm : v);
    }
}

}  // namespace

void launch_boundary_conditions(const BcArgs& a, cudaStream_t st)
{
    const Dims& d = a.d;
    bc_radius_kernel<<<dim3((d.km + 127) / 128, d.jm), 128, 0, st>>>(a);
    bc_theta_kernel<<<dim3((d.km + 127) / 128, d.im), 128, 0, st>>>(a);
    bc_phi_kernel<<<dim3((d.jm + 127) / 128, d.im), 128, 0, st>>>(a);
    bc_limits_kernel<<<dim3((d.km + 127) / 128, d.im * d.jm), 128, 0, st>>>(a);
}

}  // namespace athad
