// k_rk4.cu - RK4 time step of the ATHAD_COND atmosphere on sm_100a.
//
// Replaces cAtmosphereModel::solveRungeKutta_Atmosphere_Turb (RungeKutta_Atm_Turb.cpp:44-273)
// and cAtmosphereModel::RHS_Atmosphere_Turb (RHS_Atm_Turb.cpp:31-1080) for flat terrain.
//
// Structure: one launch per RK4 stage, one thread per cell of the full grid, k (longitude)
// on threadIdx.x so every field access of a warp is one coalesced 256-byte row segment;
// the 7-point star stencil reads its i+-1 and j+-1 neighbours from rows that neighbouring
// warps of the same CTA / plane also read, so they hit L1/L2 and DRAM sees each field about
// once per stage.  Stage semantics are Jacobi (each stage reads the previous stage's state
// everywhere); the accumulator K = k1 + 2 k2 + 2 k3 is formed in the reference's exact
// summation order so the final combination rounds as RungeKutta_Atm_Turb.cpp:253-263 does.
//
// Mirror symmetry: every theta-direction expression is written so that row j and row
// jm-1-j round identically (second differences sum the two neighbours first; the trig
// tables are mirror-exact), and the level mean pairs rows j and jm-1-j.  The result of a
// mirror-symmetric state is therefore bit-for-bit mirror symmetric.
#include "kernels.cuh"

namespace athad {

// ---------------------------------------------------------------------------------------
// computeLevelMeanTemperature (RungeKutta_Atm_Turb.cpp:24-41).  Row sums first, one warp
// per (i, j) row over all SMs: a 32-lane strided partial sum reduced by xor butterfly; then
// one CTA per level stages its row sums in shared memory (jm <= 6144) and one thread adds
// rows j and jm-1-j before weighting, so the mean of a mirrored field is identical.
// The same pass counts the non-finite values of t (nonfinite, may be null): a row whose sum
// is finite holds none, so only rows with a non-finite sum are scanned.
__global__ void __launch_bounds__(256) level_rows_kernel(Dims d, const double* __restrict__ t,
                                                         double* __restrict__ rows,
                                                         unsigned long long* __restrict__ nonfinite)
{
    pdl_trigger();
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= d.im * d.jm) return;
    const double* r = t + (long long)row * d.pitch;
    double s = 0.0;
    for (int k = lane; k < d.km; k += 32) s += __ldg(r + k);
    for (int off = 16; off >= 1; off >>= 1) s = s + __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) rows[row] = s;
    if (nonfinite && !is_finite_bits(s)) {
        unsigned int n = 0;
        for (int k = lane; k < d.km; k += 32) n += is_finite_bits(__ldg(r + k)) ? 0u : 1u;
        for (int off = 16; off >= 1; off >>= 1) n += __shfl_xor_sync(0xffffffffu, n, off);
        if (lane == 0 && n) atomicAdd(nonfinite, (unsigned long long)n);
    }
}

__global__ void __launch_bounds__(128) level_combine_kernel(Dims d, const double* __restrict__ rows,
                                                            const double* __restrict__ sin_w,
                                                            double* __restrict__ out)
{
    pdl_trigger();
    pdl_wait();
    extern __shared__ double r[];   // [jm] row sums of level i
    const int i = blockIdx.x;
    for (int j = threadIdx.x; j < d.jm; j += blockDim.x) r[j] = rows[(long long)i * d.jm + j];
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double* __restrict__ sin_w_s = sin_w;
    double sum = 0.0, wsum = 0.0;
    const int half = d.jm / 2;
    for (int j = 0; j < half; j++) {
        sum += sin_w_s[j] * (r[j] + r[d.jm - 1 - j]);
        wsum += 2.0 * sin_w_s[j] * (double)d.km;
    }
    if (d.jm & 1) {
        sum += sin_w_s[half] * r[half];
        wsum += sin_w_s[half] * (double)d.km;
    }
    out[i] = (wsum > 0.0) ? sum / wsum : 1.0;
}

void launch_level_mean(const Dims& d, const double* t, const double* sin_w, double* out,
                       double* row_sum, cudaStream_t st, unsigned long long* nonfinite)
{
    const int rows = d.im * d.jm;
    level_rows_kernel<<<(rows + 7) / 8, 256, 0, st>>>(d, t, row_sum, nonfinite);
    launch_dependent(level_combine_kernel, dim3(d.im), dim3(128), d.jm * sizeof(double), st,
                     d, (const double*)row_sum, sin_w, out);
}

// ---------------------------------------------------------------------------------------
// minmod slope limiter, RHS_Atm_Turb.cpp:26-28
__device__ __forceinline__ double minmod(double a, double b)
{
    return (a * b <= 0.0) ? 0.0 : (fabs(a) < fabs(b) ? a : b);
}

// The 7-point star of one field at one cell.
struct Star {
    double c, ip, im, jp, jm, kp, km;
};
__device__ __forceinline__ Star load_star(const double* __restrict__ F, long long c, long long sI, long long sJ)
{
    Star s;
    s.c = __ldg(F + c);
    s.ip = __ldg(F + c + sI); s.im = __ldg(F + c - sI);
    s.jp = __ldg(F + c + sJ); s.jm = __ldg(F + c - sJ);
    s.kp = __ldg(F + c + 1);  s.km = __ldg(F + c - 1);
    return s;
}
// central first differences (RHS_Atm_Turb.cpp:122, 224, 328)
__device__ __forceinline__ double d1r(const Star& s, const RK4Args& a) { return (s.ip - s.im) * a.inv_2dr; }
__device__ __forceinline__ double d1t(const Star& s, const RK4Args& a) { return (s.jp - s.jm) * a.inv_2dthe; }
__device__ __forceinline__ double d1p(const Star& s, const RK4Args& a) { return (s.kp - s.km) * a.inv_2dphi; }
// second differences (:123, :329); the meridional one sums the two neighbours first, the
// mirror-exact form of :225
__device__ __forceinline__ double d2r(const Star& s, const RK4Args& a) { return (s.ip - 2.0 * s.c + s.im) * a.inv_dr2; }
__device__ __forceinline__ double d2t(const Star& s, const RK4Args& a) { return ((s.jp + s.jm) - 2.0 * s.c) * a.inv_dthe2; }
__device__ __forceinline__ double d2p(const Star& s, const RK4Args& a) { return (s.kp - 2.0 * s.c + s.km) * a.inv_dphi2; }
// minmod-limited advective gradients (:788-814), inv_dx = 2 * inv_2dx (:762-764)
__device__ __forceinline__ double ar(const Star& s, const RK4Args& a) { return minmod(s.c - s.im, s.ip - s.c) * (2.0 * a.inv_2dr); }
__device__ __forceinline__ double at(const Star& s, const RK4Args& a) { return minmod(s.c - s.jm, s.jp - s.c) * (2.0 * a.inv_2dthe); }
__device__ __forceinline__ double ap(const Star& s, const RK4Args& a) { return minmod(s.c - s.km, s.kp - s.c) * (2.0 * a.inv_2dphi); }

// Stage update of one field (RungeKutta_Atm_Turb.cpp:167-182, 199-209, 226-236, 253-263).
// Field n: 0 t, 1 u, 2 v, 3 w, 4 c, 5 cloud, 6 ice, 7 gr, 8 co2, 9 tke, 10 dis.
// single-use operands (time level n, accumulator) with the streaming hint
// (ATHAD_RK4_STREAM_LOADS), so they do not displace the stencil fields' lines from L1:
// 1.745 -> 1.717 ms per FP64 step at 41x181x361 (the mixed step, whose single-use operands
// are FP32, runs 2 % slower with it and keeps plain loads)
#ifndef ATHAD_RK4_STREAM_LOADS
#define ATHAD_RK4_STREAM_LOADS 1
#endif
__device__ __forceinline__ double ld_once(const double* p)
{
#if ATHAD_RK4_STREAM_LOADS
    return __ldcs(p);
#else
    return __ldg(p);
#endif
}
// the same for the accumulator, which the launch also writes (same thread, same cell): a
// coherent load either way
__device__ __forceinline__ double ld_acc(const double* p)
{
#if ATHAD_RK4_STREAM_LOADS
    return __ldcs(p);
#else
    return *p;
#endif
}

template <int STAGE>
__device__ __forceinline__ void stage_update(const RK4Args& a, int n, long long c, double kn)
{
    const double yn = ld_once(a.Yn[n] + c);
    double kk, coef;
    if (STAGE == 1) {
        a.K[n][c] = kn;
        kk = kn; coef = a.half_dt;
    } else if (STAGE < 4) {
        const double acc = ld_acc(a.K[n] + c) + 2.0 * kn;
        a.K[n][c] = acc;
        kk = kn; coef = (STAGE == 3) ? a.dt : a.half_dt;
    } else {
        kk = ld_acc(a.K[n] + c) + kn; coef = a.dt_sixth;
    }
    const double y = yn + kk * coef;
    double out;
    if (n >= 4 && n <= 7) out = smax(0.0, y);
    else if (n == 9) out = safe_clamp(y, 0.0, a.tke_max_nd);
    else if (n == 10) out = smax(1.0e-10, y);
    else out = y;
    a.Yout[n][c] = out;
    if (STAGE == 4 && a.store_n) a.Yn_store[n][c] = out;   // storeIntermediateData3D fused
}

// One RK4 stage.  The right-hand side is evaluated in the order that keeps the fewest
// values live (turbulence, momentum, temperature, tracers), each term with the operation
// order of RHS_Atm_Turb.cpp; stencil values a later phase needs again are re-read, which
// hits L1.
#ifndef ATHAD_RK4_MIN_BLOCKS
#define ATHAD_RK4_MIN_BLOCKS 7   // 72 registers per thread, 7 CTAs of 128 threads per SM
#endif

#ifndef ATHAD_RK4_BX
#define ATHAD_RK4_BX 32          // CTA: BX longitudes x BY rows of one level
#endif
#ifndef ATHAD_RK4_BY
#define ATHAD_RK4_BY 4
#endif

// Shared-memory staging of the stencil tiles (ATHAD_RK4_SMEM=1): the CTA's BY x BX cells of
// level i with a one-cell ring in j and k, for the 11 stage fields and p_dyn, loaded once
// per launch; the centre, meridional and zonal neighbours then come from shared memory and
// only the radial neighbours (levels i +- 1) from global memory (L1/L2).  Same results bit
// for bit.  Off: measured at 41x181x361 (FP64 step, reference initial state) 1.743 ms
// against 1.744 ms without it at 32 x 4 and 7 CTAs per SM, 1.76 ms at 6 CTAs, 1.94 ms with
// 32 x 8 tiles (a third less halo, half the CTAs per SM): the DRAM traffic is already
// 1.17x the algorithmic bytes, the neighbours the tiles would serve hit L1/L2 today, and
// the staging adds a barrier and its own loads.
#ifndef ATHAD_RK4_SMEM
#define ATHAD_RK4_SMEM 0
#endif
constexpr int kTileJ = ATHAD_RK4_BY + 2, kTileK = ATHAD_RK4_BX + 2, kTileFields = 12;
constexpr int kTileCells = kTileJ * kTileK;

__device__ __forceinline__ const double* stage_field(const RK4Args& a, int n)
{
    return (n < 11) ? a.Yin[n] : a.p_dyn;
}

// every thread of the CTA takes part (before any thread returns); levels 0 and im-1 hold
// boundary cells only and stage nothing
__device__ __forceinline__ void stage_tiles(const RK4Args& a, double (*tile)[kTileJ][kTileK], int i)
{
    const Dims& d = a.d;
    if (i <= 0 || i >= d.im - 1) return;
    const int j0 = blockIdx.y * ATHAD_RK4_BY - 1, k0 = blockIdx.x * ATHAD_RK4_BX - 1;
    const int tid = threadIdx.y * ATHAD_RK4_BX + threadIdx.x;
    constexpr int kThreads = ATHAD_RK4_BX * ATHAD_RK4_BY;
#pragma unroll
    for (int e0 = 0; e0 < kTileCells; e0 += kThreads) {
        const int e = e0 + tid;
        if (e >= kTileCells) break;
        const int tj = e / kTileK, tk = e - tj * kTileK;
        const int jj = j0 + tj, kk = k0 + tk;
        if (jj < 0 || jj >= d.jm || kk < 0 || kk >= d.km) continue;
        const long long g = idx3(d, i, jj, kk);
#pragma unroll
        for (int n = 0; n < kTileFields; n++) tile[n][tj][tk] = __ldg(stage_field(a, n) + g);
    }
}

#ifndef ATHAD_RK4_TRACER_UNROLL
#define ATHAD_RK4_TRACER_UNROLL 5    // 41x181x361: 1.92 ms per step with 1, 1.64 ms with 5
#endif
constexpr int kTracerUnroll64 = ATHAD_RK4_TRACER_UNROLL;

template <int STAGE>
__global__ void __launch_bounds__(ATHAD_RK4_BX * ATHAD_RK4_BY, ATHAD_RK4_MIN_BLOCKS * 128 / (ATHAD_RK4_BX * ATHAD_RK4_BY))
rk4_stage_kernel(const RK4Args a)
{
    pdl_trigger();
    pdl_wait();
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    // the even stages walk the radial planes from the top down (ATHAD_RK4_SERPENTINE, kernels.cuh)
#if ATHAD_RK4_SERPENTINE
    const int i = (STAGE % 2 == 0) ? d.im - 1 - (int)blockIdx.z : (int)blockIdx.z;
#else
    const int i = blockIdx.z;
#endif
#if ATHAD_RK4_SMEM
    __shared__ double tile[kTileFields][kTileJ][kTileK];
    stage_tiles(a, tile, i);
    __syncthreads();
#endif
    if (k >= d.km || j >= d.jm) return;
    const long long c = idx3(d, i, j, k);
    const bool interior = (i > 0 && i < d.im - 1 && j > 0 && j < d.jm - 1 && k > 0 && k < d.km - 1);
    if (!interior) {
        // Boundary cells are not integrated (the reference loops run over the interior);
        // the stage buffers carry their current value so interior stencils can read them.
        if (STAGE == 1) {
#pragma unroll
            for (int n = 0; n < 11; n++) {
                const double v = __ldg(a.Yin[n] + c);
                a.Yout[n][c] = v;
                a.Ybnd[n][c] = v;
            }
        }
        if (STAGE == 4 && a.store_n) {   // the time-level copy of the cells RK4 leaves alone
#pragma unroll
            for (int n = 0; n < 11; n++) a.Yn_store[n][c] = a.Yout[n][c];
        }
        return;
    }
    const long long sI = d.plane, sJ = d.pitch;
    const GeoIJ* G = a.geo + (i * d.jm + j);
    const double exp_rm = G->exp_rm, inv_rm = G->inv_rm, inv_rmsinthe = G->inv_rmsinthe;
#if ATHAD_RK4_SMEM
    const int ty = threadIdx.y + 1, tx = threadIdx.x + 1;
    auto star = [&](int n) {
        Star s;
        s.c = tile[n][ty][tx];
        s.jp = tile[n][ty + 1][tx]; s.jm = tile[n][ty - 1][tx];
        s.kp = tile[n][ty][tx + 1]; s.km = tile[n][ty][tx - 1];
        const double* F = stage_field(a, n);
        s.ip = __ldg(F + c + sI); s.im = __ldg(F + c - sI);
        return s;
    };
#else
    auto star = [&](int n) { return load_star(stage_field(a, n), c, sI, sJ); };
#endif

    const double u_ijk = __ldg(a.Yin[1] + c), v_ijk = __ldg(a.Yin[2] + c), w_ijk = __ldg(a.Yin[3] + c);
    const double nue_ijk = __ldg(a.nue + c);
    const double u_exp = u_ijk * exp_rm, v_invrm = v_ijk * inv_rm, w_invrs = w_ijk * inv_rmsinthe;
    const double diffusion_vel_re = (a.inv_re + nue_ijk) * a.diffusion_ramp;

    // ---- turbulence: production from the velocity shear (RHS_Atm_Turb.cpp:528-561) ----
    double prod;
    {
        const Star U = star(1);
        const Star V = star(2);
        const Star W = star(3);
        const double dudr_s = d1r(U, a) * exp_rm, dvdr_s = d1r(V, a) * exp_rm, dwdr_s = d1r(W, a) * exp_rm;
        const double dudthe_s = d1t(U, a) * inv_rm, dvdthe_s = d1t(V, a) * inv_rm, dwdthe_s = d1t(W, a) * inv_rm;
        const double dudphi_s = d1p(U, a) * inv_rmsinthe, dvdphi_s = d1p(V, a) * inv_rmsinthe,
                     dwdphi_s = d1p(W, a) * inv_rmsinthe;
        const double tke_ijk = __ldg(a.Yin[9] + c), dis_ijk = __ldg(a.Yin[10] + c);
        const double dis_here = smax(dis_ijk, 1.0e-10);
        const double tke_here = smax(tke_ijk, 0.0);
        double cnue = (a.turb_model == ATHAD_TURB_K_EPSILON) ? 0.028 * tke_here * tke_here / dis_here
                                                            : tke_here / dis_here;
        cnue = smin(cnue, a.nue_max);
        const double der = 0.66667 * (dudr_s + dvdthe_s + dwdphi_s);
        prod = smax(0.0,
              (cnue * (2.0 * dudr_s - der) - 0.66667 * tke_ijk) * dudr_s
            + (cnue * (dudthe_s + dvdr_s)) * dudthe_s
            + (cnue * (dudphi_s + dwdr_s)) * dudphi_s
            + (cnue * (2.0 * dvdthe_s - der) - 0.66667 * tke_ijk) * dvdthe_s
            + (cnue * (dvdr_s + dudthe_s)) * dvdr_s
            + (cnue * (dvdphi_s + dwdthe_s)) * dvdphi_s
            + (cnue * (2.0 * dwdphi_s - der) - 0.66667 * tke_ijk) * dwdphi_s
            + (cnue * (dwdr_s + dudphi_s)) * dwdr_s
            + (cnue * (dwdthe_s + dvdphi_s)) * dwdthe_s);
    }

    // ---- tke and omega/epsilon: closure, sources, transport, diffusion ----
    //      (RHS_Atm_Turb.cpp:563-721, 835-836, 936-942, 1074-1075)
    {
        const double exp_2_rm = G->exp_2_rm, inv_rm2 = G->inv_rm2, inv_rm2sinthe2 = G->inv_rm2sinthe2;
        const double cos_rm2sin = G->costhe_inv_rm2sinthe, two_over_rm_exp = G->two_over_rm_exp;
        const Star TK = star(9);
        const Star DI = star(10);
        const double tke_ijk = TK.c, dis_ijk = DI.c;
        const double dtkedr = d1r(TK, a), dtkedthe = d1t(TK, a), dtkedphi = d1p(TK, a);
        const double ddisdr = d1r(DI, a), ddisdthe = d1t(DI, a), ddisdphi = d1p(DI, a);
        const double tke_s = smax(tke_ijk, 1.0e-10), dis_s = smax(dis_ijk, 1.0e-10);
        const double dis_src_max = 20.0 * dis_s * dis_s, tke_src_max = 20.0 * tke_s * dis_s;
        double diffusion_tke_re, diffusion_dis_re, tke_source, dis_source;
        if (a.turb_model == ATHAD_TURB_K_EPSILON) {
            diffusion_tke_re = a.inv_re + nue_ijk / 1.0;
            diffusion_dis_re = a.inv_re + nue_ijk / 1.3;
            const double P_k = prod, Y_k = dis_s;
            const double P_w = 1.35 * (dis_s / tke_s) * P_k;
            const double Y_w = 1.80 * dis_s * dis_s / tke_s;
            tke_source = sclamp(P_k - Y_k, -tke_src_max, tke_src_max);
            dis_source = sclamp(P_w - Y_w, -dis_src_max, dis_src_max);
        } else if (a.turb_model == ATHAD_TURB_K_OMEGA) {
            diffusion_tke_re = a.inv_re + 0.6 * nue_ijk;
            diffusion_dis_re = a.inv_re + 0.5 * nue_ijk;
            const double P_k = smin(prod, 20.0 * 0.09 * tke_s * dis_s);
            const double Y_k = 0.09 * tke_s * dis_s;
            const double P_w = 0.52 * (dis_s / tke_s) * P_k;
            const double Y_w = 0.0708 * dis_s * dis_s;
            const double cross = dtkedr * ddisdr + dtkedthe * inv_rm * ddisdthe * inv_rm
                               + dtkedphi * inv_rmsinthe * ddisdphi * inv_rmsinthe;
            const double sig_d = (cross <= 0.0) ? 0.0 : 0.125;
            const double D_w = sig_d * cross / dis_s;
            tke_source = sclamp(P_k - Y_k, -tke_src_max, tke_src_max);
            dis_source = sclamp(P_w - Y_w + D_w, -dis_src_max, dis_src_max);
        } else {   // k-omega SST
            const double bet_star = 0.09, sig_w2 = 1.168;
            // wall distance, RHS_Atm_Turb.cpp:640-671 (flat terrain: min(i, j, k));
            // ATHAD_WALL_MIRROR measures the meridional distance to the nearer pole
            double d_j = (double)j;
            if (a.wall_mode == ATHAD_WALL_MIRROR) { const int jr = d.jm - 1 - j; if (jr < j) d_j = (double)jr; }
            double d_close = (double)i;
            if (d_j <= d_close) d_close = d_j;
            if ((double)k <= d_close) d_close = (double)k;
            const double cross = dtkedr * ddisdr + dtkedthe * inv_rm * ddisdthe * inv_rm
                               + dtkedphi * inv_rmsinthe * ddisdphi * inv_rmsinthe;
            const double CD_kw = smax((2.0 * sig_w2) / dis_ijk * cross, 1.0e-20);
            const double arg1 = smin(smax(
                sqrt(tke_ijk) / (bet_star * dis_ijk * d_close),
                (500.0 * a.nue_air_nd) / (d_close * d_close * dis_ijk)),
                (4.0 * sig_w2 * tke_ijk) / (CD_kw * d_close * d_close));
            // pow(arg1, 4) as two squarings: both within two ulp of the exact value
            const double a2 = arg1 * arg1;
            const double F1 = tanh(a2 * a2);
            const double bk = F1 * 1.176 + (1.0 - F1) * 1.0;
            const double bw = F1 * 2.0 + (1.0 - F1) * sig_w2;
            diffusion_tke_re = a.inv_re + nue_ijk / bk;
            diffusion_dis_re = a.inv_re + nue_ijk / bw;
            const double P_k = smin(prod, 20.0 * bet_star * tke_s * dis_s);
            const double Y_k = bet_star * tke_s * dis_s;
            const double P_w = (F1 * 0.413 + (1.0 - F1) * 0.2) * P_k * dis_s / tke_s;
            const double Y_w = (F1 * 0.0333 + (1.0 - F1) * 0.0368) * dis_s * dis_s;
            const double D_w = 2.0 * (1.0 - F1) * sig_w2 / dis_s * cross;
            tke_source = sclamp(P_k - Y_k, -tke_src_max, tke_src_max);
            dis_source = sclamp(P_w - Y_w + D_w, -dis_src_max, dis_src_max);
        }
        diffusion_tke_re *= a.diffusion_ramp;
        diffusion_dis_re *= a.diffusion_ramp;
        const double tr_tke = u_exp * dtkedr + v_invrm * dtkedthe + w_invrs * dtkedphi;
        const double tr_dis = u_exp * ddisdr + v_invrm * ddisdthe + w_invrs * ddisdphi;
        const double diffusion_tke = (d2r(TK, a) * exp_2_rm + dtkedr * two_over_rm_exp
            + d2t(TK, a) * inv_rm2 + dtkedthe * cos_rm2sin + d2p(TK, a) * inv_rm2sinthe2) * diffusion_tke_re;
        const double diffusion_dis = (d2r(DI, a) * exp_2_rm + ddisdr * two_over_rm_exp
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
        const double exp_2_rm = G->exp_2_rm, inv_rm2 = G->inv_rm2, inv_rm2sinthe2 = G->inv_rm2sinthe2;
        const double inv_rm2sinthe = G->inv_rm2sinthe;
        const double cos_rm2sin = G->costhe_inv_rm2sinthe, two_over_rm_exp = G->two_over_rm_exp;
        const double sinthe = G->sinthe, costhe = G->costhe, v_metric = G->v_metric;
        const Star P = star(11);
        const double dpdr = (P.ip - P.im) * a.inv_2dr;
        const double dpdthe = (P.jp - P.jm) * a.inv_2dthe;
        const double dpdphi = (P.kp - P.km) * a.inv_2dphi;
        const double dpdr_exp = dpdr * exp_rm, dpdthe_invrm = dpdthe * inv_rm, dpdphi_invrs = dpdphi * inv_rmsinthe;
        const double nontrad = a.nontrad ? 1.0 : 0.0;
        const double cotanthe = a.curvature ? costhe / sinthe : 0.0;
        double drag_profile = 1.0 - (double)(i - 0) / 5.0;
        if (drag_profile < 0.0) drag_profile = 0.0;
        if (drag_profile > 1.0) drag_profile = 1.0;
        const double surf_drag = a.drag_pref * drag_profile;
        double dudthe, dudphi, dvdphi, part_v;
        {   // u
            const Star U = star(1);
            dudthe = d1t(U, a);
            dudphi = d1p(U, a);
            double tr_u = u_exp * ar(U, a) + v_invrm * at(U, a) + w_invrs * ap(U, a);
            if (a.curvature) tr_u += -(v_ijk * v_ijk + w_ijk * w_ijk) * inv_rm;
            const double diffusion_u = (d2r(U, a) * exp_2_rm + 2.0 * u_ijk * inv_rm2
                + d2t(U, a) * inv_rm2 + 4.0 * d1r(U, a) * inv_rm * exp_rm
                + dudthe * cos_rm2sin + d2p(U, a) * inv_rm2sinthe2) * diffusion_vel_re;
            const double t_ijk = __ldg(a.Yin[0] + c);
            const double coriolis_rad = nontrad * 2.0 * sinthe * w_ijk;
            const double rhs_u = -dpdr_exp - tr_u + diffusion_u
                + a.buoy_pref * (t_ijk - __ldg(a.t_ref + i))
                + 1.0 * a.force_nd * coriolis_rad;
            stage_update<STAGE>(a, 1, c, rhs_u);
            if (STAGE == 4) a.aux_u[c] = rhs_u + dpdr_exp;
        }
        {   // v: every term but the w-shear one, which closes the sum below
            const Star V = star(2);
            dvdphi = d1p(V, a);
            part_v = V.c;   // placeholder for register reuse
            double tr_v = u_exp * ar(V, a) + v_invrm * at(V, a) + w_invrs * ap(V, a);
            if (a.curvature) tr_v += (u_ijk * v_ijk - w_ijk * w_ijk * cotanthe) * inv_rm;
            part_v = d2r(V, a) * exp_2_rm + d1r(V, a) * two_over_rm_exp
                + d2t(V, a) * inv_rm2 + d1t(V, a) * cos_rm2sin
                - v_metric * v_ijk + d2p(V, a) * inv_rm2sinthe2
                + 2.0 * dudthe * inv_rm2;
            // w shear term of diffusion_v needs dw/dphi: only the zonal neighbours of w
            const double dwdphi = (__ldg(a.Yin[3] + c + 1) - __ldg(a.Yin[3] + c - 1)) * a.inv_2dphi;
            const double diffusion_v = (part_v - dwdphi * 2.0 * costhe * inv_rm2sinthe2) * diffusion_vel_re;
            const double coriolis_the = 2.0 * costhe * w_ijk;
            const double rhs_v = -dpdthe_invrm - tr_v + diffusion_v
                + 1.0 * a.force_nd * coriolis_the
                + a.coeff_MC_vel * __ldg(a.MC_v + c)
                - surf_drag * v_ijk;
            stage_update<STAGE>(a, 2, c, rhs_v);
            if (STAGE == 4) a.aux_v[c] = rhs_v + dpdthe_invrm;
        }
        {   // w
            const Star W = star(3);
            double tr_w = u_exp * ar(W, a) + v_invrm * at(W, a) + w_invrs * ap(W, a);
            if (a.curvature) tr_w += (w_ijk * u_ijk + v_ijk * w_ijk * cotanthe) * inv_rm;
            const double diffusion_w = (d2r(W, a) * exp_2_rm + d1r(W, a) * two_over_rm_exp
                + d2t(W, a) * inv_rm2 + d1t(W, a) * cos_rm2sin
                - v_metric * w_ijk + d2p(W, a) * inv_rm2sinthe2
                + 2.0 * dudphi * inv_rm2sinthe
                + dvdphi * 2.0 * costhe * inv_rm2sinthe2) * diffusion_vel_re;
            const double coriolis_phi = -2.0 * (costhe * v_ijk + nontrad * sinthe * u_ijk);
            const double rhs_w = -dpdphi_invrs - tr_w + diffusion_w
                + 1.0 * a.force_nd * coriolis_phi
                + a.coeff_MC_vel * __ldg(a.MC_w + c)
                - surf_drag * w_ijk;
            stage_update<STAGE>(a, 3, c, rhs_w);
            if (STAGE == 4) a.aux_w[c] = rhs_w + dpdphi_invrs;
        }
        // ---- temperature (RHS_Atm_Turb.cpp:752, 829, 866-868, 963-992) ----
        {
            const Star T = star(0);
            const double t_ijk = T.c;
            const double r_h = __ldg(a.r_humid + c);
            const double pressure_t = a.coeff_energy_p * (u_exp * dpdr + v_invrm * dpdthe + w_invrs * dpdphi);
            const double tr_t = u_exp * ar(T, a) + v_invrm * at(T, a) + w_invrs * ap(T, a);
            const double diffusion_t_re = (a.inv_re + nue_ijk) / a.pr_turb * a.diffusion_ramp;
            const double diffusion_t = (d2r(T, a) * exp_2_rm + d1r(T, a) * two_over_rm_exp
                + d2t(T, a) * inv_rm2 + d1t(T, a) * cos_rm2sin + d2p(T, a) * inv_rm2sinthe2) * diffusion_t_re;
            double rhs_t = pressure_t - tr_t + diffusion_t
                + a.coeff_MC_t * __ldg(a.MC_t + c)
                + a.coeff_energy * (__ldg(a.S_c + c) + __ldg(a.S_r + c)) * a.lv * r_h
                + a.coeff_energy * (__ldg(a.S_i + c) + __ldg(a.S_s + c) + __ldg(a.S_g + c)) * a.ls * r_h;
            const double k_a = 1.0 / (4.0 * 86400.0), k_s = 1.0 / (0.4 * 86400.0), sigma_b = 0.7;
            const double p_surf = __ldg(a.p_stat + idx3(d, 0, j, k));
            const double sigma = (p_surf > 0.0) ? __ldg(a.p_stat + c) / p_surf : 0.0;
            double bl = (sigma - sigma_b) / (1.0 - sigma_b);
            if (bl < 0.0) bl = 0.0;
            const double k_T = k_a + (k_s - k_a) * bl * G->cos4lat;
            rhs_t -= (k_T * a.L_atm / a.u_0) * (t_ijk - __ldg(a.t_eq + c));
            stage_update<STAGE>(a, 0, c, rhs_t);
        }
    }
    // ---- moisture and tracers (RHS_Atm_Turb.cpp:830-834, 911-934, 1059-1072) ----
    {
        const double exp_2_rm = G->exp_2_rm, inv_rm2 = G->inv_rm2, inv_rm2sinthe2 = G->inv_rm2sinthe2;
        const double cos_rm2sin = G->costhe_inv_rm2sinthe, two_over_rm_exp = G->two_over_rm_exp;
        const double dlnrho_dr_i = a.tracer_diff_flux ? __ldg(a.dlnrho + i) * exp_2_rm : 0.0;
        const double r_h = __ldg(a.r_humid + c);
#pragma unroll kTracerUnroll64
        for (int n = 4; n <= 8; n++) {
            const Star Q = star(n);
            const double coef = (n == 8) ? a.diff_co2_re_inv : a.diff_prec_re_inv;
            const double tr = (n <= 6) ? (u_exp * ar(Q, a) + v_invrm * at(Q, a) + w_invrs * ap(Q, a))
                                       : (u_exp * d1r(Q, a) + v_invrm * d1t(Q, a) + w_invrs * d1p(Q, a));
            const double q1r = d1r(Q, a);
            const double dif = (d2r(Q, a) * exp_2_rm + q1r * two_over_rm_exp
                + d2t(Q, a) * inv_rm2 + d1t(Q, a) * cos_rm2sin
                + d2p(Q, a) * inv_rm2sinthe2
                + q1r * dlnrho_dr_i) * coef;
            double rhs;
            if (n == 4)      rhs = -tr + dif + 1.0 * __ldg(a.S_v + c) * r_h + a.coeff_MC_q * __ldg(a.MC_q + c);
            else if (n == 5) rhs = -tr + dif + 1.0 * __ldg(a.S_c + c) * r_h;
            else if (n == 6) rhs = -tr + dif + 1.0 * __ldg(a.S_i + c) * r_h;
            else if (n == 7) rhs = -tr + dif + 1.0 * __ldg(a.S_g + c) * r_h;
            else             rhs = -tr + dif;
            stage_update<STAGE>(a, n, c, rhs);
        }
    }
}

void launch_rk4_stage(int stage, const RK4Args& a, cudaStream_t st)
{
    const dim3 block(ATHAD_RK4_BX, ATHAD_RK4_BY, 1);
    const dim3 grid((a.d.km + ATHAD_RK4_BX - 1) / ATHAD_RK4_BX, (a.d.jm + ATHAD_RK4_BY - 1) / ATHAD_RK4_BY, a.d.im);
    switch (stage) {
        case 1: launch_dependent(rk4_stage_kernel<1>, grid, block, 0, st, a); break;
        case 2: launch_dependent(rk4_stage_kernel<2>, grid, block, 0, st, a); break;
        case 3: launch_dependent(rk4_stage_kernel<3>, grid, block, 0, st, a); break;
        default: launch_dependent(rk4_stage_kernel<4>, grid, block, 0, st, a); break;
    }
}

}  // namespace athad
