// k_diag.cu - diagnostics on the device that read the model state:
//
//   searchMinMax_3D (MinMax_Atm.cpp:51-109): the largest and smallest finite value of a field
//     and the first cell in (i, j, k) order holding each;
//   UtilsAtm::findResiduumAtm (UtilsAtm.h:70-220): the largest rms velocity-derivative
//     residual of the band i = 10..30, its cell, the grid average and the non-finite cells;
//   ThermoAtm::standAtm_DewPoint_HumidRel (ThermoAtm.h:400-516): standard-atmosphere
//     temperature, dew point and relative humidity of every cell.
//
// The scans run one warp per (i, j) row, lane-strided over the longitudes, keeping the first
// position of a strictly larger (smaller) value, and combine lanes preferring the smaller
// longitude on a tie; one CTA then combines the rows in order, preferring the smaller row.
// Positions are the serial scan's whatever the launch shape; sums run in a fixed order.
// Compiled without fused multiply-add: the residuals and the standard-atmosphere profile
// are the oracle's bit for bit.
#include <cfloat>
#include <climits>

#include "kernels.cuh"
#include "thermo.cuh"

namespace athad {

namespace {

struct Best {
    double v;
    long long at;    // linear (row, k) position; -1 = none
};

__device__ __forceinline__ Best pick_max(Best a, Best b)
{
    if (b.at < 0) return a;
    if (a.at < 0) return b;
    if (b.v > a.v || (b.v == a.v && b.at < a.at)) return b;
    return a;
}
__device__ __forceinline__ Best pick_min(Best a, Best b)
{
    if (b.at < 0) return a;
    if (a.at < 0) return b;
    if (b.v < a.v || (b.v == a.v && b.at < a.at)) return b;
    return a;
}
__device__ __forceinline__ Best shfl(Best x, int off)
{
    Best y;
    y.v = __shfl_xor_sync(0xffffffffu, x.v, off);
    y.at = __shfl_xor_sync(0xffffffffu, x.at, off);
    return y;
}

__global__ void __launch_bounds__(256) minmax_rows_kernel(Dims d, const double* __restrict__ x,
                                                          double* __restrict__ rv, long long* __restrict__ ra)
{
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= d.im * d.jm) return;
    const double* r = x + (long long)row * d.pitch;
    // the serial scan starts from -DBL_MAX / DBL_MAX and keeps strictly larger / smaller
    // finite values, so a value equal to the start value is never taken
    Best mx{-DBL_MAX, -1}, mn{DBL_MAX, -1};
    for (int k = lane; k < d.km; k += 32) {
        const double v = r[k];
        if (!isfinite(v)) continue;
        const long long at = (long long)row * d.km + k;
        if (v > mx.v) { mx.v = v; mx.at = at; }
        if (v < mn.v) { mn.v = v; mn.at = at; }
    }
    for (int off = 16; off >= 1; off >>= 1) {
        mx = pick_max(mx, shfl(mx, off));
        mn = pick_min(mn, shfl(mn, off));
    }
    if (lane == 0) {
        rv[2 * row] = mx.v; ra[2 * row] = mx.at;
        rv[2 * row + 1] = mn.v; ra[2 * row + 1] = mn.at;
    }
}

__global__ void __launch_bounds__(1024) minmax_final_kernel(int rows, const double* __restrict__ rv,
                                                            const long long* __restrict__ ra,
                                                            double* __restrict__ out_v, long long* __restrict__ out_a)
{
    Best mx{-DBL_MAX, -1}, mn{DBL_MAX, -1};
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
        mx = pick_max(mx, Best{rv[2 * r], ra[2 * r]});
        mn = pick_min(mn, Best{rv[2 * r + 1], ra[2 * r + 1]});
    }
    for (int off = 16; off >= 1; off >>= 1) {
        mx = pick_max(mx, shfl(mx, off));
        mn = pick_min(mn, shfl(mn, off));
    }
    __shared__ Best smx[32], smn[32];
    if ((threadIdx.x & 31) == 0) { smx[threadIdx.x >> 5] = mx; smn[threadIdx.x >> 5] = mn; }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int nw = (blockDim.x + 31) >> 5;
        mx = (threadIdx.x < nw) ? smx[threadIdx.x] : Best{-DBL_MAX, -1};
        mn = (threadIdx.x < nw) ? smn[threadIdx.x] : Best{DBL_MAX, -1};
        for (int off = 16; off >= 1; off >>= 1) {
            mx = pick_max(mx, shfl(mx, off));
            mn = pick_min(mn, shfl(mn, off));
        }
        if (threadIdx.x == 0) {
            out_v[0] = mx.v; out_a[0] = mx.at;
            out_v[1] = mn.v; out_a[1] = mn.at;
        }
    }
}

// ---- findResiduumAtm ----------------------------------------------------------------

struct ResRow {
    Best mx;
    double sum;
    long long cnt, nnan, nkey;    // nkey: first non-finite cell's (j*km + k)*im + i
};

__device__ __forceinline__ ResRow res_combine(ResRow a, ResRow b)
{
    ResRow r;
    r.mx = pick_max(a.mx, b.mx);
    r.sum = a.sum + b.sum;
    r.cnt = a.cnt + b.cnt;
    r.nnan = a.nnan + b.nnan;
    r.nkey = (b.nkey < a.nkey) ? b.nkey : a.nkey;
    return r;
}
__device__ __forceinline__ ResRow res_shfl(ResRow x, int off)
{
    ResRow y;
    y.mx = shfl(x.mx, off);
    y.sum = __shfl_xor_sync(0xffffffffu, x.sum, off);
    y.cnt = __shfl_xor_sync(0xffffffffu, x.cnt, off);
    y.nnan = __shfl_xor_sync(0xffffffffu, x.nnan, off);
    y.nkey = __shfl_xor_sync(0xffffffffu, x.nkey, off);
    return y;
}
__device__ __forceinline__ ResRow res_empty() { return ResRow{Best{0.0, -1}, 0.0, 0, 0, LLONG_MAX}; }

// one warp per (i, j) row of the band, j = 1..jm-2; lanes over k = 1..km-2
__global__ void __launch_bounds__(256) residuum_rows_kernel(ResiduumArgs a, int rows)
{
    const Dims& d = a.d;
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= rows) return;
    const int i = a.i0 + row / (d.jm - 2);
    const int j = 1 + row % (d.jm - 2);
    const double rm = a.rad[i];
    const double exp_rm = 1.0 / (rm + 1.0);
    const double rmsinthe = rm * a.sinthe[j];
    const long long base = idx3(d, i, j, 0);
    const long long sI = d.plane, sJ = d.pitch;
    ResRow r = res_empty();
    for (int k = 1 + lane; k < d.km - 1; k += 32) {
        const long long c = base + k;
        const double dudr = (a.u[c + sI] - a.u[c - sI]) / (2.0 * a.dr) * exp_rm;
        const double dvdthe = (a.v[c + sJ] - a.v[c - sJ]) / (2.0 * rm * a.dthe);
        const double dwdphi = (a.w[c + 1] - a.w[c - 1]) / (2.0 * rmsinthe * a.dphi);
        const double res = sqrt((dudr * dudr + dvdthe * dvdthe + dwdphi * dwdphi) / 3.0);
        if (!isfinite(res)) {
            const long long key = ((long long)j * d.km + k) * d.im + i;
            if (key < r.nkey) r.nkey = key;
            r.nnan++;
            continue;
        }
        r.sum += res;
        r.cnt++;
        // only residuals above the starting value 0 become the residuum (UtilsAtm.h:133)
        if (res > 0.0 && (r.mx.at < 0 || res > r.mx.v)) { r.mx.v = res; r.mx.at = ((long long)i * d.jm + j) * d.km + k; }
    }
    for (int off = 16; off >= 1; off >>= 1) r = res_combine(r, res_shfl(r, off));
    if (lane == 0) {
        double* sv = a.scratch;
        long long* sl = reinterpret_cast<long long*>(a.scratch);
        sv[6 * (long long)row + 0] = r.mx.v;
        sl[6 * (long long)row + 1] = r.mx.at;
        sv[6 * (long long)row + 2] = r.sum;
        sl[6 * (long long)row + 3] = r.cnt;
        sl[6 * (long long)row + 4] = r.nnan;
        sl[6 * (long long)row + 5] = r.nkey;
    }
}

__global__ void __launch_bounds__(1024) residuum_final_kernel(ResiduumArgs a, int rows)
{
    const double* sv = a.scratch;
    const long long* sl = reinterpret_cast<const long long*>(a.scratch);
    ResRow r = res_empty();
    for (int q = threadIdx.x; q < rows; q += blockDim.x) {
        ResRow x{Best{sv[6 * (long long)q], sl[6 * (long long)q + 1]}, sv[6 * (long long)q + 2],
                 sl[6 * (long long)q + 3], sl[6 * (long long)q + 4], sl[6 * (long long)q + 5]};
        r = res_combine(r, x);
    }
    for (int off = 16; off >= 1; off >>= 1) r = res_combine(r, res_shfl(r, off));
    __shared__ ResRow part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = r;
    __syncthreads();
    if (threadIdx.x < 32) {
        const int nw = (blockDim.x + 31) >> 5;
        r = (threadIdx.x < nw) ? part[threadIdx.x] : res_empty();
        for (int off = 16; off >= 1; off >>= 1) r = res_combine(r, res_shfl(r, off));
        if (threadIdx.x == 0) {
            unsigned long long* o = a.out;
            o[0] = (unsigned long long)__double_as_longlong(r.mx.v);
            o[1] = (unsigned long long)r.mx.at;
            o[2] = (unsigned long long)__double_as_longlong(r.sum);
            o[3] = (unsigned long long)r.cnt;
            o[4] = (unsigned long long)r.nnan;
            o[5] = (unsigned long long)r.nkey;
        }
    }
}

// ---- co2Column / waterBudget ----------------------------------------------------------

__device__ __forceinline__ double budget_dp(const BudgetArgs& a, long long c, int i)
{
    return (i < a.d.im - 1) ? (a.p_stat[c] - a.p_stat[c + a.d.plane]) * 100.0 : a.p_stat[c] * 100.0;
}

// one warp per (i, j) row: air mass, water mass, CO2 mass of the cells with a positive layer
// pressure drop, and the plain sum of the water mass fraction (ThermoAtm.h:942-1034, 1102-1122)
__global__ void __launch_bounds__(256) budget_rows_kernel(BudgetArgs a)
{
    const Dims& d = a.d;
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= d.im * d.jm) return;
    const int i = row / d.jm;
    const long long base = (long long)row * d.pitch;
    double s_air = 0.0, s_w = 0.0, s_c = 0.0, s_q = 0.0;
    for (int k = lane; k < d.km; k += 32) {
        const long long c = base + k;
        const double q_w = fmax(0.0, a.c[c]) + fmax(0.0, a.cloud[c]) + fmax(0.0, a.ice[c]) + fmax(0.0, a.gr[c]);
        s_q += q_w;
        const double dp = budget_dp(a, c, i);
        if (!(dp > 0.0)) continue;
        const double u_air = dp / a.g;
        s_air += u_air;
        s_w += q_w * u_air;
        s_c += fmax(0.0, a.co2[c]) * u_air;
    }
    for (int off = 16; off >= 1; off >>= 1) {
        s_air += __shfl_xor_sync(0xffffffffu, s_air, off);
        s_w += __shfl_xor_sync(0xffffffffu, s_w, off);
        s_c += __shfl_xor_sync(0xffffffffu, s_c, off);
        s_q += __shfl_xor_sync(0xffffffffu, s_q, off);
    }
    if (lane == 0) {
        double* r = a.rows + 4 * (long long)row;
        r[0] = s_air; r[1] = s_w; r[2] = s_c; r[3] = s_q;
    }
}

// one CTA per level: the rows weighted by cos(latitude), summed in a fixed order
__global__ void __launch_bounds__(256) budget_levels_kernel(BudgetArgs a)
{
    const Dims& d = a.d;
    const int i = blockIdx.x;
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int j = threadIdx.x; j < d.jm; j += blockDim.x) {
        const double w = a.coslat[j];
        const double* r = a.rows + 4 * ((long long)i * d.jm + j);
        v[0] += w * r[0]; v[1] += w * r[1]; v[2] += w * r[2]; v[3] += w * r[3];
        v[4] += w;
    }
    __shared__ double part[5][8];
    for (int q = 0; q < 5; q++) {
        double x = v[q];
        for (int off = 16; off >= 1; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
        if ((threadIdx.x & 31) == 0) part[q][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double x = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) x += part[threadIdx.x][w];
        if (threadIdx.x == 4) x *= (double)d.km;       // sum of coslat over every (j, k)
        a.levels[6 * i + threadIdx.x] = x;
    }
    if (threadIdx.x == 5) a.levels[6 * i + 5] = 0.0;
}

// co2_total: the column CO2 path, summed up the column as ThermoAtm.h:1105-1120 does
__global__ void __launch_bounds__(128) co2_column_kernel(BudgetArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (k >= d.km) return;
    double col = 0.0;
    for (int i = 0; i < d.im; i++) {
        const long long c = idx3(d, i, j, k);
        const double dp = budget_dp(a, c, i);
        if (!(dp > 0.0)) continue;
        col += fmax(0.0, a.co2[c]) * (dp / a.g);
    }
    a.co2_total[(long long)j * d.pitch + k] = col;
}

// ---- standAtm_DewPoint_HumidRel ------------------------------------------------------

// one thread per cell; every output is a function of the cell and of its column's surface
// temperature, so the reference's column loop (and its copy of the tropopause value to the
// levels above it) becomes TempStand = TS_surface - 6.5e-3 * height[min(i, i_trop)]
__global__ void __launch_bounds__(128) stand_atm_kernel(StandAtmArgs a)
{
    using namespace thermo;
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const int i = blockIdx.z;
    if (k >= d.km) return;
    const long long c = idx3(d, i, j, k);
    const double t_0 = a.t_0;
    const double ts_surface = a.t[idx3(d, 0, j, k)] * t_0 - t_0;
    const int it = a.i_trop[j];
    a.temp_stand[c] = ts_surface - 6.5e-3 * a.height[(i <= it) ? i : it];
    const double t_u = a.t[c] * t_0;
    const double E = (t_u > t_0) ? saturation_pressure(t_u) : sublimation_pressure(t_u);
    const double x_v = x_H2O_of(a.c[c], a.co2[c], a.M_bg);
    double e = x_v * a.p_stat[c];
    const bool zero_vapour = (e <= 0.0);
    if (zero_vapour) e = 1e-3;
    a.temp_dew[c] = dew_point(e) - t_0;
    a.humid_rel[c] = (E <= 0.0) ? NO_SATURATION : (zero_vapour ? 0.0 : e / E * 100.0);
}

}  // namespace

void launch_find_residuum(const ResiduumArgs& a, cudaStream_t st)
{
    const int rows = (a.i1 >= a.i0 && a.d.jm > 2) ? (a.i1 - a.i0 + 1) * (a.d.jm - 2) : 0;
    if (rows > 0) residuum_rows_kernel<<<(rows + 7) / 8, 256, 0, st>>>(a, rows);
    residuum_final_kernel<<<1, 1024, 0, st>>>(a, rows);
}

void launch_budgets(const BudgetArgs& a, cudaStream_t st)
{
    const int rows = a.d.im * a.d.jm;
    budget_rows_kernel<<<(rows + 7) / 8, 256, 0, st>>>(a);
    budget_levels_kernel<<<a.d.im, 256, 0, st>>>(a);
    if (a.co2_total) co2_column_kernel<<<dim3((a.d.km + 127) / 128, a.d.jm), 128, 0, st>>>(a);
}

void launch_stand_atm(const StandAtmArgs& a, cudaStream_t st)
{
    stand_atm_kernel<<<dim3((a.d.km + 127) / 128, a.d.jm, a.d.im), 128, 0, st>>>(a);
}

void launch_min_max(const Dims& d, const double* x, double* scratch, double* out_v, long long* out_a,
                    cudaStream_t st)
{
    const int rows = d.im * d.jm;
    double* rv = scratch;
    long long* ra = reinterpret_cast<long long*>(scratch + 2 * (size_t)rows);
    minmax_rows_kernel<<<(rows + 7) / 8, 256, 0, st>>>(d, x, rv, ra);
    minmax_final_kernel<<<1, 1024, 0, st>>>(rows, rv, ra, out_v, out_a);
}

}  // namespace athad
