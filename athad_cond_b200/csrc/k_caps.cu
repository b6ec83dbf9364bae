// k_caps.cu - the moist iteration's bookkeeping after the ice scheme and the moist
// convection, on sm_100a:
//
//   moist_caps_kernel      UtilsAtm::precipitationSum (UtilsAtm.h:51-65), the +-1e-3 caps of
//                          the microphysics sources (cAtmosphereModel.cpp:1277-1297) and the
//                          cloud + ice cap at cloud_cap (:1310-1334): elementwise;
//   ceiling_rows_kernel    c kept in [0, 1 - co2] (:1369-1391), one warp per (i, j) row with
//                          the row's air mass and clipped water summed in a fixed order;
//   ceiling_sum_kernel     the row sums added in a fixed order by one CTA.
//
// The reference sums the air mass and the clipped water with an OpenMP reduction, whose
// result depends on the thread count; here the order is fixed, so the sums are
// deterministic (and differ from a serial sum only by rounding).
#include "kernels.cuh"

namespace athad {

namespace {

__global__ void __launch_bounds__(128) moist_caps_kernel(CapsArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= d.km) return;
    const long long c = idx3(d, i, j, k);
    a.Precipitation[c] = a.P_rain[c] + a.P_snow[c] + a.P_graupel[c] + a.P_conv[c];
    const double S_max = 1.0e-3;
#pragma unroll
    for (int s = 0; s < 7; s++) {
        double* S = a.S[s];
        const double v = S[c];
        if (!is_finite_bits(v)) S[c] = 0.0;
        else if (v > S_max) S[c] = S_max;
        else if (v < -S_max) S[c] = -S_max;
    }
    double cv = a.c[c], cld = a.cloud[c], ic = a.ice[c];
    if (!is_finite_bits(cv)) cv = 0.0;
    if (!is_finite_bits(cld)) cld = 0.0;
    if (!is_finite_bits(ic)) ic = 0.0;
    if (cv < 0.0) cv = 0.0;
    if (cld < 0.0) cld = 0.0;
    if (ic < 0.0) ic = 0.0;
    const double one_m = 1.0 - a.co2[c];
    const double cv_max = (0.0 < one_m) ? one_m : 0.0;
    if (cv > cv_max) cv = cv_max;
    const double sum = cld + ic;
    if (sum > a.cloud_cap) {
        const double scale = a.cloud_cap / sum;
        cld *= scale;
        ic *= scale;
    }
    a.c[c] = cv; a.cloud[c] = cld; a.ice[c] = ic;
}

__global__ void __launch_bounds__(256) ceiling_rows_kernel(CapsArgs a)
{
    const Dims& d = a.d;
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= d.im * d.jm) return;
    const int i = row / d.jm;
    const long long base = (long long)row * d.pitch;
    double w = 0.0, q = 0.0;
    unsigned hits = 0;
    for (int k = lane; k < d.km; k += 32) {
        const long long c = base + k;
        double cv = a.c[c];
        if (cv < 0.0) cv = 0.0;
        const double ps = a.p_stat[c];
        const double dp_Pa = (i < d.im - 1) ? (ps - a.p_stat[c + d.plane]) * 100.0 : ps * 100.0;
        const double u_air = (dp_Pa > 0.0) ? dp_Pa / a.g : 0.0;
        w += u_air;
        const double one_m = 1.0 - a.co2[c];
        const double c_ceiling = (0.0 < one_m) ? one_m : 0.0;
        if (cv > c_ceiling) {
            q += (cv - c_ceiling) * u_air;
            cv = c_ceiling;
            hits++;
        }
        a.c[c] = cv;
    }
    for (int off = 16; off >= 1; off >>= 1) {
        w += __shfl_xor_sync(0xffffffffu, w, off);
        q += __shfl_xor_sync(0xffffffffu, q, off);
        hits += __shfl_xor_sync(0xffffffffu, hits, off);
    }
    if (lane == 0) {
        a.row_q[row] = q;
        a.row_w[row] = w;
        if (hits) atomicAdd(a.count, (unsigned long long)hits);
    }
}

__global__ void __launch_bounds__(1024) ceiling_sum_kernel(CapsArgs a)
{
    const int rows = a.d.im * a.d.jm;
    double q = 0.0, w = 0.0;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) { q += a.row_q[r]; w += a.row_w[r]; }
    __shared__ double sq[32], sw[32];
    for (int off = 16; off >= 1; off >>= 1) {
        q += __shfl_xor_sync(0xffffffffu, q, off);
        w += __shfl_xor_sync(0xffffffffu, w, off);
    }
    if ((threadIdx.x & 31) == 0) { sq[threadIdx.x >> 5] = q; sw[threadIdx.x >> 5] = w; }
    __syncthreads();
    if (threadIdx.x < 32) {
        q = sq[threadIdx.x]; w = sw[threadIdx.x];
        for (int off = 16; off >= 1; off >>= 1) {
            q += __shfl_xor_sync(0xffffffffu, q, off);
            w += __shfl_xor_sync(0xffffffffu, w, off);
        }
        if (threadIdx.x == 0) { a.sums[0] = q; a.sums[1] = w; }
    }
}

}  // namespace

void launch_moist_caps(const CapsArgs& a, cudaStream_t st)
{
    moist_caps_kernel<<<dim3((a.d.km + 127) / 128, a.d.jm, a.d.im), 128, 0, st>>>(a);
}

void launch_vapour_ceiling(const CapsArgs& a, cudaStream_t st)
{
    const int rows = a.d.im * a.d.jm;
    ceiling_rows_kernel<<<(rows + 7) / 8, 256, 0, st>>>(a);
    ceiling_sum_kernel<<<1, 1024, 0, st>>>(a);
}

}  // namespace athad
