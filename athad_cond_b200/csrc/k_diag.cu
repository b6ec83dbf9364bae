// k_diag.cu - diagnostics on the device: cAtmosphereModel::searchMinMax_3D
// (MinMax_Atm.cpp:51-109), the largest and smallest finite value of a field and the first
// cell in (i, j, k) order holding each.
//
// One warp per (i, j) row scans its longitudes lane-strided, keeping the first position of a
// strictly larger (smaller) value, and combines lanes preferring the smaller longitude on a
// tie; one CTA then combines the rows in order, preferring the smaller row.  The result is
// the serial scan's, whatever the launch shape.
#include <cfloat>

#include "kernels.cuh"

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

}  // namespace

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
