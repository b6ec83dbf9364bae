// k_filters.cu - the smoothing filters of the model iteration on sm_100a, flat terrain
// (every cell is fluid; the orographic, steep-massif and coastal filters flag nothing):
//
//   athad_post_rk4_filters (cAtmosphereModel.cpp:1507-1520)
//     AtomUtils::polar_zonal_filter of u, v, w (lib/Utils.cpp:542-611): per row j a
//       number of periodic 1-2-1 passes along k that grows toward the poles;
//     AtomUtils::radial_shapiro_filter of u (:831-873): two 1-2-1 passes along i;
//     AtomUtils::radial_shapiro_filter_ho of v, w (:884-940): two 4th-order passes along
//       i, the 1-2-1 where i+-2 is outside the column;
//   athad_damp_wiggles (:429-531): one 1-2-1 pass along k (periodic), j (clamped) and i
//     (clamped), the moist iteration's de-checkerboarding of t, ice, c, cloud
//     (cAtmosphereModel.cpp:1225-1228).
//
// Every pass of the reference works from a snapshot of the field.  Along k a CTA holds
// its row in shared memory and iterates its passes there; along i a thread walks its
// column with the snapshot values it still needs in registers; along j one out-of-place
// launch.  Compiled without fused multiply-add: bit-identical to the reference.
#include "kernels.cuh"

namespace athad {

namespace {

// periodic 1-2-1 passes along k of one row per CTA; passes[j] of them (zero: untouched)
__global__ void __launch_bounds__(128) zonal_rows_kernel(FilterArgs a, int nfields, int const_passes)
{
    extern __shared__ double row[];          // two buffers of km
    const Dims& d = a.d;
    const int j = blockIdx.x, i = blockIdx.y, q = blockIdx.z;
    if (q >= nfields) return;
    const int np = const_passes >= 0 ? const_passes : a.polar_passes[j];
    if (np == 0) return;
    double* x = a.field[q] + idx3(d, i, j, 0);
    const double* xs = a.src[q] ? a.src[q] + idx3(d, i, j, 0) : x;
    double* b0 = row;
    double* b1 = row + d.km;
    for (int k = threadIdx.x; k < d.km; k += blockDim.x) b0[k] = xs[k];
    __syncthreads();
    for (int pass = 0; pass < np; pass++) {
        for (int k = threadIdx.x; k < d.km; k += blockDim.x) {
            const int km1 = (k == 0) ? d.km - 1 : k - 1;
            const int kp1 = (k == d.km - 1) ? 0 : k + 1;
            b1[k] = b0[k] + 0.25 * (b0[km1] - 2.0 * b0[k] + b0[kp1]);
        }
        __syncthreads();
        double* t = b0; b0 = b1; b1 = t;
    }
    for (int k = threadIdx.x; k < d.km; k += blockDim.x) x[k] = b0[k];
}

// two passes along i of one column per thread: field 0 (u) 1-2-1, fields 1-2 (v, w) the
// 4th-order Shapiro filter; rows 0 and im-1 untouched
__global__ void __launch_bounds__(128) radial_columns_kernel(FilterArgs a)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, q = blockIdx.z;
    if (k >= d.km) return;
    double* x = a.field[q] + idx3(d, 0, j, k);
    const long long s = d.plane;
    const int im = d.im;
    for (int pass = 0; pass < 2; pass++) {
        // snapshot window o[i-2 .. i+2] of the values before this pass
        double om2 = 0.0, om1 = x[0], o0 = x[s], op1 = (im > 2) ? x[2 * s] : 0.0;
        for (int i = 1; i < im - 1; i++) {
            const double op2 = (i + 2 <= im - 1) ? x[(i + 2) * s] : 0.0;
            double v;
            if (q != 0 && i - 2 >= 0 && i + 2 <= im - 1) {
                const double d4 = op2 - 4.0 * op1 + 6.0 * o0 - 4.0 * om1 + om2;
                v = o0 - 0.0625 * d4;
            } else {
                v = o0 + 0.25 * (om1 - 2.0 * o0 + op1);
            }
            x[i * s] = v;
            om2 = om1; om1 = o0; o0 = op1; op1 = op2;
        }
    }
}

// damp_wiggles along j then along i (both clamped), one thread per cell, out of place: the
// radial pass reads only the meridional pass's values at i-1, i, i+1 of its own column, so
// the thread forms those three (from the zonal pass's output) and writes the cell's result.
// The meridional pass adds the two neighbours first, so the result at row jm-1-j is bit for
// bit the result at row j of the mirrored field; the reference's left-to-right
// (v[j-1] - 2 v[j]) + v[j+1] rounds the mirrored rows differently (an ulp at most).
__global__ void __launch_bounds__(128) wiggle_ji_kernel(Dims d, const double* __restrict__ src, double* __restrict__ dst)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= d.km) return;
    const int jm1 = (j > 0) ? j - 1 : 0, jp1 = (j < d.jm - 1) ? j + 1 : d.jm - 1;
    const int im1 = (i > 0) ? i - 1 : 0, ip1 = (i < d.im - 1) ? i + 1 : d.im - 1;
    double v[3];
    const int ii[3] = {im1, i, ip1};
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const double c = src[idx3(d, ii[q], j, k)];
        v[q] = c + 0.25 * ((src[idx3(d, ii[q], jm1, k)] + src[idx3(d, ii[q], jp1, k)]) - 2.0 * c);
    }
    dst[idx3(d, i, j, k)] = v[1] + 0.25 * (v[0] - 2.0 * v[1] + v[2]);
}

}  // namespace

void launch_post_rk4_filters(const FilterArgs& a, cudaStream_t st)
{
    const Dims& d = a.d;
    zonal_rows_kernel<<<dim3(d.jm, d.im, 3), 128, 2 * d.km * sizeof(double), st>>>(a, 3, -1);
    radial_columns_kernel<<<dim3((d.km + 127) / 128, d.jm, 3), 128, 0, st>>>(a);
}

void launch_damp_wiggles(const Dims& d, double* f, double* scratch, cudaStream_t st)
{
    FilterArgs a{};
    a.d = d;
    a.field[0] = scratch;
    a.src[0] = f;
    // along k: the row kernel with one pass, reading f's rows and writing scratch
    zonal_rows_kernel<<<dim3(d.jm, d.im, 1), 128, 2 * d.km * sizeof(double), st>>>(a, 1, 1);
    wiggle_ji_kernel<<<dim3((d.km + 127) / 128, d.jm, d.im), 128, 0, st>>>(d, scratch, f);
}

}  // namespace athad
