// k_noalloc.cu - an entry point that allocates no device memory.
//
// Some hosts of this library cannot call cudaMalloc at the point where they need the
// result: a process that reserved its whole HBM budget up front and admits work only
// against that budget, a real-time loop that must not pay cudaMalloc's implicit device
// synchronisation in its step, or a caller whose device memory is handed to it by another
// runtime.  athad_density_profile_noalloc gives them the density profile of
// ThermoAtm::densities (the horizontal mean rho_bar(i) and d ln rho_bar / d rad.z) from a
// density field they already hold on the device, without a context.
//
// Its scratch (the per-row partial sums) lives in the file-scope device array below, of a
// fixed size: every GPU that loads this library keeps it until the process exits.  Host
// code cannot use the array's name as a device address, so the address is looked up once
// per device with cudaGetSymbolAddress, on that device's first call (make that first call
// before any stream capture).  The address is kept for the life of the process, so
// resetting a device (cudaDeviceReset) between calls is not supported.  All calls share the
// array: calls that overlap on the GPU (different streams or host threads) race on it.
// Every entry a call reads is written earlier in the same call, so nothing needs clearing
// between calls.  A CUDA error already pending when the call starts is left pending and
// reported (ATHAD_ERR_CUDA) before anything is launched.
#include <cmath>
#include <mutex>

#include "kernels.cuh"

namespace athad {

// Scratch: row sums and row counts of up to ATHAD_NOALLOC_MAX_ROWS (i, j) rows.
static __device__ __align__(256) double g_noalloc_scratch[2 * ATHAD_NOALLOC_MAX_ROWS];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[kMaxDevices] = {};

// per-(i,j) row sum and count of the positive densities, fixed warp order
__global__ void __launch_bounds__(256) noalloc_rowsum_kernel(const double* __restrict__ r, int im, int jm,
                                                             int km, long long pitch, double* __restrict__ sum,
                                                             double* __restrict__ cnt)
{
    const int lane = threadIdx.x & 31;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= im * jm) return;
    const double* p = r + (long long)row * pitch;
    double s = 0.0, q = 0.0;
    for (int k = lane; k < km; k += 32) {
        const double v = p[k];
        if (v > 0.0) { s += v; q += 1.0; }
    }
    for (int off = 16; off >= 1; off >>= 1) {
        s = s + __shfl_xor_sync(0xffffffffu, s, off);
        q = q + __shfl_xor_sync(0xffffffffu, q, off);
    }
    if (lane == 0) { sum[row] = s; cnt[row] = q; }
}

// rho_bar(i) from the row sums (rows j and jm-1-j paired, cos-latitude weights of
// ThermoAtm.h:1636), then its log-derivative (:1652-1659); one thread per level
__global__ void noalloc_profile_kernel(int im, int jm, double inv_2dr, double inv_dr,
                                       double* __restrict__ sum, const double* __restrict__ cnt,
                                       double* __restrict__ rho_base, double* __restrict__ dlnrho)
{
    const int i = threadIdx.x;
    if (i < im) {
        double num = 0.0, den = 0.0;
        for (int j = 0; j <= jm / 2; j++) {
            const int jr = jm - 1 - j;
            if (jr < j) break;
            const double cl = cos((j / (double)(jm - 1) - 0.5) * M_PI);
            const double s0 = sum[i * jm + j], c0 = cnt[i * jm + j];
            if (jr != j) {
                num += cl * (s0 + sum[i * jm + jr]);
                den += cl * (c0 + cnt[i * jm + jr]);
            } else {
                num += cl * s0;
                den += cl * c0;
            }
        }
        const double rb = (den > 0.0) ? num / den : 0.0;
        rho_base[i] = rb;
        sum[i * jm] = (rb > 0.0) ? log(rb) : 0.0;   // ln rho_bar, read back below
    }
    __syncthreads();
    if (i < im) {
        double v = 0.0;
        if (i >= 1 && i < im - 1) v = (sum[(i + 1) * jm] - sum[(i - 1) * jm]) * inv_2dr;
        else if (i == 0 && im > 1) v = (sum[1 * jm] - sum[0]) * inv_dr;
        else if (i == im - 1 && im > 1) v = (sum[(im - 1) * jm] - sum[(im - 2) * jm]) * inv_dr;
        dlnrho[i] = v;
    }
}

}  // namespace
}  // namespace athad

using namespace athad;

extern "C" athad_status athad_density_profile_noalloc(const double* r_humid, int32_t im, int32_t jm,
                                                       int32_t km, size_t pitch, double* rho_base,
                                                       double* dlnrho_dr, void* cuda_stream)
{
    if (!r_humid || !rho_base || !dlnrho_dr) return ATHAD_ERR_INVALID;
    if (im < 2 || jm < 1 || km < 1 || pitch < (size_t)km) return ATHAD_ERR_INVALID;
    if (im > ATHAD_NOALLOC_MAX_IM || (long long)im * jm > ATHAD_NOALLOC_MAX_ROWS) return ATHAD_ERR_INVALID;
    if (cudaPeekAtLastError() != cudaSuccess) return ATHAD_ERR_CUDA;   // an earlier call's error
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return ATHAD_ERR_NO_DEVICE;
    }
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_ptr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                return ATHAD_ERR_CUDA;
            }
            g_noalloc_ptr[dev] = (double*)p;
        }
        scratch = g_noalloc_ptr[dev];
    }
    cudaStream_t st = (cudaStream_t)cuda_stream;
    double* sum = scratch;
    double* cnt = scratch + ATHAD_NOALLOC_MAX_ROWS;
    const int rows = im * jm;
    noalloc_rowsum_kernel<<<(rows + 7) / 8, 256, 0, st>>>(r_humid, im, jm, km, (long long)pitch, sum, cnt);
    const double dr = 1.0 / (double)(im - 1);
    noalloc_profile_kernel<<<1, ((im + 31) / 32) * 32, 0, st>>>(im, jm, 1.0 / (2.0 * dr), 1.0 / dr, sum, cnt,
                                                               rho_base, dlnrho_dr);
    if (cudaGetLastError() != cudaSuccess) return ATHAD_ERR_CUDA;
    return ATHAD_OK;
}
