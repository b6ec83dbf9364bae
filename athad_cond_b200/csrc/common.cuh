// common.cuh - device-side helpers shared by the sm_100a kernels of the ATHAD_COND
// hot path: comparison helpers with the C++ standard library's exact semantics, the
// IEEE non-finite test of lib/Utils.h:121-125, field addressing and the launch-time
// constants every kernel receives by value.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/athad_gpu.h"

#define ATHAD_HD __host__ __device__ __forceinline__

namespace athad {

// std::max / std::min / std::clamp exactly: (a < b) ? b : a etc.  fmax/fmin differ on NaN
// and signed zero, and the reference's results depend on which operand survives.
ATHAD_HD double smax(double a, double b) { return (a < b) ? b : a; }
ATHAD_HD double smin(double a, double b) { return (b < a) ? b : a; }
ATHAD_HD double sclamp(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

ATHAD_HD bool is_finite_bits(double v)
{
#ifdef __CUDA_ARCH__
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
#else
    unsigned long long b;
    __builtin_memcpy(&b, &v, sizeof b);
#endif
    return (b & 0x7FF0000000000000ULL) != 0x7FF0000000000000ULL;
}

// safe_clamp of RungeKutta_Atm_Turb.cpp:76-81
ATHAD_HD double safe_clamp(double v, double lo, double hi)
{
    if (!is_finite_bits(v)) return lo;
    return (v < lo) ? lo : (v > hi) ? hi : v;
}

// Per-(i,j) metric factors of cAtmosphereModel::CellGeometry (cAtmosphereModel.h:170-178),
// built on the host once per context exactly as RungeKutta_Atm_Turb.cpp:104-135 builds
// them, with mirror-symmetric sin/cos tables.
struct GeoIJ {
    double exp_rm, exp_2_rm, sinthe, sinthe2, costhe;
    double inv_rm, inv_rm2, inv_rmsinthe, inv_rm2sinthe, inv_rm2sinthe2, costhe_inv_rm2sinthe;
    // products the right-hand side forms from the factors above, evaluated once per (i,j)
    // with the same operations: 2*inv_rm*exp_rm (RHS_Atm_Turb.cpp:858),
    // (1 + costhe^2/sinthe2)*inv_rm2 (:864), sinthe2^2 (:985)
    double two_over_rm_exp, v_metric, cos4lat;
};

// Grid extents and the strides of a pitched field: element (i,j,k) is at
// ((i*jm + j)*pitch + k).
struct Dims {
    int im, jm, km;
    int pitch;            // row length in elements (>= km, multiple of 32)
    long long plane;      // jm * pitch
    long long fstride;    // im * jm * pitch: distance between consecutive fields
};

ATHAD_HD long long idx3(const Dims& d, int i, int j, int k)
{
    return ((long long)i * d.jm + j) * d.pitch + k;
}

// Programmatic dependent launch (sm_90 and later): a kernel launched with launch_dependent
// may be scheduled while the kernel before it in the stream is still running; it calls
// pdl_wait() before its first global memory access, which returns once that kernel has
// completed and its writes are visible, so stream order holds for every access.  The
// kernel before it calls pdl_trigger() to let the dependent's CTAs onto the SMs its last
// wave frees instead of after its completion.  Both are no-ops in a kernel launched
// without the attribute (the batched RK4 kernels, the kernels shared with other paths).
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_dependent(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                    cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

}  // namespace athad
