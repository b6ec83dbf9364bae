// k_thermo.cu - the device thermodynamics (thermo.cuh) evaluated on the GPU for given
// inputs (athad_thermo_eval): the functions every column kernel calls, exposed so that the
// reference's own known answers (test/saturation_selftest.cpp, test/cond_column_selftest.cpp)
// can be checked against the device code itself rather than only through the kernels.
#include <vector>

#include "kernels.cuh"
#include "thermo.cuh"

namespace athad {
namespace {

// __host__ __device__: tests/host_thermo.cu evaluates the same source on the host
__host__ __device__ double eval_one(int fn, const double* x)
{
    switch (fn) {
        case ATHAD_THERMO_SATURATION_PRESSURE:      return thermo::saturation_pressure(x[0]);
        case ATHAD_THERMO_SUBLIMATION_PRESSURE:     return thermo::sublimation_pressure(x[0]);
        case ATHAD_THERMO_LATENT_HEAT:              return thermo::latent_heat(x[0]);
        case ATHAD_THERMO_SATURATION_MASS_FRACTION: return thermo::saturation_mass_fraction(x[0], x[1], x[2]);
        case ATHAD_THERMO_DEW_POINT:                return thermo::dew_point(x[0]);
        case ATHAD_THERMO_CP_OF:                    return thermo::cp_of(x[0], x[1], x[2], x[3]);
        case ATHAD_THERMO_M_NONWATER:               return thermo::M_nonwater(x[0], x[1], x[2]);
        case ATHAD_THERMO_MOIST_LAPSE:              return thermo::moist_lapse(x[0], x[1], x[2], x[3], x[4], x[5]);
        case ATHAD_THERMO_R_OF:                     return thermo::R_of(x[0], x[1], x[2]);
        case ATHAD_THERMO_SATURATION_MASS_FRACTION_AT:
            return thermo::saturation_mass_fraction_at(x[0], x[1], x[2]);
        case ATHAD_THERMO_DQSAT_DT:                 return thermo::dqsat_dT(x[0], x[1], x[2]);
        default:                                    return 0.0;
    }
}

__global__ void thermo_eval_kernel(int fn, int n, int stride, const double* in, double* out)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) out[q] = eval_one(fn, in + (long long)q * stride);
}

int arity(int fn)
{
    switch (fn) {
        case ATHAD_THERMO_SATURATION_PRESSURE: case ATHAD_THERMO_SUBLIMATION_PRESSURE:
        case ATHAD_THERMO_LATENT_HEAT: case ATHAD_THERMO_DEW_POINT:
            return 1;
        case ATHAD_THERMO_SATURATION_MASS_FRACTION: case ATHAD_THERMO_M_NONWATER: case ATHAD_THERMO_R_OF:
        case ATHAD_THERMO_SATURATION_MASS_FRACTION_AT: case ATHAD_THERMO_DQSAT_DT:
            return 3;
        case ATHAD_THERMO_CP_OF:
            return 4;
        case ATHAD_THERMO_MOIST_LAPSE:
            return 6;
        default:
            return 0;
    }
}

}  // namespace
}  // namespace athad

using namespace athad;

extern "C" int32_t athad_thermo_arity(int32_t fn) { return arity(fn); }

extern "C" athad_status athad_thermo_eval(int32_t fn, int32_t n, const double* in, double* out)
{
    const int a = arity(fn);
    if (a == 0 || n < 0 || (n > 0 && (!in || !out))) return ATHAD_ERR_INVALID;
    if (n == 0) return ATHAD_OK;
    if (cudaPeekAtLastError() != cudaSuccess) return ATHAD_ERR_CUDA;
    double* d_in = nullptr;
    double* d_out = nullptr;
    const size_t bin = (size_t)n * a * sizeof(double), bout = (size_t)n * sizeof(double);
    if (cudaMalloc((void**)&d_in, bin) != cudaSuccess || cudaMalloc((void**)&d_out, bout) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(d_in);
        return ATHAD_ERR_OOM;
    }
    athad_status s = ATHAD_OK;
    if (cudaMemcpy(d_in, in, bin, cudaMemcpyHostToDevice) != cudaSuccess) s = ATHAD_ERR_CUDA;
    if (s == ATHAD_OK) {
        thermo_eval_kernel<<<(n + 127) / 128, 128>>>(fn, n, a, d_in, d_out);
        if (cudaGetLastError() != cudaSuccess) s = ATHAD_ERR_CUDA;
    }
    if (s == ATHAD_OK && cudaMemcpy(out, d_out, bout, cudaMemcpyDeviceToHost) != cudaSuccess) s = ATHAD_ERR_CUDA;
    cudaFree(d_in);
    cudaFree(d_out);
    return s;
}
