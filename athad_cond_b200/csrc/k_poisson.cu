// k_poisson.cu - pressure-Poisson relaxation of the ATHAD_COND atmosphere on sm_100a.
//
// Replaces PressureSolverAtm::run (PressureSolverAtm.h:27-594) for flat terrain, and the
// gradient correction of PressureSolverAtm::project_initial_velocity (:713-749).
//
// A sweep is the clamped divergence of aux_u/v/w (the Poisson source, from the reference's
// operands) into a scratch field, the two colours, the boundary passes and the ceiling:
// five launches, each after the first issued as a programmatic dependent launch.  Within
// one colour every cell reads only cells of the other colour, so the in-place update is
// order-independent and the result equals the serial red-black sweep bit for bit.
#include <algorithm>

#include "kernels.cuh"

namespace athad {

// The aux radial boundary (PressureSolverAtm.h:106-121) and the clamped divergence source
// (:415-473, central differences) in one launch.  c43 and c13 are `const int` members
// initialised from 4.0/3.0 and 1.0/3.0 (cAtmosphereModel.h:158): 1 and 0.  The threads of
// the planes i = 0 and im-1 write the boundary values; the interior cells next to them form
// the same value from the interior instead of reading it, so the launch has no order.
__device__ __forceinline__ double aux_u_lid(const PoissonArgs& a, double inner, double second)
{
    const double c43 = 1.0, c13 = 0.0;
    return a.anelastic ? 0.0 : c43 * inner - c13 * second;
}

// the aux values of the planes i = 0 and im-1 at (j, k), formed from the interior
__device__ __forceinline__ void aux_lid_cell(const PoissonArgs& a, int i, int j, int k)
{
    const Dims& d = a.d;
    const double c43 = 1.0, c13 = 0.0;
    const long long cb = idx3(d, i, j, k);
    const long long s = (i == 0) ? d.plane : -d.plane;   // toward the interior
    a.aux_u[cb] = aux_u_lid(a, a.aux_u[cb + s], a.aux_u[cb + 2 * s]);
    a.aux_v[cb] = c43 * a.aux_v[cb + s] - c13 * a.aux_v[cb + 2 * s];
    a.aux_w[cb] = c43 * a.aux_w[cb + s] - c13 * a.aux_w[cb + 2 * s];
}

// the clamped divergence source of fluid cell c = (i, j, k); it reads aux_u/v/w of the
// interior only (the lid through aux_u_lid)
__device__ __forceinline__ double cell_source(const PoissonArgs& a, const PoiIJ& P, int i, long long c,
                                              bool& clamped)
{
    const Dims& d = a.d;
    const long long sI = d.plane, sJ = d.pitch;
    const double u_c = __ldg(a.aux_u + c);
    const double u_up = (i + 1 == d.im - 1) ? aux_u_lid(a, u_c, __ldg(a.aux_u + c - sI)) : __ldg(a.aux_u + c + sI);
    const double u_dn = (i - 1 == 0) ? aux_u_lid(a, u_c, __ldg(a.aux_u + c + sI)) : __ldg(a.aux_u + c - sI);
    const double du_dr = (u_up - u_dn) * a.inv_2dr;
    const double dv_dthe = (__ldg(a.aux_v + c + sJ) - __ldg(a.aux_v + c - sJ)) * a.inv_2dthe;
    const double dw_dphi = (__ldg(a.aux_w + c + 1) - __ldg(a.aux_w + c - 1)) * a.inv_2dphi;
    double div_src = du_dr * P.exp_rm + dv_dthe * P.inv_rm + dw_dphi * P.inv_rmsinthe;
    if (a.anelastic) div_src += u_c * __ldg(a.dlnrho + i) * P.exp_rm;
    if (a.metric_div) div_src += (2.0 * u_c + __ldg(a.aux_v + c) * P.costhe / P.sinthe) * P.inv_rm;
    const double src_max = P.denom * 2.0;   // p_dyn_cap = 2 (:148)
    clamped = false;
    if (!is_finite_bits(div_src)) div_src = 0.0;
    else if (div_src > src_max) { div_src = src_max; clamped = true; }
    else if (div_src < -src_max) { div_src = -src_max; clamped = true; }
    return div_src;
}

// clamped sources are rare, so a warp adds its count only when it has one: no atomics and
// no block barrier on the common path (the fluid cells, (im-2)(jm-2)(km-2) per sweep, are
// counted by the host)
__device__ __forceinline__ void count_clamped(const PoissonArgs& a, bool clamped)
{
    const unsigned nc = __popc(__ballot_sync(0xffffffffu, clamped));
    if ((threadIdx.x & 31) == 0 && nc && a.counters) atomicAdd(a.counters + 1, (unsigned long long)nc);
}

// The source into a scratch field (the sweep's colours and the Poisson solve read it), with
// the aux boundary
__global__ void __launch_bounds__(256) poisson_src_kernel(PoissonArgs a)
{
    pdl_trigger();
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    // the sweep's "a value reached the ceiling" flag starts clear (the colours set it)
    if (a.counters && (blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0)
        a.counters[5] = 0ull;
    if ((i == 0 || i == d.im - 1) && k >= 1 && k < d.km - 1 && j >= 1 && j < d.jm - 1) aux_lid_cell(a, i, j, k);
    const bool fluid = (k >= 1 && k < d.km - 1 && j >= 1 && j < d.jm - 1 && i >= 1 && i < d.im - 1);
    bool clamped = false;
    if (fluid) {
        const long long c = idx3(d, i, j, k);
        const PoiIJ P = a.poi[i * d.jm + j];
        a.src[c] = cell_source(a, P, i, c, clamped);
    }
    count_clamped(a, clamped);
}

// one colour of the red-black sweep, PressureSolverAtm.h:225-486 (update :475-480); thread
// kk of row (i, j) takes the kk-th cell of the colour, k = 2 kk + ((i + j + COLOUR) & 1),
// so every lane of a warp updates a cell
// ATHAD_POISSON_SRC_FIELD 1: the source formed by its own launch into a scratch field that
// both colours read; 0: each colour forms its cells' sources from aux_u/v/w.  The pressure
// call at 41x181x361 inside the model iteration (PDL on, mixed form, 300 iterations):
// 59.1 us with the source field, 68.8 us forming the sources in the colours (46 registers,
// 5 CTAs of 256 per SM), 63.7 us at 8 CTAs (spills), 60.0 us at 6.
#ifndef ATHAD_POISSON_SRC_FIELD
#define ATHAD_POISSON_SRC_FIELD 1
#endif
#ifndef ATHAD_POISSON_MIN_BLOCKS
#define ATHAD_POISSON_MIN_BLOCKS 1
#endif
template <int COLOUR>
__global__ void __launch_bounds__(256, ATHAD_POISSON_MIN_BLOCKS) poisson_colour_kernel(PoissonArgs a)
{
    pdl_trigger();
    pdl_wait();
    const Dims& d = a.d;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    const int k = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((i + j + COLOUR) & 1);
    const bool fluid = !(k < 1 || k >= d.km - 1 || j < 1 || j >= d.jm - 1 || i < 1 || i >= d.im - 1);
    bool clamped = false, beyond = false;
    if (fluid) {
        const long long c = idx3(d, i, j, k);
        const PoiIJ P = a.poi[i * d.jm + j];
#if ATHAD_POISSON_SRC_FIELD
        const double src = __ldg(a.src + c);
#else
        const double src = cell_source(a, P, i, c, clamped);
#endif
        const long long sI = d.plane, sJ = d.pitch;
        const double* p = a.p;
        const double pip = p[c + sI], pim = p[c - sI];
        const double num_a = a.anelastic ? P.exp_2_rm * __ldg(a.dlnrho + i) * a.inv_2dr : 0.0;
        const double v = ((pip + pim) * P.num1
                        + (p[c + sJ] + p[c - sJ]) * P.num2
                        + (p[c + 1] + p[c - 1]) * P.num3
                        + (pip - pim) * num_a
                        - src) * P.inv_denom;
        a.p[c] = v;
        beyond = !(fabs(v) <= a.ceiling);      // non-finite included
    }
    count_clamped(a, clamped);
    // one atomic per warp that has such a value (rare): the ceiling pass runs only then
    if (__any_sync(0xffffffffu, beyond) && (threadIdx.x & 31) == 0 && a.counters)
        atomicOr(a.counters + 5, 1ull);
}

// The three boundary passes (radial, pole, seam, PressureSolverAtm.h:504-552) in one launch.
// Run in that order, they leave every boundary cell a value that depends on interior cells
// only: lin(a, b) = 1 * a - 0 * b (c43, c13) for the radial and seam extrapolations, copies
// for the lid and the poles, the seam the average of its two extrapolations.  Each thread
// forms the final value of one boundary cell from the interior, which this launch does not
// write, so the cells need no order.  The face groups overlap at edges and corners, where
// two threads write the same value.
__device__ __forceinline__ double bc_lin(double a, double b) { return 1.0 * a - 0.0 * b; }

// after the radial pass, at (i, j, k) with j and k interior
__device__ __forceinline__ double bc_radial(const Dims& d, const double* p, int i, int j, int k)
{
    if (i == 0) return bc_lin(p[idx3(d, 1, j, k)], p[idx3(d, 2, j, k)]);
    if (i == d.im - 1) return p[idx3(d, d.im - 2, j, k)];
    return p[idx3(d, i, j, k)];
}
// after the radial and pole passes, k interior
__device__ __forceinline__ double bc_pole(const Dims& d, const double* p, int i, int j, int k)
{
    const int jj = (j == 0) ? 1 : (j == d.jm - 1) ? d.jm - 2 : j;
    return bc_radial(d, p, i, jj, k);
}
__device__ __forceinline__ double bc_final(const Dims& d, const double* p, int i, int j, int k)
{
    if (k == 0 || k == d.km - 1) {
        const double r0 = bc_lin(bc_pole(d, p, i, j, 1), bc_pole(d, p, i, j, 2));
        const double r1 = bc_lin(bc_pole(d, p, i, j, d.km - 2), bc_pole(d, p, i, j, d.km - 3));
        return (r0 + r1) / 2.0;
    }
    return bc_pole(d, p, i, j, k);
}

// one flat grid over the three face groups: the planes i = 0, im-1 (2 jm km cells), the rows
// j = 0, jm-1 (2 im km) and the seam columns k = 0, km-1 (2 im jm)
__global__ void __launch_bounds__(128) poisson_bc_kernel(PoissonArgs a)
{
    pdl_trigger();
    pdl_wait();
    const Dims& d = a.d;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n_planes = 2LL * d.jm * d.km, n_rows = 2LL * d.im * d.km, n_seam = 2LL * d.im * d.jm;
    int i, j, k;
    bool plane = false;
    if (t < n_planes) {
        const int side = (int)(t / ((long long)d.jm * d.km));
        const int r = (int)(t % ((long long)d.jm * d.km));
        i = side ? d.im - 1 : 0; j = r / d.km; k = r % d.km;
        plane = true;
    } else if ((t -= n_planes) < n_rows) {
        const int side = (int)(t / ((long long)d.im * d.km));
        const int r = (int)(t % ((long long)d.im * d.km));
        j = side ? d.jm - 1 : 0; i = r / d.km; k = r % d.km;
    } else if ((t -= n_rows) < n_seam) {
        const int side = (int)(t / ((long long)d.im * d.jm));
        const int r = (int)(t % ((long long)d.im * d.jm));
        k = side ? d.km - 1 : 0; i = r / d.jm; j = r % d.jm;
    } else {
        return;
    }
    a.p[idx3(d, i, j, k)] = bc_final(d, a.p, i, j, k);
    if (a.aux_lid && plane && k >= 1 && k < d.km - 1 && j >= 1 && j < d.jm - 1)
        aux_lid_cell(a, i, j, k);   // the aux radial boundary, PressureSolverAtm.h:106-121
}

// aux_lid: also the aux radial boundary (a sweep whose source launch wrote it passes 0)
static void launch_bcs(const PoissonArgs& a, cudaStream_t st)
{
    const Dims& d = a.d;
    const long long n = 2LL * d.jm * d.km + 2LL * d.im * d.km + 2LL * d.im * d.jm;
    launch_dependent(poisson_bc_kernel, dim3((unsigned)((n + 127) / 128)), dim3(128), 0, st, a);
}

// |p_dyn| ceiling (:583-594); writes only where the value changes.  A thread takes four
// consecutive longitudes of one pitched row (two 16-byte loads; the pitch is a multiple of
// 32), so a warp has 1 KB of loads in flight
__device__ __forceinline__ bool ceiling_of(double v, double cap, double& out)
{
    if (!is_finite_bits(v)) { out = 0.0; return true; }
    if (v > cap) { out = cap; return true; }
    if (v < -cap) { out = -cap; return true; }
    return false;
}

__global__ void __launch_bounds__(256) poisson_ceiling_kernel(PoissonArgs a)
{
    pdl_wait();
    const Dims& d = a.d;
    // the sweep's clamped sources into the call's count (counters[0]), the accumulator
    // cleared for the next sweep: every launch that added to it has completed, and the
    // next source launch waits for this one, so no memset precedes a call
    if (blockIdx.x == 0 && threadIdx.x == 0 && a.counters) {
        const unsigned long long n = a.counters[1];
        a.counters[0] = a.first_sweep ? n : a.counters[0] + n;
        a.counters[1] = 0ull;
    }
    // Every cell is a value the colours just formed or a boundary value copied or averaged
    // from such values, so when no colour formed a value beyond the ceiling (or a
    // non-finite one) the ceiling changes nothing and the launch ends here.
    if (a.counters && a.counters[5] == 0ull) return;
    const long long n = (long long)d.im * d.plane;
    for (long long q = 4LL * ((long long)blockIdx.x * blockDim.x + threadIdx.x); q < n;
         q += 4LL * gridDim.x * blockDim.x) {
        const int k0 = (int)(q % d.pitch);
        const double2* p2 = reinterpret_cast<const double2*>(a.p + q);
        const double2 v01 = p2[0], v23 = p2[1];
        const double v[4] = {v01.x, v01.y, v23.x, v23.y};
#pragma unroll
        for (int e = 0; e < 4; e++) {
            double w;
            if (k0 + e < d.km && ceiling_of(v[e], a.ceiling, w)) a.p[q + e] = w;
        }
    }
}

void launch_poisson_prepare(const PoissonArgs& a, cudaStream_t st)
{
    const Dims& d = a.d;
    const dim3 block(32, 8), grid((d.km + 31) / 32, (d.jm + 7) / 8, d.im);
    poisson_src_kernel<<<grid, block, 0, st>>>(a);
}

void launch_poisson_sweep(const PoissonArgs& a, cudaStream_t st)
{
    const Dims& d = a.d;
    const dim3 block(32, 8), grid((d.km + 31) / 32, (d.jm + 7) / 8, d.im);
    const dim3 half_grid(((d.km + 1) / 2 + 31) / 32, (d.jm + 7) / 8, d.im);
    // each launch after the first waits for the one before it (pdl_wait) but is scheduled
    // during its tail
#if ATHAD_POISSON_SRC_FIELD
    poisson_src_kernel<<<grid, block, 0, st>>>(a);
    launch_dependent(poisson_colour_kernel<0>, half_grid, block, 0, st, a);
#else
    poisson_colour_kernel<0><<<half_grid, block, 0, st>>>(a);
#endif
    launch_dependent(poisson_colour_kernel<1>, half_grid, block, 0, st, a);
#if ATHAD_POISSON_SRC_FIELD
    PoissonArgs b = a;
    b.aux_lid = 0;   // the source launch wrote the aux boundary (aux is constant in a sweep)
    launch_bcs(b, st);
#else
    launch_bcs(a, st);
#endif
    // one wave of CTAs, each striding over the grid: when no value reached the ceiling (the
    // usual case) the launch costs one short wave
    const long long quads = (long long)d.im * d.plane / 4;
    const long long blocks = std::min<long long>((quads + 255) / 256, 148LL * 4);
    launch_dependent(poisson_ceiling_kernel, dim3((unsigned)blocks), dim3(256), 0, st, a);
}

// the boundary conditions of a sweep alone (radial, pole, seam), PressureSolverAtm.h:504-552
void launch_poisson_bcs(const PoissonArgs& a, cudaStream_t st)
{
    launch_bcs(a, st);
}

// gradient correction of project_initial_velocity, PressureSolverAtm.h:728-749
__global__ void __launch_bounds__(256) project_correct_kernel(PoissonArgs a, double* u, double* v, double* w)
{
    const Dims& d = a.d;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k < 1 || k >= d.km - 1 || j < 1 || j >= d.jm - 1 || i < 1 || i >= d.im - 1) return;
    const long long c = idx3(d, i, j, k);
    const PoiIJ P = a.poi[i * d.jm + j];
    const long long sI = d.plane, sJ = d.pitch;
    const double* p = a.p;
    const double dpdr = (p[c + sI] - p[c - sI]) * a.inv_2dr;
    const double dpdthe = (p[c + sJ] - p[c - sJ]) * a.inv_2dthe;
    const double dpdphi = (p[c + 1] - p[c - 1]) * a.inv_2dphi;
    u[c] -= dpdr * P.exp_rm;
    v[c] -= dpdthe * P.inv_rm;
    w[c] -= dpdphi * P.inv_rmsinthe;
}

void launch_project_correct(const PoissonArgs& a, double* u, double* v, double* w, cudaStream_t st)
{
    const Dims& d = a.d;
    const dim3 block(32, 8), grid((d.km + 31) / 32, (d.jm + 7) / 8, d.im);
    project_correct_kernel<<<grid, block, 0, st>>>(a, u, v, w);
}

// ---------------------------------------------------------------------------------------
__global__ void fill_kernel(Dims d, double* dst, double v)
{
    const long long n = d.fstride;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x)
        dst[q] = v;
}

void launch_fill(const Dims& d, double* dst, double v, cudaStream_t st)
{
    fill_kernel<<<148 * 4, 256, 0, st>>>(d, dst, v);
}

// Packed (i,j,k) rows of km values -> pitched rows.  One warp-row of 32 threads per 32
// longitudes, 8 rows per CTA; reads and writes are both coalesced.
__global__ void __launch_bounds__(256) repitch_kernel(Dims d, const double* __restrict__ packed,
                                                      double* __restrict__ dst)
{
    const int rows = d.im * d.jm;
    for (int row = blockIdx.y * 8 + threadIdx.y; row < rows; row += gridDim.y * 8) {
        const double* s = packed + (long long)row * d.km;
        double* o = dst + (long long)row * d.pitch;
        for (int k = blockIdx.x * 32 + threadIdx.x; k < d.km; k += gridDim.x * 32) o[k] = s[k];
    }
}

void launch_repitch(const Dims& d, const double* packed, double* dst, cudaStream_t st)
{
    const int rows = d.im * d.jm;
    const int gy = (rows + 7) / 8 < 65535 ? (rows + 7) / 8 : 65535;
    repitch_kernel<<<dim3((d.km + 31) / 32, gy), dim3(32, 8), 0, st>>>(d, packed, dst);
}

}  // namespace athad
