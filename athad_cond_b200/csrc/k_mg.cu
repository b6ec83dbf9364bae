// k_mg.cu - the pressure-Poisson equation of PressureSolverAtm solved to a tolerance
// (athad_pressure_solve): the fixed point that the reference's red-black sweeps
// (PressureSolverAtm.h:225-552) relax towards, reached in a few dozen iterations instead
// of the tens of thousands of sweeps a relaxative solve of 15.9 M points would need.
//
// The system.  Unknowns are the interior cells; the boundary cells are eliminated with the
// reference's boundary conditions (radial and pole copies, the seam average of the two
// seam-adjacent meridians), so at the fixed point A p = -src with
//   (A p)_c = denom p_c - num1 (p_i+1 + p_i-1) - num2 (p_j+1 + p_j-1) - num3 (p_k+1 + p_k-1)
// and the eliminated neighbours folded into the diagonal / the seam coupling.  With the
// metric fix (and without the anelastic term) num1 depends only on the level i and num2 on
// i, so S = W A with W = diag(1 / num1(i)) is symmetric: the i-couplings become -1.  S is
// singular (constants) and positive semi-definite; the right-hand side is projected onto
// its range (mean removed) and the solution returned with zero mean.
//
// The solver.  Conjugate gradients on S in FP64 (residuals, dot products and the solution
// update; the true residual rhs - S x is recomputed every few iterations, an iterative
// refinement of the recursively updated one), preconditioned by one FP32 multigrid
// V-cycle: aggregation of 2 x 2 cells in (j, k) with Galerkin coarse operators (the
// levels are not coarsened in i, where the coupling is a hundred times stronger), and a
// zebra line smoother solving each radial column exactly (Thomas algorithm, factors
// precomputed per column class).  Dot products and norms are reduced in a fixed order
// (per-block partial sums, then one block), so a solve is deterministic.
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.cuh"

namespace athad {

namespace {

constexpr int kMaxLevels = 16;
#ifndef ATHAD_MG_NU
#define ATHAD_MG_NU 2            // symmetric zebra sweeps before and after the coarse correction
#endif
#ifndef ATHAD_MG_COARSE_SWEEPS
#define ATHAD_MG_COARSE_SWEEPS 4 // symmetric sweeps on the coarsest level
#endif
#ifndef ATHAD_MG_CSCALE
#define ATHAD_MG_CSCALE 1.7f     // scale of the prolongated coarse correction (61x361x721:
                                 // 1.0 -> 86 CG iterations, 1.7 -> 44; with NU 2, 27)
#endif

template <typename T>
struct OpView {
    int ni, nj, nk, pitch;
    long long plane;
    const T* diag;   // [ni][nj][3]   column class kc: 0 first k, 1 interior, 2 last k
    const T* ci;     // [ni][nj][3]   coupling i <-> i+1
    const T* cj;     // [ni][nj][3]   coupling j <-> j+1
    const T* ck;     // [ni][nj]      coupling k <-> k+1
    const T* cs;     // [ni][nj]      seam coupling k = 0 <-> k = nk-1
};

__device__ __forceinline__ int kclass(int k, int nk) { return (k == 0) ? 0 : (k == nk - 1) ? 2 : 1; }

// off-diagonal part of row (i, j, k) of the operator applied to x
template <typename T>
__device__ __forceinline__ T offdiag(const OpView<T>& o, const T* __restrict__ x, int i, int j, int k, long long c)
{
    const int kc = kclass(k, o.nk);
    const int ij = i * o.nj + j;
    T s = 0;
    if (i > 0) s += o.ci[(ij - o.nj) * 3 + kc] * x[c - o.plane];
    if (i < o.ni - 1) s += o.ci[ij * 3 + kc] * x[c + o.plane];
    if (j > 0) s += o.cj[(ij - 1) * 3 + kc] * x[c - o.pitch];
    if (j < o.nj - 1) s += o.cj[ij * 3 + kc] * x[c + o.pitch];
    const T ckv = o.ck[ij];
    if (k > 0) s += ckv * x[c - 1];
    if (k < o.nk - 1) s += ckv * x[c + 1];
    if (k == 0) s += o.cs[ij] * x[c + (o.nk - 1)];
    else if (k == o.nk - 1) s += o.cs[ij] * x[c - (o.nk - 1)];
    return s;
}

// r = f - S e (FP32, one level)
__global__ void __launch_bounds__(128) mg_residual_kernel(OpView<float> o, const float* __restrict__ e,
                                                          const float* __restrict__ f, float* __restrict__ r)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= o.nk) return;
    const long long c = i * o.plane + (long long)j * o.pitch + k;
    const float d = o.diag[(i * o.nj + j) * 3 + kclass(k, o.nk)];
    r[c] = f[c] - (d * e[c] + offdiag(o, e, i, j, k, c));
}

// q = S x in FP64, with per-block partial sums of x.q
__global__ void __launch_bounds__(128) mg_apply64_kernel(OpView<double> o, const double* __restrict__ x,
                                                         double* __restrict__ q, double* __restrict__ partial)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    double v = 0.0;
    if (k < o.nk) {
        const long long c = i * o.plane + (long long)j * o.pitch + k;
        const double d = o.diag[(i * o.nj + j) * 3 + kclass(k, o.nk)];
        const double s = d * x[c] + offdiag(o, x, i, j, k, c);
        q[c] = s;
        v = x[c] * s;
    }
    __shared__ double red[4];
    for (int off = 16; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0)
        partial[((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = (red[0] + red[1]) + (red[2] + red[3]);
}

// r = rhs - S x in FP64 (the true residual), partial sums of (r num1(i))^2, the squared
// norm of the A-form residual
__global__ void __launch_bounds__(128) mg_true_residual_kernel(OpView<double> o, const double* __restrict__ x,
                                                               const double* __restrict__ rhs, double* __restrict__ r,
                                                               const double* __restrict__ inv_w,
                                                               double* __restrict__ partial)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    double v = 0.0;
    if (k < o.nk) {
        const long long c = i * o.plane + (long long)j * o.pitch + k;
        const double d = o.diag[(i * o.nj + j) * 3 + kclass(k, o.nk)];
        const double s = rhs[c] - (d * x[c] + offdiag(o, x, i, j, k, c));
        r[c] = s;
        const double a = s * inv_w[i];
        v = a * a;
    }
    __shared__ double red[4];
    for (int off = 16; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0)
        partial[((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = (red[0] + red[1]) + (red[2] + red[3]);
}

// per-block partial sums of a.b; of (a num1(i))^2 when b is null (the squared norm of the
// corresponding A-form vector); of a when both b and inv_w are null
__global__ void __launch_bounds__(128) mg_dot_kernel(int nk, int nj, int pitch, long long plane,
                                                     const double* __restrict__ a, const double* __restrict__ b,
                                                     const double* __restrict__ inv_w, double* __restrict__ partial)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    double v = 0.0;
    if (k < nk) {
        const long long c = i * plane + (long long)j * pitch + k;
        if (b) v = a[c] * b[c];
        else if (inv_w) { const double s = a[c] * inv_w[i]; v = s * s; }
        else v = a[c];
    }
    __shared__ double red[4];
    for (int off = 16; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0)
        partial[((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = (red[0] + red[1]) + (red[2] + red[3]);
}

// fixed-order sum of n partials into out[slot] (one block of 1024 threads)
__global__ void __launch_bounds__(1024) mg_sum_kernel(const double* __restrict__ partial, long long n,
                                                      double* __restrict__ out, int slot)
{
    double v = 0.0;
    for (long long q = threadIdx.x; q < n; q += blockDim.x) v += partial[q];
    __shared__ double red[32];
    for (int off = 16; off >= 1; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = red[threadIdx.x];
        for (int off = 16; off >= 1; off >>= 1) w += __shfl_xor_sync(0xffffffffu, w, off);
        if (threadIdx.x == 0) out[slot] = w;
    }
}

// y += a x  (a read from device memory: a = s[num] / s[den] * sign)
__global__ void mg_axpy_kernel(long long n, const double* __restrict__ s, int num, int den, double sign,
                               const double* __restrict__ x, double* __restrict__ y)
{
    const double a = sign * s[num] / s[den];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        y[q] += a * x[q];
}

// d = z + (s[num] / s[den]) d
__global__ void mg_xpby_kernel(long long n, const double* __restrict__ s, int num, int den,
                               const double* __restrict__ z, double* __restrict__ d)
{
    const double b = s[num] / s[den];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        d[q] = z[q] + b * d[q];
}

__global__ void mg_copy_scalar_kernel(double* s, int dst, int src) { s[dst] = s[src]; }

__global__ void mg_to_f32_kernel(long long n, const double* __restrict__ a, float* __restrict__ b)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        b[q] = (float)a[q];
}

__global__ void mg_to_f64_kernel(long long n, const float* __restrict__ a, double* __restrict__ b)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        b[q] = (double)a[q];
}

// subtract s[slot] / count from every unknown (padding untouched)
__global__ void __launch_bounds__(128) mg_sub_mean_kernel(int nk, int pitch, long long plane, double* __restrict__ a,
                                                          const double* __restrict__ s, int slot, double count)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nk) return;
    const long long c = blockIdx.z * plane + (long long)blockIdx.y * pitch + k;
    a[c] -= s[slot] / count;
}

// zebra line relaxation of the columns of one colour ((j + k) & 1 == colour): each radial
// column solved exactly with the horizontal neighbours fixed.  The seam neighbour of the
// columns k = 0 and k = nk-1 is read from `seam` (the two seam planes before the
// half-sweep), because with an odd nk both ends have the same colour.
//
// A CTA takes 32 columns of one row j with four warps: warp q forms the right-hand sides
// (the horizontal neighbours fixed) of levels q, q+4, ... of all 32 columns and stages them
// in shared memory with the elimination factors, so the independent loads of a column run
// four ways in parallel; then warp 0 runs the two sequential recurrences of its 32 columns
// out of shared memory.  Element (i, column t) of an array is at [i * 32 + t].
__device__ __forceinline__ float smooth_rhs(const OpView<float>& o, const float* __restrict__ f,
                                            const float* __restrict__ e, const float* __restrict__ seam,
                                            int i, int j, int k, int kc, long long c)
{
    const int ij = i * o.nj + j;
    float s = f[c];
    if (j > 0) s -= o.cj[(ij - 1) * 3 + kc] * e[c - o.pitch];
    if (j < o.nj - 1) s -= o.cj[ij * 3 + kc] * e[c + o.pitch];
    const float ckv = o.ck[ij];
    if (k > 0) s -= ckv * e[c - 1];
    if (k < o.nk - 1) s -= ckv * e[c + 1];
    if (k == 0) s -= o.cs[ij] * seam[(long long)(o.ni * o.nj) + ij];        // plane k = nk-1
    else if (k == o.nk - 1) s -= o.cs[ij] * seam[ij];                       // plane k = 0
    return s;
}

__global__ void __launch_bounds__(128) mg_smooth_split_kernel(OpView<float> o, const float* __restrict__ tm,
                                                              const float* __restrict__ tc, const float* __restrict__ f,
                                                              float* __restrict__ e, const float* __restrict__ seam,
                                                              int colour)
{
    extern __shared__ float sm[];   // rhs, forward factor m_i, coupling c_{i-1}, backward factor: [4][ni][32]
    const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
    const int j = blockIdx.y;
    const int k = 2 * (blockIdx.x * 32 + lane) + ((colour + j) & 1);
    const bool valid = k < o.nk;
    const int ni = o.ni;
    float* rhs = sm;
    float* fm = sm + ni * 32;
    float* fc = sm + 2 * ni * 32;
    float* bc = sm + 3 * ni * 32;
    const int kc = valid ? kclass(k, o.nk) : 1;
    const long long c0 = (long long)j * o.pitch + k;
    if (valid) {
#pragma unroll 2
        for (int i = q; i < ni; i += 4) {
            const int ij = i * o.nj + j;
            rhs[i * 32 + lane] = smooth_rhs(o, f, e, seam, i, j, k, kc, i * o.plane + c0);
            fm[i * 32 + lane] = tm[ij * 3 + kc];
            fc[i * 32 + lane] = (i > 0) ? o.ci[(ij - o.nj) * 3 + kc] : 0.0f;
            bc[i * 32 + lane] = tc[ij * 3 + kc];
        }
    }
    __syncthreads();
    if (q != 0 || !valid) return;
    // forward elimination: y_i = (rhs_i - c_{i-1} y_{i-1}) m_i
    float y = 0.0f;
    for (int i = 0; i < ni; i++) {
        float s = rhs[i * 32 + lane];
        if (i > 0) s -= fc[i * 32 + lane] * y;
        y = s * fm[i * 32 + lane];
        rhs[i * 32 + lane] = y;
    }
    // back substitution: x_i = y_i - c'_i x_{i+1}
    float x = y;
    e[(ni - 1) * o.plane + c0] = x;
    for (int i = ni - 2; i >= 0; i--) {
        x = rhs[i * 32 + lane] - bc[i * 32 + lane] * x;
        e[i * o.plane + c0] = x;
    }
}

// the same relaxation one thread per column with the right-hand side in the scratch field
// w, for columns too tall for the shared-memory form
__global__ void __launch_bounds__(128) mg_smooth_kernel(OpView<float> o, const float* __restrict__ tm,
                                                        const float* __restrict__ tc, const float* __restrict__ f,
                                                        float* __restrict__ e, const float* __restrict__ seam,
                                                        float* __restrict__ w, int colour)
{
    const int j = blockIdx.y;
    const int k = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((colour + j) & 1);
    if (k >= o.nk) return;
    const int kc = kclass(k, o.nk);
    const long long c0 = (long long)j * o.pitch + k;
#pragma unroll 4
    for (int i = 0; i < o.ni; i++) w[i * o.plane + c0] = smooth_rhs(o, f, e, seam, i, j, k, kc, i * o.plane + c0);
    float y_prev = 0.0f;
    for (int i = 0; i < o.ni; i++) {
        const long long c = i * o.plane + c0;
        const int ij = i * o.nj + j;
        float s = w[c];
        if (i > 0) s -= o.ci[(ij - o.nj) * 3 + kc] * y_prev;
        y_prev = s * tm[ij * 3 + kc];
        e[c] = y_prev;
    }
    float x_next = y_prev;
    for (int i = o.ni - 2; i >= 0; i--) {
        const long long c = i * o.plane + c0;
        x_next = e[c] - tc[(i * o.nj + j) * 3 + kc] * x_next;
        e[c] = x_next;
    }
}

// the two seam planes (k = 0, k = nk-1) of e into seam[2][ni][nj]
__global__ void mg_seam_copy_kernel(int ni, int nj, int nk, int pitch, long long plane, const float* __restrict__ e,
                                    float* __restrict__ seam)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= ni * nj) return;
    const int i = q / nj, j = q % nj;
    const long long c = i * plane + (long long)j * pitch;
    seam[q] = e[c];
    seam[(long long)ni * nj + q] = e[c + nk - 1];
}

// coarse f = sum of the fine residuals of the 2 x 2 (j, k) aggregate
__global__ void __launch_bounds__(128) mg_restrict_kernel(int nk_f, int nj_f, int pitch_f, long long plane_f,
                                                          const float* __restrict__ r, int nk_c, int pitch_c,
                                                          long long plane_c, float* __restrict__ fc)
{
    const int K = blockIdx.x * blockDim.x + threadIdx.x;
    const int J = blockIdx.y, i = blockIdx.z;
    if (K >= nk_c) return;
    const int j0 = 2 * J, k0 = 2 * K;
    const long long b = i * plane_f;
    float s = r[b + (long long)j0 * pitch_f + k0];
    if (k0 + 1 < nk_f) s += r[b + (long long)j0 * pitch_f + k0 + 1];
    if (j0 + 1 < nj_f) {
        s += r[b + (long long)(j0 + 1) * pitch_f + k0];
        if (k0 + 1 < nk_f) s += r[b + (long long)(j0 + 1) * pitch_f + k0 + 1];
    }
    fc[i * plane_c + (long long)J * pitch_c + K] = s;
}

// fine e += scale * coarse e of the aggregate.  A piecewise-constant prolongation
// under-corrects smooth errors; a constant scale keeps the V-cycle symmetric.
__global__ void __launch_bounds__(128) mg_prolong_kernel(int nk_f, int pitch_f, long long plane_f, float* __restrict__ e,
                                                         int pitch_c, long long plane_c, const float* __restrict__ ec)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= nk_f) return;
    e[i * plane_f + (long long)j * pitch_f + k] += ATHAD_MG_CSCALE * ec[i * plane_c + (long long)(j >> 1) * pitch_c + (k >> 1)];
}

// right-hand side of S: rhs_c = -src_c / num1(i) at every interior cell
__global__ void __launch_bounds__(128) mg_rhs_kernel(Dims d, const double* __restrict__ src, int nk, int pitch,
                                                     long long plane, const double* __restrict__ inv_w,
                                                     double* __restrict__ rhs)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= nk) return;
    const double s = src[idx3(d, i + 1, j + 1, k + 1)];
    rhs[i * plane + (long long)j * pitch + k] = -s / inv_w[i];
}

// interior unknowns into p_dyn
__global__ void __launch_bounds__(128) mg_store_kernel(Dims d, const double* __restrict__ x, int nk, int pitch,
                                                       long long plane, double* __restrict__ p)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, i = blockIdx.z;
    if (k >= nk) return;
    p[idx3(d, i + 1, j + 1, k + 1)] = x[i * plane + (long long)j * pitch + k];
}

}  // namespace

// ---- host side ---------------------------------------------------------------------------

struct MGLevel {
    int ni = 0, nj = 0, nk = 0, pitch = 0;
    long long plane = 0, n = 0;
    float* e = nullptr; float* f = nullptr; float* r = nullptr;
    float* coef = nullptr;      // diag, ci, cj (3 per (i,j)), ck, cs (1 per (i,j)), tm, tc (3 per (i,j))
    OpView<float> op{};
    float* tm = nullptr; float* tc = nullptr;
};

struct MGSolver {
    int nlev = 0;
    MGLevel L[kMaxLevels];
    OpView<double> op64{};
    double* coef64 = nullptr;
    double* inv_w = nullptr;                       // num1(i) per interior level
    double *x = nullptr, *r = nullptr, *z = nullptr, *d = nullptr, *q = nullptr, *rhs = nullptr;
    double* partial = nullptr;
    double* scal = nullptr;                        // device scalars
    float* seam = nullptr;
    long long nblocks = 0;
    char* mem = nullptr;
    size_t bytes = 0;
    cudaGraphExec_t iter_graph[2] = {nullptr, nullptr};   // one CG iteration (plain, refined)
    double* h = nullptr;                                  // pinned copy of the device scalars
};

void mg_free(MGSolver* s)
{
    if (!s) return;
    for (int g = 0; g < 2; g++)
        if (s->iter_graph[g]) cudaGraphExecDestroy(s->iter_graph[g]);
    if (s->h) cudaFreeHost(s->h);
    cudaFree(s->mem);
    delete s;
}

namespace {

inline long long rup(long long v, long long a) { return (v + a - 1) / a * a; }

// Galerkin coarsening of a level's coefficients (host, FP64): 2 x 2 aggregates in (j, k)
void coarsen(int ni, int nj, int nk, const std::vector<double>& D, const std::vector<double>& CI,
             const std::vector<double>& CJ, const std::vector<double>& CK, const std::vector<double>& CS,
             std::vector<double>& Dc, std::vector<double>& CIc, std::vector<double>& CJc,
             std::vector<double>& CKc, std::vector<double>& CSc)
{
    const int nJ = (nj + 1) / 2, nK = (nk + 1) / 2;
    auto kcf = [&](int k) { return (k == 0) ? 0 : (k == nk - 1) ? 2 : 1; };
    Dc.assign((size_t)ni * nJ * 3, 0.0); CIc.assign(Dc.size(), 0.0); CJc.assign(Dc.size(), 0.0);
    CKc.assign((size_t)ni * nJ, 0.0); CSc.assign(CKc.size(), 0.0);
    for (int i = 0; i < ni; i++)
        for (int J = 0; J < nJ; J++) {
            const int j0 = 2 * J, j1 = (2 * J + 1 < nj) ? 2 * J + 1 : -1;
            for (int kcC = 0; kcC < 3; kcC++) {
                const int K = (kcC == 0) ? 0 : (kcC == 2) ? nK - 1 : 1;
                const int k0 = 2 * K, k1 = (2 * K + 1 < nk) ? 2 * K + 1 : -1;
                const int ks[2] = {k0, k1}, js[2] = {j0, j1};
                double dg = 0.0, ci = 0.0, cj = 0.0;
                for (int a = 0; a < 2; a++) {
                    if (js[a] < 0) continue;
                    for (int b = 0; b < 2; b++) {
                        if (ks[b] < 0) continue;
                        const size_t f3 = ((size_t)i * nj + js[a]) * 3 + kcf(ks[b]);
                        dg += D[f3];
                        ci += CI[f3];
                    }
                }
                if (j1 >= 0)                                   // internal j couplings
                    for (int b = 0; b < 2; b++)
                        if (ks[b] >= 0) dg += 2.0 * CJ[((size_t)i * nj + j0) * 3 + kcf(ks[b])];
                if (k1 >= 0)                                   // internal k couplings
                    for (int a = 0; a < 2; a++)
                        if (js[a] >= 0) dg += 2.0 * CK[(size_t)i * nj + js[a]];
                const int jl = (j1 >= 0) ? j1 : j0;            // coupling J <-> J+1 crosses jl <-> jl+1
                if (J + 1 < nJ)
                    for (int b = 0; b < 2; b++)
                        if (ks[b] >= 0) cj += CJ[((size_t)i * nj + jl) * 3 + kcf(ks[b])];
                const size_t c3 = ((size_t)i * nJ + J) * 3 + kcC;
                Dc[c3] = dg; CIc[c3] = ci; CJc[c3] = cj;
            }
            double ck = 0.0, cs = 0.0;
            for (int a = 0; a < 2; a++) {
                const int jj = (a == 0) ? j0 : j1;
                if (jj < 0) continue;
                ck += CK[(size_t)i * nj + jj];
                cs += CS[(size_t)i * nj + jj];
            }
            CKc[(size_t)i * nJ + J] = ck;
            CSc[(size_t)i * nJ + J] = cs;
        }
}

void thomas_factors(int ni, int nj, const std::vector<double>& D, const std::vector<double>& CI,
                    std::vector<double>& TM, std::vector<double>& TC)
{
    TM.assign(D.size(), 0.0);
    TC.assign(D.size(), 0.0);
    for (int j = 0; j < nj; j++)
        for (int kc = 0; kc < 3; kc++) {
            double cprev = 0.0;
            for (int i = 0; i < ni; i++) {
                const size_t q = ((size_t)i * nj + j) * 3 + kc;
                const double a = (i > 0) ? CI[((size_t)(i - 1) * nj + j) * 3 + kc] : 0.0;
                const double m = 1.0 / (D[q] - a * cprev);
                TM[q] = m;
                cprev = CI[q] * m;
                TC[q] = cprev;
            }
        }
}

}  // namespace

// Build the hierarchy for a context (one allocation).  Returns nullptr on failure.
MGSolver* mg_build(athad_ctx* ctx, std::string& err)
{
    const Dims& d = ctx->L.d;
    const int ni = d.im - 2, nj = d.jm - 2, nk = d.km - 2;
    if (ni < 2 || nj < 2 || nk < 3) { err = "pressure_solve: grid too small"; return nullptr; }
    // per-(i,j) coefficients of the full grid
    std::vector<PoiIJ> poi((size_t)d.im * d.jm);
    if (cudaMemcpy(poi.data(), ctx->poi, poi.size() * sizeof(PoiIJ), cudaMemcpyDeviceToHost) != cudaSuccess) {
        cudaGetLastError(); err = "pressure_solve: reading the operator"; return nullptr;
    }
    // level 0 (FP64): S = W A, W = diag(1/num1(i))
    std::vector<double> D((size_t)ni * nj * 3), CI(D.size()), CJ(D.size()), CK((size_t)ni * nj), CS(CK.size());
    std::vector<double> inv_w(ni);
    for (int i = 0; i < ni; i++) {
        inv_w[i] = poi[(size_t)(i + 1) * d.jm + 1].num1;
        for (int j = 0; j < nj; j++) {
            const PoiIJ& P = poi[(size_t)(i + 1) * d.jm + (j + 1)];
            const double w = 1.0 / P.num1;
            for (int kc = 0; kc < 3; kc++) {
                double dg = w * P.denom;
                if (i == 0) dg -= 1.0;                   // p[i=0] = p[1]
                if (i == ni - 1) dg -= 1.0;              // lid copy
                if (j == 0) dg -= w * P.num2;            // pole copies
                if (j == nj - 1) dg -= w * P.num2;
                if (kc != 1) dg -= 0.5 * w * P.num3;     // seam average: half of the seam neighbour is this cell
                const size_t q = ((size_t)i * nj + j) * 3 + kc;
                D[q] = dg;
                CI[q] = (i < ni - 1) ? -1.0 : 0.0;
                CJ[q] = (j < nj - 1) ? -w * P.num2 : 0.0;
            }
            CK[(size_t)i * nj + j] = -w * P.num3;
            CS[(size_t)i * nj + j] = -0.5 * w * P.num3;
        }
    }
    // levels
    struct HostLevel { int ni, nj, nk; std::vector<double> D, CI, CJ, CK, CS, TM, TC; };
    std::vector<HostLevel> H;
    H.push_back({ni, nj, nk, D, CI, CJ, CK, CS, {}, {}});
    while ((int)H.size() < kMaxLevels) {
        const HostLevel& f = H.back();
        if (f.nj < 8 || f.nk < 16) break;
        HostLevel c;
        c.ni = f.ni; c.nj = (f.nj + 1) / 2; c.nk = (f.nk + 1) / 2;
        coarsen(f.ni, f.nj, f.nk, f.D, f.CI, f.CJ, f.CK, f.CS, c.D, c.CI, c.CJ, c.CK, c.CS);
        H.push_back(std::move(c));
    }
    for (auto& h : H) thomas_factors(h.ni, h.nj, h.D, h.CI, h.TM, h.TC);

    MGSolver* s = new MGSolver();
    s->nlev = (int)H.size();
    // sizes
    size_t bytes = 0;
    auto add = [&](size_t b) { size_t off = bytes; bytes += (size_t)rup((long long)b, 256); return off; };
    std::vector<size_t> off_e(s->nlev), off_f(s->nlev), off_r(s->nlev), off_c(s->nlev);
    for (int l = 0; l < s->nlev; l++) {
        MGLevel& L = s->L[l];
        L.ni = H[l].ni; L.nj = H[l].nj; L.nk = H[l].nk;
        L.pitch = (int)rup(L.nk, 32);
        L.plane = (long long)L.nj * L.pitch;
        L.n = (long long)L.ni * L.plane;
        off_e[l] = add(L.n * sizeof(float));
        off_f[l] = add(L.n * sizeof(float));
        off_r[l] = add(L.n * sizeof(float));
        off_c[l] = add((size_t)L.ni * L.nj * (3 * 5 + 2) * sizeof(float));
    }
    const MGLevel& L0 = s->L[0];
    const size_t off_c64 = add((size_t)ni * nj * (3 * 3 + 2) * sizeof(double));
    const size_t off_w = add(ni * sizeof(double));
    size_t off_v[6];
    for (int v = 0; v < 6; v++) off_v[v] = add(L0.n * sizeof(double));
    s->nblocks = (long long)((L0.nk + 127) / 128) * L0.nj * L0.ni;
    const size_t off_p = add(s->nblocks * sizeof(double));
    const size_t off_s = add(64 * sizeof(double));
    const size_t off_seam = add((size_t)2 * ni * nj * sizeof(float));
    if (cudaMalloc((void**)&s->mem, bytes) != cudaSuccess) {
        cudaGetLastError(); delete s; err = "pressure_solve: out of device memory"; return nullptr;
    }
    s->bytes = bytes;
    bool ok = cudaMemset(s->mem, 0, bytes) == cudaSuccess;
    for (int l = 0; l < s->nlev && ok; l++) {
        MGLevel& L = s->L[l];
        L.e = (float*)(s->mem + off_e[l]);
        L.f = (float*)(s->mem + off_f[l]);
        L.r = (float*)(s->mem + off_r[l]);
        L.coef = (float*)(s->mem + off_c[l]);
        const size_t m3 = (size_t)L.ni * L.nj * 3, m1 = (size_t)L.ni * L.nj;
        std::vector<float> buf(m3 * 5 + m1 * 2);
        for (size_t q = 0; q < m3; q++) {
            buf[q] = (float)H[l].D[q]; buf[m3 + q] = (float)H[l].CI[q]; buf[2 * m3 + q] = (float)H[l].CJ[q];
            buf[3 * m3 + q] = (float)H[l].TM[q]; buf[4 * m3 + q] = (float)H[l].TC[q];
        }
        for (size_t q = 0; q < m1; q++) { buf[5 * m3 + q] = (float)H[l].CK[q]; buf[5 * m3 + m1 + q] = (float)H[l].CS[q]; }
        ok = cudaMemcpy(L.coef, buf.data(), buf.size() * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess;
        L.op = {L.ni, L.nj, L.nk, L.pitch, L.plane, L.coef, L.coef + m3, L.coef + 2 * m3, L.coef + 5 * m3,
                L.coef + 5 * m3 + m1};
        L.tm = L.coef + 3 * m3;
        L.tc = L.coef + 4 * m3;
    }
    if (ok) {
        s->coef64 = (double*)(s->mem + off_c64);
        const size_t m3 = (size_t)ni * nj * 3, m1 = (size_t)ni * nj;
        std::vector<double> buf(m3 * 3 + m1 * 2);
        for (size_t q = 0; q < m3; q++) { buf[q] = D[q]; buf[m3 + q] = CI[q]; buf[2 * m3 + q] = CJ[q]; }
        for (size_t q = 0; q < m1; q++) { buf[3 * m3 + q] = CK[q]; buf[3 * m3 + m1 + q] = CS[q]; }
        ok = cudaMemcpy(s->coef64, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess;
        s->op64 = {ni, nj, nk, L0.pitch, L0.plane, s->coef64, s->coef64 + m3, s->coef64 + 2 * m3,
                   s->coef64 + 3 * m3, s->coef64 + 3 * m3 + m1};
        s->inv_w = (double*)(s->mem + off_w);
        if (ok) ok = cudaMemcpy(s->inv_w, inv_w.data(), ni * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess;
        double** vec[6] = {&s->x, &s->r, &s->z, &s->d, &s->q, &s->rhs};
        for (int v = 0; v < 6; v++) *vec[v] = (double*)(s->mem + off_v[v]);
        s->partial = (double*)(s->mem + off_p);
        s->scal = (double*)(s->mem + off_s);
        s->seam = (float*)(s->mem + off_seam);
    }
    if (ok) ok = cudaMallocHost((void**)&s->h, 8 * sizeof(double)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError(); cudaFree(s->mem); delete s; err = "pressure_solve: building the hierarchy"; return nullptr;
    }
    return s;
}

namespace {

inline dim3 cells_grid(int nk, int nj, int ni) { return dim3((nk + 127) / 128, nj, ni); }

void smooth(const MGLevel& L, float* seam, int colour, cudaStream_t st)
{
    mg_seam_copy_kernel<<<(L.ni * L.nj + 255) / 256, 256, 0, st>>>(L.ni, L.nj, L.nk, L.pitch, L.plane, L.e, seam);
    const int half = (L.nk + 1) / 2;
    const size_t smem = (size_t)4 * 32 * L.ni * sizeof(float);
    if (smem <= 48 * 1024)   // columns of up to 96 levels in shared memory
        mg_smooth_split_kernel<<<dim3((half + 31) / 32, L.nj), 128, smem, st>>>(L.op, L.tm, L.tc, L.f, L.e, seam,
                                                                              colour);
    else
        mg_smooth_kernel<<<dim3((half + 127) / 128, L.nj), 128, 0, st>>>(L.op, L.tm, L.tc, L.f, L.e, seam,
                                                                       L.r, colour);
}

// one V-cycle on level l: L[l].e ~= S_l^-1 L[l].f, starting from zero
void vcycle(MGSolver* s, int l, cudaStream_t st)
{
    MGLevel& L = s->L[l];
    cudaMemsetAsync(L.e, 0, L.n * sizeof(float), st);
    if (l == s->nlev - 1) {
        for (int it = 0; it < ATHAD_MG_COARSE_SWEEPS; it++) { smooth(L, s->seam, 0, st); smooth(L, s->seam, 1, st); }
        for (int it = 0; it < ATHAD_MG_COARSE_SWEEPS; it++) { smooth(L, s->seam, 1, st); smooth(L, s->seam, 0, st); }
        return;
    }
    for (int it = 0; it < ATHAD_MG_NU; it++) { smooth(L, s->seam, 0, st); smooth(L, s->seam, 1, st); }
    mg_residual_kernel<<<cells_grid(L.nk, L.nj, L.ni), 128, 0, st>>>(L.op, L.e, L.f, L.r);
    MGLevel& C = s->L[l + 1];
    mg_restrict_kernel<<<cells_grid(C.nk, C.nj, C.ni), 128, 0, st>>>(L.nk, L.nj, L.pitch, L.plane, L.r, C.nk,
                                                                       C.pitch, C.plane, C.f);
    vcycle(s, l + 1, st);
    mg_prolong_kernel<<<cells_grid(L.nk, L.nj, L.ni), 128, 0, st>>>(L.nk, L.pitch, L.plane, L.e, C.pitch, C.plane, C.e);
    for (int it = 0; it < ATHAD_MG_NU; it++) { smooth(L, s->seam, 1, st); smooth(L, s->seam, 0, st); }
}

// z = M^-1 r (FP32 V-cycle)
void precondition(MGSolver* s, cudaStream_t st)
{
    const MGLevel& L0 = s->L[0];
    mg_to_f32_kernel<<<148 * 8, 256, 0, st>>>(L0.n, s->r, s->L[0].f);
    vcycle(s, 0, st);
    mg_to_f64_kernel<<<148 * 8, 256, 0, st>>>(L0.n, s->L[0].e, s->z);
}

void dot(MGSolver* s, const double* a, const double* b, int slot, cudaStream_t st)
{
    const MGLevel& L0 = s->L[0];
    mg_dot_kernel<<<cells_grid(L0.nk, L0.nj, L0.ni), 128, 0, st>>>(L0.nk, L0.nj, L0.pitch, L0.plane, a, b, s->inv_w,
                                                                   s->partial);
    mg_sum_kernel<<<1, 1024, 0, st>>>(s->partial, s->nblocks, s->scal, slot);
}

// true residual r = rhs - S x with its A-form norm into scal[3]
void true_residual(MGSolver* s, cudaStream_t st)
{
    const MGLevel& L0 = s->L[0];
    mg_true_residual_kernel<<<cells_grid(L0.nk, L0.nj, L0.ni), 128, 0, st>>>(s->op64, s->x, s->rhs, s->r, s->inv_w,
                                                                             s->partial);
    mg_sum_kernel<<<1, 1024, 0, st>>>(s->partial, s->nblocks, s->scal, 3);
}

// One conjugate-gradient iteration, all scalars on the device: q = S d, alpha = rz / d.q,
// x += alpha d, r -= alpha q, the residual norm (recursive, or the true residual when
// `refine`) copied to the pinned host scalars, z = M^-1 r, beta = r.z / rz, d = z + beta d.
void enqueue_cg_iteration(MGSolver* s, bool refine, cudaStream_t st)
{
    const MGLevel& L0 = s->L[0];
    const long long n = L0.n;
    mg_apply64_kernel<<<cells_grid(L0.nk, L0.nj, L0.ni), 128, 0, st>>>(s->op64, s->d, s->q, s->partial);
    mg_sum_kernel<<<1, 1024, 0, st>>>(s->partial, s->nblocks, s->scal, 1);
    mg_axpy_kernel<<<148 * 8, 256, 0, st>>>(n, s->scal, 0, 1, 1.0, s->d, s->x);
    mg_axpy_kernel<<<148 * 8, 256, 0, st>>>(n, s->scal, 0, 1, -1.0, s->q, s->r);
    if (refine) true_residual(s, st);
    else dot(s, s->r, nullptr, 3, st);
    cudaMemcpyAsync(s->h, s->scal, 5 * sizeof(double), cudaMemcpyDeviceToHost, st);
    precondition(s, st);
    dot(s, s->r, s->z, 2, st);
    mg_xpby_kernel<<<148 * 8, 256, 0, st>>>(n, s->scal, 2, 0, s->z, s->d);
    mg_copy_scalar_kernel<<<1, 1, 0, st>>>(s->scal, 0, 2);
}

}  // namespace

}  // namespace athad

using namespace athad;

extern "C" athad_status athad_pressure_solve(athad_ctx* ctx, double rel_tol, int32_t max_iter,
                                             athad_solve_report* out)
{
    if (!ctx || !(rel_tol > 0.0) || max_iter < 1) return fail(ctx, ATHAD_ERR_INVALID, "pressure_solve: bad argument");
    if (ctx->p.anelastic) return fail(ctx, ATHAD_ERR_UNSUPPORTED, "pressure_solve: the anelastic operator is not symmetric");
    cudaStream_t st = ctx->stream;
    if (!ctx->mg) {
        // the hierarchy is built on first use (one allocation, kept by the context)
        athad_status s0 = cuda_check(ctx, cudaStreamSynchronize(st), "pressure_solve sync");
        if (s0 != ATHAD_OK) return s0;
        std::string err;
        ctx->mg = mg_build(ctx, err);
        if (!ctx->mg) return fail(ctx, ATHAD_ERR_OOM, err.c_str());
    }
    MGSolver* s = ctx->mg;
    const MGLevel& L0 = s->L[0];
    const Dims& d = ctx->L.d;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, st);
    // the sweep's source (aux boundary values, clamped divergence), rhs = -src / num1
    PoissonArgs pa;
    std::memset(&pa, 0, sizeof pa);
    pa.d = d; pa.poi = ctx->poi; pa.dlnrho = ctx->prof[ATHAD_PROF_DLNRHO_DR];
    pa.aux_u = ctx->field[ATHAD_AUX_U]; pa.aux_v = ctx->field[ATHAD_AUX_V]; pa.aux_w = ctx->field[ATHAD_AUX_W];
    pa.src = ctx->src; pa.p = ctx->field[ATHAD_P_DYN]; pa.counters = nullptr;   // clamps not counted
    pa.inv_2dr = 1.0 / (2.0 * ctx->dr); pa.inv_2dthe = 1.0 / (2.0 * ctx->dthe); pa.inv_2dphi = 1.0 / (2.0 * ctx->dphi);
    pa.anelastic = 0; pa.metric_div = ctx->p.metric_divergence;
    pa.ceiling = 0.0;
    launch_poisson_prepare(pa, st);
    const dim3 g0 = cells_grid(L0.nk, L0.nj, L0.ni);
    const double count = (double)L0.ni * L0.nj * L0.nk;
    const long long n = L0.n;
    mg_rhs_kernel<<<g0, 128, 0, st>>>(d, ctx->src, L0.nk, L0.pitch, L0.plane, s->inv_w, s->rhs);
    // project onto the range of S: remove the mean
    mg_dot_kernel<<<g0, 128, 0, st>>>(L0.nk, L0.nj, L0.pitch, L0.plane, s->rhs, nullptr, nullptr, s->partial);
    mg_sum_kernel<<<1, 1024, 0, st>>>(s->partial, s->nblocks, s->scal, 5);
    mg_sub_mean_kernel<<<g0, 128, 0, st>>>(L0.nk, L0.pitch, L0.plane, s->rhs, s->scal, 5, count);
    dot(s, s->rhs, nullptr, 4, st);                                   // ||b||^2 (A form)
    cudaMemsetAsync(s->x, 0, n * sizeof(double), st);
    cudaMemcpyAsync(s->r, s->rhs, n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    precondition(s, st);
    cudaMemcpyAsync(s->d, s->z, n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    dot(s, s->r, s->z, 0, st);                                        // rz
    ATHAD_CHECK_LAUNCH(ctx, "pressure_solve setup");
    double h[5] = {0, 0, 0, 0, 0};
    athad_status stt = cuda_check(ctx, cudaMemcpyAsync(h, s->scal, sizeof h, cudaMemcpyDeviceToHost, st), "pressure_solve norm");
    if (stt == ATHAD_OK) stt = cuda_check(ctx, cudaStreamSynchronize(st), "pressure_solve");
    if (stt != ATHAD_OK) { cudaEventDestroy(t0); cudaEventDestroy(t1); return stt; }

    athad_solve_report rep;
    std::memset(&rep, 0, sizeof rep);
    rep.precond_levels = s->nlev;
    if (!s->iter_graph[0] && h[4] > 0.0) {   // capture the two iteration variants once
        for (int g = 0; g < 2 && stt == ATHAD_OK; g++) {
            cudaGraph_t graph = nullptr;
            stt = cuda_check(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "capture");
            if (stt != ATHAD_OK) break;
            enqueue_cg_iteration(s, g == 1, st);
            stt = cuda_check(ctx, cudaStreamEndCapture(st, &graph), "end capture");
            if (stt == ATHAD_OK) stt = cuda_check(ctx, cudaGraphInstantiate(&s->iter_graph[g], graph, 0), "instantiate");
            if (graph) cudaGraphDestroy(graph);
        }
    }
    double res = (h[4] > 0.0) ? 1.0 : 0.0;
    int it = 0;
    for (it = 1; it <= max_iter && h[4] > 0.0 && stt == ATHAD_OK; it++) {
        const bool refine = (it % 8 == 0);
        stt = cuda_check(ctx, cudaGraphLaunch(s->iter_graph[refine ? 1 : 0], st), "pressure_solve iteration");
        if (stt == ATHAD_OK) stt = cuda_check(ctx, cudaStreamSynchronize(st), "pressure_solve");
        if (stt != ATHAD_OK) break;
        res = std::sqrt(s->h[3] / h[4]);
        if (it <= 64) rep.history[it - 1] = res;
        if (res <= rel_tol) {
            if (refine) break;
            // confirm with the true residual before stopping
            true_residual(s, st);
            cudaMemcpyAsync(s->h, s->scal, 5 * sizeof(double), cudaMemcpyDeviceToHost, st);
            stt = cuda_check(ctx, cudaStreamSynchronize(st), "pressure_solve");
            if (stt != ATHAD_OK) break;
            res = std::sqrt(s->h[3] / h[4]);
            if (it <= 64) rep.history[it - 1] = res;
            if (res <= rel_tol) break;
        }
    }
    if (stt != ATHAD_OK) { cudaEventDestroy(t0); cudaEventDestroy(t1); return stt; }
    // zero-mean solution into p_dyn, boundary cells by the reference's boundary conditions
    mg_dot_kernel<<<g0, 128, 0, st>>>(L0.nk, L0.nj, L0.pitch, L0.plane, s->x, nullptr, nullptr, s->partial);
    mg_sum_kernel<<<1, 1024, 0, st>>>(s->partial, s->nblocks, s->scal, 6);
    mg_sub_mean_kernel<<<g0, 128, 0, st>>>(L0.nk, L0.pitch, L0.plane, s->x, s->scal, 6, count);
    mg_store_kernel<<<g0, 128, 0, st>>>(d, s->x, L0.nk, L0.pitch, L0.plane, ctx->field[ATHAD_P_DYN]);
    launch_poisson_bcs(pa, st);
    cudaEventRecord(t1, st);
    stt = cuda_check(ctx, cudaEventSynchronize(t1), "pressure_solve");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (stt != ATHAD_OK) return stt;
    ATHAD_CHECK_LAUNCH(ctx, "pressure_solve");
    rep.iterations = (h[4] > 0.0) ? ((it > max_iter) ? max_iter : it) : 0;
    rep.converged = (res <= rel_tol) ? 1 : 0;
    rep.rel_residual = res;
    rep.seconds = ms * 1e-3;
    if (out) *out = rep;
    return ATHAD_OK;
}
