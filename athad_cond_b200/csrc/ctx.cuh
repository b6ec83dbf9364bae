// ctx.cuh - the context object behind the opaque athad_ctx handle of include/athad_gpu.h,
// shared by the C ABI translation units (athad_gpu.cu, batch.cu).
#pragma once

#include <string>
#include <vector>

#include "kernels.cuh"

namespace athad {

struct MGSolver;                 // pressure_solve hierarchy (k_mg.cu), built on first use
void mg_free(MGSolver* s);

constexpr int kNY = 11;   // prognostic fields t..dis
constexpr int kNonfiniteSlot = 24;   // counters word of the level mean's non-finite count

struct Layout {
    Dims d;
    size_t field_elems;   // im*jm*pitch
    size_t f2d_elems;     // jm*pitch
    size_t n_fields;      // ATHAD_NFIELDS + internal 3-D buffers
    size_t bytes;
};

// stage A, stage B, accumulator K, Poisson source, upload staging (packed rows)
constexpr int kInternal3D = 3 * kNY + 2;

inline size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// FP32 buffers of the mixed-precision RK4 step: stage A, stage B, accumulator K, level n
// (11 each) and the packed forcing
constexpr int kMixed32 = 4 * kNY + ATHAD_MF_COUNT;

inline Layout make_layout(const athad_grid& g, int precision)
{
    Layout L;
    L.d.im = g.im; L.d.jm = g.jm; L.d.km = g.km;
    L.d.pitch = (int)round_up((size_t)g.km, 32);
    L.d.plane = (long long)g.jm * L.d.pitch;
    L.field_elems = round_up((size_t)g.im * L.d.plane, 64);
    L.d.fstride = (long long)L.field_elems;
    L.f2d_elems = round_up((size_t)g.jm * L.d.pitch, 64);
    L.n_fields = ATHAD_NFIELDS + kInternal3D;
    size_t b = L.n_fields * L.field_elems * sizeof(double);
    b += ATHAD_NFIELDS2D * L.f2d_elems * sizeof(double);
    b += ATHAD_NPROFILES * round_up((size_t)g.im, 64) * sizeof(double);
    b += round_up((size_t)g.im * g.jm * sizeof(GeoIJ), 256);
    b += round_up((size_t)g.im * g.jm * sizeof(PoiIJ), 256);
    b += 8 * round_up((size_t)(g.im > g.jm ? g.im : g.jm), 64) * sizeof(double);  // sin_w, height, step, coslat, step_mc, cose, res_sin, rad
    b += round_up((size_t)g.jm * sizeof(int), 256);                                   // tropopause levels
    b += 2 * round_up((size_t)g.im * g.jm, 64) * sizeof(double);                    // row sums
    b += 256;                                                                         // counters
    b += round_up((size_t)g.jm * sizeof(int), 256);                                   // polar passes
    b += round_up((size_t)g.im * sizeof(TurbLevel), 256);                             // turbulence levels
    if (precision == ATHAD_PRECISION_MIXED) {
        b += (size_t)kMixed32 * round_up(L.field_elems * sizeof(float), 256);
        b += round_up((size_t)g.im * g.jm * sizeof(GeoF), 256);
    }
    L.bytes = b;
    return L;
}


}  // namespace athad

using namespace athad;

struct athad_ctx {
    athad_grid grid{};
    athad_params p{};
    Layout L{};
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    char* slab = nullptr;
    double* field[ATHAD_NFIELDS] = {};
    double* stA[kNY] = {};
    double* stB[kNY] = {};
    double* stK[kNY] = {};
    double* src = nullptr;
    double* upload_stage = nullptr;   // im*jm*km packed doubles
    float* mA[kNY] = {};              // mixed precision: FP32 stage buffers, accumulator,
    float* mB[kNY] = {};              // level n and packed forcing; FP32 geometry
    float* mK[kNY] = {};
    float* mYn[kNY] = {};
    float* mF[ATHAD_MF_COUNT] = {};
    GeoF* geof = nullptr;
    double* f2d[ATHAD_NFIELDS2D] = {};
    double* prof[ATHAD_NPROFILES] = {};
    GeoIJ* geo = nullptr;
    PoiIJ* poi = nullptr;
    double* sin_w = nullptr;
    double* height = nullptr;
    double* step_f = nullptr;
    double* coslat = nullptr;
    double* step_mc = nullptr;
    double* cose = nullptr;
    double* row_sum = nullptr;
    double* row_cnt = nullptr;
    unsigned long long* counters = nullptr;   // 32 words: [0..1] poisson, [2] satadj ceiling,
                                              // [3], [8..9] vapour ceiling, [12..15] min/max,
                                              // [16..21] residuum, [kNonfiniteSlot] level mean
    int* polar_passes = nullptr;              // [jm] zonal filter passes per row
    TurbLevel* turb_lev = nullptr;            // [im] TurbulenceAtm per-level constants
    double* res_sin = nullptr;                // [jm] findResiduumAtm's max(0.55, sin theta_j)
    double* rad_d = nullptr;                  // [im] rad.z
    int* i_trop = nullptr;                    // [jm] tropopause level per row (standAtm)
    bool trop_set = false;
    bool level_mean_valid = false;            // t_ref_level computed (or uploaded) since creation
                                              // or the last initial state
    double residuum_old = 1.0e-5;             // cAtmosphereModel.h:164
    // the budgets' first-call references (cAtmosphereModel.h:89-109; <= 0 / empty = unset)
    double q_co2_ref = -1.0, q_h2o_ref = -1.0, q_h2o_fixed_ref = -1.0;
    std::vector<double> air_levels, h2o_levels;
    // asynchronous checkpoints (athad_checkpoint_begin): a device snapshot of the fields,
    // copied to the host on a side stream while the compute stream goes on
    double* ckpt_buf = nullptr;
    int ckpt_cap = 0;                         // fields the snapshot holds
    cudaStream_t ckpt_stream = nullptr;
    cudaEvent_t ckpt_ready = nullptr, ckpt_done = nullptr;
    double dr = 0, dthe = 0, dphi = 0, shell_len = 0, metric_r0 = 0;
    double layer_height1 = 0;   // get_layer_height(1): the first layer's height, float-rounded
    std::vector<double> rad;
    std::vector<double> height_h;             // [im] get_layer_height(i), float values (host copy)
    int64_t poisson_sweeps_since_reset = 0;
    MGSolver* mg = nullptr;
    cudaEvent_t ev_step0 = nullptr, ev_step1 = nullptr;   // around the last athad_rk4_step
    bool step_timed = false;
    std::string err;
};

inline athad_status fail(athad_ctx* c, athad_status s, const char* msg)
{
    if (c) c->err = msg;
    return s;
}

inline athad_status cuda_check(athad_ctx* c, cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return ATHAD_OK;
    if (c) c->err = std::string(what) + ": " + cudaGetErrorString(e);
    return (e == cudaErrorMemoryAllocation) ? ATHAD_ERR_OOM : ATHAD_ERR_CUDA;
}

#define ATHAD_CHECK_LAUNCH(ctx, what)                                         \
    do {                                                                      \
        athad_status _s = cuda_check((ctx), cudaGetLastError(), (what));      \
        if (_s != ATHAD_OK) return _s;                                        \
    } while (0)

namespace athad {
void mixed_args(athad_ctx* ctx, const athad_step_scalars* s, RK4MArgs& a);
// the boundary conditions of athad_boundary_conditions, with (wall_bc = 1) or without the
// turbulence wall values
athad_status boundary_conditions(athad_ctx* ctx, int wall_bc);
// ThermoAtm::forces' Coriolis and buoyancy arrays (k_init.cu); t_ref null: reference 1
void launch_forces(athad_ctx* ctx, const double* t_ref);
}
