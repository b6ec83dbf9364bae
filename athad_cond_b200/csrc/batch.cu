// batch.cu - ensembles of contexts advanced together (athad_batch_* of include/athad_gpu.h).
//
// A batch owns no field memory: its members are ordinary mixed-precision contexts, each
// with its own grid and parameters.  One batched model iteration enqueues each member's
// column physics at that member's own cadence (pressure sweep every 4th iteration,
// saturation adjustment + moist convection + densities every 2nd) on a few side streams
// forked from the batch's stream and joined back to it, so that the small kernels of
// different members run side by side (a member's column kernels fill only part of the
// GPU: one thread per column, or latency-bound recurrences), then on the batch's stream the
// level mean of all members in one launch, the four RK4 stages of all members as one
// persistent launch each (k_rk4m.cu), with the time-level copy fused into stage 4, and a
// tiny launch that advances the members' device-side iteration counters.
//
// Step scalars live on the device: every member's buoyancy ramp min(1, n / ramp_iters) is
// formed inside the stage kernels from its iteration counter, so one captured CUDA graph
// of an iteration stays valid from step to step.  Graphs are keyed by what changes the
// launch list: each member's cadence (pressure sweep? column physics?), its pressure
// ceiling (above 300 iterations) and the tile shape; a batch replays at most a handful.
#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "ctx.cuh"

namespace athad {

__global__ void batch_advance_kernel(BatchStep* step, int n)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m < n && step[m].active) step[m].iter += 1;
}

}  // namespace athad

namespace {

constexpr int kMaxShapes = 8;

struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
};

}  // namespace

constexpr int kSideStreams = 8;   // concurrent column-physics lanes of a batched iteration

struct athad_batch {
    std::vector<athad_ctx*> m;
    std::vector<cudaStream_t> side;     // member q's column physics runs on side[q % size]
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    std::vector<int32_t> iter;          // host mirror of each member's next iteration number
    std::vector<uint8_t> active;
    athad_batch_step step{};
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    char* dev = nullptr;                // device tables, one allocation
    RK4MArgs* d_args = nullptr;
    BatchStep* d_step = nullptr;
    int* d_tiles = nullptr;             // [shapes][n+1]
    LevelMeanMember* d_lm = nullptr;
    int n_shapes = 0;
    int shape = 0;
    int grid[kMaxShapes] = {};
    int total_tiles[kMaxShapes] = {};
    int total_levels = 0, max_jm = 0;
    std::map<std::vector<uint8_t>, GraphEntry> graphs;
    std::string err;
};

static athad_status bfail(athad_batch* b, athad_status s, const std::string& msg)
{
    if (b) b->err = msg;
    return s;
}

static athad_status bcuda(athad_batch* b, cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return ATHAD_OK;
    if (b) b->err = std::string(what) + ": " + cudaGetErrorString(e);
    return (e == cudaErrorMemoryAllocation) ? ATHAD_ERR_OOM : ATHAD_ERR_CUDA;
}

static void drop_graphs(athad_batch* b)
{
    for (auto& kv : b->graphs)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    b->graphs.clear();
}

// Enqueue one iteration of every active member on b->stream (also used under capture).
static athad_status enqueue_iteration(athad_batch* b)
{
    const int n = (int)b->m.size();
    const int ns = (int)b->side.size();
    athad_status sf = bcuda(b, cudaEventRecord(b->fork, b->stream), "batch fork");
    for (int q = 0; q < ns && sf == ATHAD_OK; q++) sf = bcuda(b, cudaStreamWaitEvent(b->side[q], b->fork, 0), "batch fork");
    if (sf != ATHAD_OK) return sf;
    for (int q = 0; q < n; q++) {
        if (!b->active[q]) continue;
        athad_ctx* c = b->m[q];
        cudaStream_t saved = c->stream;
        c->stream = b->side[q % ns];
        const int it = b->iter[q];
        athad_status s = ATHAD_OK;
        if (it % 4 == 0) s = athad_pressure_sweep(c, 1, it);
        if (s == ATHAD_OK && it % 2 == 0) {
            s = athad_saturation_adjust(c);
            if (s == ATHAD_OK) s = athad_moist_convection(c, it);
            if (s == ATHAD_OK) s = athad_densities(c, 0);
        }
        c->stream = saved;
        if (s != ATHAD_OK) return bfail(b, s, std::string("member ") + std::to_string(q) + ": " + c->err);
    }
    for (int q = 0; q < ns; q++) {   // join: the batched kernels below read every member's state
        athad_status sj = bcuda(b, cudaEventRecord(b->join[q], b->side[q]), "batch join");
        if (sj == ATHAD_OK) sj = bcuda(b, cudaStreamWaitEvent(b->stream, b->join[q], 0), "batch join");
        if (sj != ATHAD_OK) return sj;
    }
    launch_batch_level_mean(b->d_lm, n, b->total_levels, b->max_jm, b->d_step, b->stream);
    athad_status s = bcuda(b, cudaGetLastError(), "batch level mean");
    if (s != ATHAD_OK) return s;
    BatchTables T;
    T.args = b->d_args;
    T.step = b->d_step;
    T.tile_start = b->d_tiles + (size_t)b->shape * (n + 1);
    T.n = n;
    T.total_tiles = b->total_tiles[b->shape];
    for (int stage = 1; stage <= 4; stage++) {
        launch_rk4m_batch_stage(stage, b->shape, T, b->grid[b->shape], b->stream);
        s = bcuda(b, cudaGetLastError(), "batch rk4 stage");
        if (s != ATHAD_OK) return s;
    }
    // the time-level copy's precipitation fluxes (UtilsAtm.h:41-42); the stage kernel wrote
    // the eleven prognostic fields' level n
    for (int q = 0; q < n; q++) {
        if (!b->active[q]) continue;
        athad_ctx* c = b->m[q];
        s = bcuda(b, cudaMemcpyAsync(c->field[ATHAD_P_RAINN], c->field[ATHAD_P_RAIN],
                                     2 * c->L.field_elems * sizeof(double), cudaMemcpyDeviceToDevice,
                                     b->stream), "batch precipitation level n");
        if (s != ATHAD_OK) return s;
    }
    batch_advance_kernel<<<(n + 127) / 128, 128, 0, b->stream>>>(b->d_step, n);
    return bcuda(b, cudaGetLastError(), "batch advance");
}

static std::vector<uint8_t> graph_key(const athad_batch* b)
{
    std::vector<uint8_t> key;
    key.reserve(b->m.size() + 1);
    key.push_back((uint8_t)b->shape);
    for (size_t q = 0; q < b->m.size(); q++) {
        const int it = b->iter[q];
        uint8_t k = 0;
        if (b->active[q]) {
            k |= 1;
            if (it % 4 == 0) k |= 2;
            if (it % 2 == 0) k |= 4;
            if (it > 300) k |= 8;     // pressure ceiling 3 instead of 10
        }
        key.push_back(k);
    }
    return key;
}

static void advance_host(athad_batch* b)
{
    for (size_t q = 0; q < b->m.size(); q++)
        if (b->active[q]) b->iter[q] += 1;
}

extern "C" {

athad_status athad_batch_create(athad_ctx* const* members, int32_t n_members, const athad_batch_step* step,
                                const int32_t* first_iter, athad_batch** out)
{
    if (!out) return ATHAD_ERR_INVALID;
    *out = nullptr;
    if (!members || n_members < 1 || !step || step->dt <= 0.0 || step->buoyancy_ramp_iters < 1)
        return ATHAD_ERR_INVALID;
    for (int q = 0; q < n_members; q++) {
        if (!members[q]) return ATHAD_ERR_INVALID;
        if (members[q]->p.precision != ATHAD_PRECISION_MIXED) return ATHAD_ERR_UNSUPPORTED;
        for (int r = 0; r < q; r++)
            if (members[r] == members[q]) return ATHAD_ERR_INVALID;
    }
    // the batch runs the members on its own streams: what is queued on theirs (an initial
    // state, an upload) must be complete first
    for (int q = 0; q < n_members; q++)
        if (cudaStreamSynchronize(members[q]->stream) != cudaSuccess) { cudaGetLastError(); return ATHAD_ERR_CUDA; }
    athad_batch* b = new (std::nothrow) athad_batch();
    if (!b) return ATHAD_ERR_OOM;
    b->m.assign(members, members + n_members);
    b->iter.resize(n_members);
    b->active.assign(n_members, 1);
    for (int q = 0; q < n_members; q++) b->iter[q] = first_iter ? first_iter[q] : 1;
    b->step = *step;
    const int n = n_members;
    b->n_shapes = std::min(batch_shape_count(), kMaxShapes);

    // host tables
    std::vector<RK4MArgs> args(n);
    std::vector<BatchStep> steps(n);
    std::vector<LevelMeanMember> lm(n);
    std::vector<int> tiles((size_t)b->n_shapes * (n + 1));
    int level0 = 0;
    for (int q = 0; q < n; q++) {
        athad_ctx* c = members[q];
        athad_step_scalars sc{step->dt, step->diffusion_ramp, 1.0, 0, 0};
        mixed_args(c, &sc, args[q]);
        for (int f = 0; f < kNY; f++) {
            args[q].Yout[f] = c->mA[f];      // stage buffer A
            args[q].Ybnd[f] = c->mB[f];      // stage buffer B
            args[q].Yn_store[f] = c->field[ATHAD_TN + f];
        }
        args[q].store_n = 1;
        BatchStep& s = steps[q];
        std::memset(&s, 0, sizeof s);
        s.half_dt_f = (float)(0.5 * step->dt);
        s.dt_f = (float)step->dt;
        s.diffusion_ramp = (float)step->diffusion_ramp;
        s.drag_pref = args[q].drag_pref;
        s.half_dt = 0.5 * step->dt;
        s.dt_sixth = step->dt / 6.0;
        s.g = c->p.g; s.dt = step->dt; s.u_0 = c->p.u_0;
        s.iter = b->iter[q];
        s.ramp_iters = step->buoyancy_ramp_iters;
        s.write_diag = 0;
        s.active = 1;
        lm[q].d = c->L.d;
        lm[q].t = c->field[ATHAD_T];
        lm[q].sin_w = c->sin_w;
        lm[q].out = c->prof[ATHAD_PROF_T_REF_LEVEL];
        lm[q].level0 = level0;
        level0 += c->L.d.im;
        b->max_jm = std::max(b->max_jm, c->L.d.jm);
    }
    b->total_levels = level0;
    for (int sh = 0; sh < b->n_shapes; sh++) {
        const BatchShape S = batch_shape_info(sh);
        int acc = 0;
        for (int q = 0; q < n; q++) {
            tiles[(size_t)sh * (n + 1) + q] = acc;
            const Dims& d = members[q]->L.d;
            acc += d.im * ((d.jm + S.by - 1) / S.by) * ((d.km + S.bx - 1) / S.bx);
        }
        tiles[(size_t)sh * (n + 1) + n] = acc;
        b->total_tiles[sh] = acc;
        b->grid[sh] = batch_shape_grid(sh);
    }
    b->shape = 0;

    // device tables
    const size_t a_bytes = round_up(sizeof(RK4MArgs) * n, 256);
    const size_t s_bytes = round_up(sizeof(BatchStep) * n, 256);
    const size_t t_bytes = round_up(sizeof(int) * tiles.size(), 256);
    const size_t l_bytes = round_up(sizeof(LevelMeanMember) * n, 256);
    athad_status st = ATHAD_OK;
    if (cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError(); delete b; return ATHAD_ERR_CUDA;
    }
    b->stream = b->own_stream;
    if (cudaMalloc((void**)&b->dev, a_bytes + s_bytes + t_bytes + l_bytes) != cudaSuccess) {
        cudaGetLastError(); cudaStreamDestroy(b->own_stream); delete b; return ATHAD_ERR_OOM;
    }
    b->d_args = (RK4MArgs*)b->dev;
    b->d_step = (BatchStep*)(b->dev + a_bytes);
    b->d_tiles = (int*)(b->dev + a_bytes + s_bytes);
    b->d_lm = (LevelMeanMember*)(b->dev + a_bytes + s_bytes + t_bytes);
    st = bcuda(b, cudaMemcpyAsync(b->d_args, args.data(), sizeof(RK4MArgs) * n, cudaMemcpyHostToDevice, b->stream), "args");
    if (st == ATHAD_OK) st = bcuda(b, cudaMemcpyAsync(b->d_step, steps.data(), sizeof(BatchStep) * n, cudaMemcpyHostToDevice, b->stream), "steps");
    if (st == ATHAD_OK) st = bcuda(b, cudaMemcpyAsync(b->d_tiles, tiles.data(), sizeof(int) * tiles.size(), cudaMemcpyHostToDevice, b->stream), "tiles");
    if (st == ATHAD_OK) st = bcuda(b, cudaMemcpyAsync(b->d_lm, lm.data(), sizeof(LevelMeanMember) * n, cudaMemcpyHostToDevice, b->stream), "levels");
    if (st == ATHAD_OK) st = bcuda(b, cudaStreamSynchronize(b->stream), "batch create sync");
    // the side streams and events of the column-physics fork/join
    if (st == ATHAD_OK) st = bcuda(b, cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "batch events");
    const int ns = std::min(n, kSideStreams);
    for (int q = 0; q < ns && st == ATHAD_OK; q++) {
        cudaStream_t s = nullptr;
        cudaEvent_t e = nullptr;
        st = bcuda(b, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "batch side stream");
        if (st == ATHAD_OK) b->side.push_back(s);
        if (st == ATHAD_OK) st = bcuda(b, cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "batch events");
        if (st == ATHAD_OK) b->join.push_back(e);
    }
    if (st != ATHAD_OK) {
        for (cudaStream_t s : b->side) cudaStreamDestroy(s);
        for (cudaEvent_t e : b->join) cudaEventDestroy(e);
        if (b->fork) cudaEventDestroy(b->fork);
        cudaFree(b->dev); cudaStreamDestroy(b->own_stream); delete b;
        return st;
    }
    *out = b;
    return ATHAD_OK;
}

athad_status athad_batch_destroy(athad_batch* b)
{
    if (!b) return ATHAD_ERR_INVALID;
    cudaStreamSynchronize(b->stream);
    drop_graphs(b);
    for (cudaStream_t s : b->side) { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
    for (cudaEvent_t e : b->join) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    cudaFree(b->dev);
    cudaStreamDestroy(b->own_stream);
    delete b;
    return ATHAD_OK;
}

const char* athad_batch_last_error(const athad_batch* b)
{
    return b ? b->err.c_str() : "null batch";
}

athad_status athad_batch_set_stream(athad_batch* b, void* s)
{
    if (!b) return ATHAD_ERR_INVALID;
    cudaStream_t ns = s ? (cudaStream_t)s : b->own_stream;
    if (ns != b->stream) drop_graphs(b);
    b->stream = ns;
    return ATHAD_OK;
}

athad_status athad_batch_synchronize(athad_batch* b)
{
    if (!b) return ATHAD_ERR_INVALID;
    return bcuda(b, cudaStreamSynchronize(b->stream), "batch synchronize");
}

athad_status athad_batch_member_iter(const athad_batch* b, int32_t member, int32_t* next_iter)
{
    if (!b || !next_iter || member < 0 || member >= (int32_t)b->m.size()) return ATHAD_ERR_INVALID;
    *next_iter = b->iter[member];
    return ATHAD_OK;
}

athad_status athad_batch_set_active(athad_batch* b, int32_t member, int32_t active)
{
    if (!b || member < 0 || member >= (int32_t)b->m.size()) return ATHAD_ERR_INVALID;
    const uint8_t a = active ? 1 : 0;
    if (b->active[member] == a) return ATHAD_OK;
    b->active[member] = a;
    const int32_t v = a;
    return bcuda(b, cudaMemcpyAsync(&b->d_step[member].active, &v, sizeof v, cudaMemcpyHostToDevice, b->stream),
                 "set active");
}

athad_status athad_batch_iteration(athad_batch* b)
{
    if (!b) return ATHAD_ERR_INVALID;
    athad_status s = enqueue_iteration(b);
    if (s == ATHAD_OK) advance_host(b);
    return s;
}

athad_status athad_batch_iteration_graph(athad_batch* b)
{
    if (!b) return ATHAD_ERR_INVALID;
    const std::vector<uint8_t> key = graph_key(b);
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
        if (b->graphs.size() >= 16) drop_graphs(b);
        cudaGraph_t graph = nullptr;
        athad_status s = bcuda(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        if (s != ATHAD_OK) return s;
        athad_status se = enqueue_iteration(b);
        cudaError_t ee = cudaStreamEndCapture(b->stream, &graph);
        if (se != ATHAD_OK) { if (graph) cudaGraphDestroy(graph); return se; }
        s = bcuda(b, ee, "end capture");
        if (s != ATHAD_OK) return s;
        GraphEntry g;
        s = bcuda(b, cudaGraphInstantiate(&g.exec, graph, 0), "instantiate");
        cudaGraphDestroy(graph);
        if (s != ATHAD_OK) return s;
        it = b->graphs.emplace(key, g).first;
    }
    athad_status s = bcuda(b, cudaGraphLaunch(it->second.exec, b->stream), "graph launch");
    if (s == ATHAD_OK) advance_host(b);
    return s;
}

int32_t athad_batch_shape_count(void) { return batch_shape_count(); }

athad_status athad_batch_set_shape(athad_batch* b, int32_t shape)
{
    if (!b || shape < 0 || shape >= b->n_shapes) return ATHAD_ERR_INVALID;
    if (shape != b->shape) drop_graphs(b);
    b->shape = shape;
    return ATHAD_OK;
}

athad_status athad_batch_autotune(athad_batch* b, int32_t reps, int32_t* best_shape, float* ms_per_shape)
{
    if (!b || reps < 1) return ATHAD_ERR_INVALID;
    const int n = (int)b->m.size();
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cudaGetLastError(); return bfail(b, ATHAD_ERR_CUDA, "autotune events");
    }
    float best = 3.4e38f;
    int best_id = b->shape;
    athad_status s = ATHAD_OK;
    for (int sh = 0; sh < b->n_shapes && s == ATHAD_OK; sh++) {
        BatchTables T;
        T.args = b->d_args; T.step = b->d_step;
        T.tile_start = b->d_tiles + (size_t)sh * (n + 1);
        T.n = n; T.total_tiles = b->total_tiles[sh];
        // stages 1-3 write only the members' private FP32 buffers, which the next
        // iteration's stage 1 rewrites, so timing them leaves the model state unchanged
        for (int stage = 1; stage <= 3; stage++) launch_rk4m_batch_stage(stage, sh, T, b->grid[sh], b->stream);
        cudaEventRecord(e0, b->stream);
        for (int r = 0; r < reps; r++)
            for (int stage = 1; stage <= 3; stage++) launch_rk4m_batch_stage(stage, sh, T, b->grid[sh], b->stream);
        cudaEventRecord(e1, b->stream);
        s = bcuda(b, cudaEventSynchronize(e1), "autotune");
        float ms = 0.0f;
        if (s == ATHAD_OK) s = bcuda(b, cudaEventElapsedTime(&ms, e0, e1), "autotune time");
        ms /= (float)reps;
        if (ms_per_shape) ms_per_shape[sh] = ms;
        if (s == ATHAD_OK && ms < best) { best = ms; best_id = sh; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s != ATHAD_OK) return s;
    if (best_id != b->shape) drop_graphs(b);
    b->shape = best_id;
    if (best_shape) *best_shape = best_id;
    return ATHAD_OK;
}

}  // extern "C"
