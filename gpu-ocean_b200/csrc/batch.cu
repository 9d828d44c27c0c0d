// Batched CDKLM16 stepping: many members (an ensemble, or independent
// domains of uneven sizes) advanced by one launch per Runge-Kutta stage over
// a packed tile list, optionally replayed from a captured CUDA graph.
//
// Replaces the member-by-member stepping of the reference's ensembles
// (gpu_ocean/SWESimulators/OceanNoiseEnsemble.py:506-531,
// OceanModelEnsemble.py:105-117, EnsembleFromFiles.py:302-324), which issue
// N_members x (2 step + up to 4 boundary) launches per time step from Python.
#include <algorithm>
#include <vector>

#include "grf.cuh"
#include "trace.h"
#include "pair_dispatch.cuh"

using namespace go;

// State of the device-driven ensemble event loop: per event every member
// advances `interval` seconds of model time at the common dt with the
// reference's step(t_end) rule (CDKLM16.py:494-598: whole steps while one
// fits, then one short step), gets the model error of the event, and the
// common dt = courant x the least CFL limit over the members.
struct EventLoop {
    double interval;     // model seconds per event
    double t_now;        // model time into the current event
    double courant;
    float dt;            // common time step
    int last;            // the short last step of the event is under way
    uint32_t event;      // model-error event of the current event
    int events_left;
    long long steps;
};

// What a captured event-loop graph depends on besides the loop state.
struct EventLoopKey {
    uint32_t key0 = 0;
    float std_dev = 0.0f, corr_cells = 0.0f;
    const float* scratch = nullptr;
    bool valid = false;
    bool operator==(const EventLoopKey& o) const {
        return valid && o.valid && key0 == o.key0 && std_dev == o.std_dev && corr_cells == o.corr_cells &&
               scratch == o.scratch;
    }
};

struct go_batch {
    int n = 0;
    std::vector<go_domain*> members;
    std::vector<StageArgs> args;       // 2 per member
    std::vector<char> member_set;
    std::vector<float> dt;             // per member
    StageArgs* d_args = nullptr;
    float* d_dt = nullptr;
    int4* d_tiles = nullptr;
    int ntiles = 0;
    // column-pair shape: boundary-free tiles (d_tiles, TMA maps in d_maps)
    // and boundary-frame tiles (d_tiles_frame) launched as two kernels, the
    // frame on a high-priority side stream
    int4* d_tiles_frame = nullptr;
    int ntiles_frame = 0;
    PairMapParams* d_maps = nullptr;
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int shape = 4, rows = 32, blocks = 0;
    int arith = 0;
    Variant variant;
    bool dirty = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_steps = 0;
    GrfMember* d_grf = nullptr;        // model-error descriptors (built on first use)
    int grf_R = -1;
    size_t grf_scratch = 0;
    int grf_max_nx = 0, grf_max_ny = 0;
    // device-driven event loop (go_batch_run_events): its state, the
    // members' model times, the CFL limits, the graph and what it captured
    EventLoop* d_loop = nullptr;
    double* d_t = nullptr;
    unsigned int* d_cfl = nullptr;
    cudaStream_t loop_side = nullptr;
    cudaGraph_t loop_graph = nullptr;
    cudaGraphExec_t loop_exec = nullptr;
    EventLoopKey loop_key;
    std::vector<double> loop_t;
};

namespace {

struct BatchLaunch {
    const go_batch* b;
    int rk_step, grid;
    cudaStream_t s;
    template <int BW, int MINB, int FRIC, bool GN, bool WF, bool RCP, bool LAND, int D>
    cudaError_t run() {
        cdklm_batch_kernel<BW, MINB, FRIC, GN, WF, RCP, LAND, D><<<grid, BW, 0, s>>>(b->d_args, b->d_dt, b->d_tiles,
                                                                                 b->ntiles, rk_step);
        return cudaGetLastError();
    }
};

// Kernel variant of the members as set: friction law and grid angle from
// the domains, per-cell wind from the member arguments (a member's wind
// field is usually handed to its domain after the batch is created), land
// checks if any member may hold land.
int batch_variant(go_batch* b) {
    Variant v = go_variant(b->members[0]);
    v.wind_field = b->args[0].wx_cur != nullptr;
    v.land = false;
    for (int m = 0; m < b->n; ++m) {
        const go_domain* d = b->members[m];
        v.land = v.land || d->has_land;
        if (go_friction_mode(d) != v.fric || go_general_north(d) != v.gen_north ||
            (b->args[2 * m].wx_cur != nullptr) != v.wind_field)
            return go_fail(GO_ERR_INVALID,
                           "member %d needs a different kernel variant (friction law, grid angle or wind "
                           "field) than member 0; use one batch per variant", m);
    }
    b->variant = v;
    return GO_OK;
}

// Tiles of the column-pair kernel: per member its boundary-free rectangle
// (when every array of the member qualifies for TMA) and its boundary frame
// in short strips, with the member's TMA maps for both stages.
int batch_commit_pair(go_batch* b) {
    std::vector<int4> ti, tf;
    std::vector<PairMapParams> maps(2 * b->n);
    for (int m = 0; m < b->n; ++m) {
        const Scheme& k = b->members[m]->k;
        b->args[2 * m].rows_per_block = b->rows;
        b->args[2 * m + 1].rows_per_block = b->rows;
        bool t0 = false, t1 = false;
        int rc = go_prepare_pair(b->args[2 * m], &maps[2 * m], &t0);
        if (!rc) rc = go_prepare_pair(b->args[2 * m + 1], &maps[2 * m + 1], &t1);
        if (rc) return rc;
        const PairGrid g = pair_grid(k, b->rows, t0 && t1);
        for (int by = 0; by < g.nby; ++by) {
            const int r0 = 4 + by * g.rows;
            const int r1 = std::min(r0 + g.rows, k.ny);
            for (int bx = g.bx0; bx < g.bx1; ++bx) ti.push_back(make_int4(m, bx, r0, r1));
        }
        const int nf = pair_frame_count(g);
        for (int i = 0; i < nf; ++i) {
            int bx, r0, r1;
            pair_frame_block(g, i, bx, r0, r1);
            tf.push_back(make_int4(m, bx, r0, r1));
        }
    }
    cudaFree(b->d_tiles);
    cudaFree(b->d_tiles_frame);
    cudaFree(b->d_maps);
    b->d_tiles = b->d_tiles_frame = nullptr;
    b->d_maps = nullptr;
    if (!ti.empty()) {
        GO_CUDA(cudaMalloc(&b->d_tiles, sizeof(int4) * ti.size()));
        GO_CUDA(cudaMemcpy(b->d_tiles, ti.data(), sizeof(int4) * ti.size(), cudaMemcpyHostToDevice));
    }
    if (!tf.empty()) {
        GO_CUDA(cudaMalloc(&b->d_tiles_frame, sizeof(int4) * tf.size()));
        GO_CUDA(cudaMemcpy(b->d_tiles_frame, tf.data(), sizeof(int4) * tf.size(), cudaMemcpyHostToDevice));
    }
    GO_CUDA(cudaMalloc(&b->d_maps, sizeof(PairMapParams) * maps.size()));
    GO_CUDA(cudaMemcpy(b->d_maps, maps.data(), sizeof(PairMapParams) * maps.size(), cudaMemcpyHostToDevice));
    if (!b->side) {
        int least = 0, greatest = 0;
        GO_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        GO_CUDA(cudaStreamCreateWithPriority(&b->side, cudaStreamNonBlocking, greatest));
        GO_CUDA(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
        GO_CUDA(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
    }
    GO_CUDA(cudaMemcpy(b->d_args, b->args.data(), sizeof(StageArgs) * b->args.size(), cudaMemcpyHostToDevice));
    GO_CUDA(cudaMemcpy(b->d_dt, b->dt.data(), sizeof(float) * b->n, cudaMemcpyHostToDevice));
    b->ntiles = (int)ti.size();
    b->ntiles_frame = (int)tf.size();
    b->dirty = false;
    return GO_OK;
}

int batch_commit(go_batch* b) {
    if (!b->dirty) return GO_OK;
    for (int m = 0; m < b->n; ++m)
        if (!b->member_set[m]) return go_fail(GO_ERR_INVALID, "batch member %d has no state set", m);
    int rc = batch_variant(b);
    if (rc) return rc;
    Variant v = b->variant;
    v.shape = b->shape;
    v.rcp = b->arith == GO_ARITH_RCP;
    if (go_pair_shape(b->shape)) return batch_commit_pair(b);
    const int width = dispatch_width(v) - 4;
    std::vector<int4> tiles;
    for (int m = 0; m < b->n; ++m) {
        const Scheme& k = b->members[m]->k;
        const int gx = (k.nx + width - 1) / width;
        const int gy = (k.ny + b->rows - 1) / b->rows;
        for (int y = 0; y < gy; ++y)
            for (int x = 0; x < gx; ++x) tiles.push_back(make_int4(m, x, y, 0));
        b->args[2 * m].rows_per_block = b->rows;
        b->args[2 * m + 1].rows_per_block = b->rows;
    }
    cudaFree(b->d_tiles);
    b->d_tiles = nullptr;
    GO_CUDA(cudaMalloc(&b->d_tiles, sizeof(int4) * tiles.size()));
    GO_CUDA(cudaMemcpy(b->d_tiles, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice));
    GO_CUDA(cudaMemcpy(b->d_args, b->args.data(), sizeof(StageArgs) * b->args.size(), cudaMemcpyHostToDevice));
    GO_CUDA(cudaMemcpy(b->d_dt, b->dt.data(), sizeof(float) * b->n, cudaMemcpyHostToDevice));
    b->ntiles = (int)tiles.size();
    b->dirty = false;
    return GO_OK;
}

int batch_launch_pair(go_batch* b, int rk_step, cudaStream_t s) {
    Variant v = b->variant;
    v.shape = b->shape;
    v.rcp = b->arith == GO_ARITH_RCP;
    const bool fork_join = b->ntiles > 0 && b->ntiles_frame > 0;
    PairBatchReq r{b->d_args, b->d_dt, b->d_tiles_frame, b->ntiles_frame, b->ntiles_frame, rk_step, b->d_maps, s};
    if (fork_join) {
        GO_CUDA(cudaEventRecord(b->ev_fork, s));
        GO_CUDA(cudaStreamWaitEvent(b->side, b->ev_fork, 0));
        r.s = b->side;
    }
    if (b->ntiles_frame > 0) {
        const cudaError_t e = pair_batch_launch_frame(r, v);
        if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "batch stage launch (frame) failed: %s", cudaGetErrorString(e));
    }
    if (b->ntiles > 0) {
        r.s = s;
        r.tiles = b->d_tiles;
        r.ntiles = b->ntiles;
        r.grid = (b->blocks > 0 && b->blocks < b->ntiles) ? b->blocks : b->ntiles;
        const cudaError_t e = pair_batch_launch_interior(r, v);
        if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "batch stage launch failed: %s", cudaGetErrorString(e));
    }
    if (fork_join) {
        GO_CUDA(cudaEventRecord(b->ev_join, b->side));
        GO_CUDA(cudaStreamWaitEvent(s, b->ev_join, 0));
    }
    if (b->ntiles > 0) {
        // periodic east/west ghost columns of every member (the kernel skips
        // the others): the region's strips leave them to this copy
        StageArgs none;
        memset(&none, 0, sizeof(none));
        int most = 0;
        for (const go_domain* d : b->members) most = std::max(most, d->k.ny);
        GO_CUDA(pair_launch_periodic_columns(b->d_args, b->n, most, rk_step, none, s));
    }
    return GO_OK;
}

int batch_launch(go_batch* b, int rk_step, cudaStream_t s) {
    if (go_pair_shape(b->shape)) return batch_launch_pair(b, rk_step, s);
    int grid = b->ntiles;
    if (b->blocks > 0 && b->blocks < grid) grid = b->blocks;
    BatchLaunch L{b, rk_step, grid, s};
    Variant v = b->variant;
    v.shape = b->shape;
    v.rcp = b->arith == GO_ARITH_RCP;
    const cudaError_t e = dispatch_variant(L, v);
    if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "batch stage launch failed: %s", cudaGetErrorString(e));
    return GO_OK;
}

// CFL limit of every member in one launch: blockIdx.y is the member, whose
// current state (h0) is the input of its stage-0 arguments; the cell-mean
// bathymetry comes from the corners as the set-up computes it.
__global__ void k_batch_max_dt(const StageArgs* __restrict__ args, unsigned int* __restrict__ out) {
    const StageArgs& a = args[2 * blockIdx.y];
    const Scheme& k = a.k;
    const int n = k.nx * k.ny;
    float best = kRefFltMax;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        const int j = idx / k.nx + 2, i = idx % k.nx + 2;
        const size_t o = (size_t)j * a.pin + i;
        const float* H = a.Hi + (size_t)j * a.phi + i;
        const float Hm = cell_mean_depth(H[0], H[a.phi], H[1], H[a.phi + 1], k.land);
        best = fminf(best, cell_cfl_dt(a.eta_in[o], a.hu_in[o], a.hv_in[o], Hm, k.dx, k.dy, k.g, k.land,
                                       kRefFltMax));
    }
    block_min_to(best, out + blockIdx.y, kRefFltMax);
}

__global__ void k_fill_members(unsigned int* p, unsigned int v, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

void drop_graph(go_batch* b) {
    if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->graph_exec = nullptr;
    b->graph = nullptr;
    b->graph_steps = 0;
    if (b->loop_exec) cudaGraphExecDestroy(b->loop_exec);
    if (b->loop_graph) cudaGraphDestroy(b->loop_graph);
    b->loop_exec = nullptr;
    b->loop_graph = nullptr;
    b->loop_key.valid = false;
}

// Launches of go_batch_max_dt: every member's CFL limit (float bits) into out.
int launch_max_dt(go_batch* b, cudaStream_t s, unsigned int* out) {
    unsigned int init_bits;
    memcpy(&init_bits, &kRefFltMax, sizeof(init_bits));
    k_fill_members<<<(b->n + 255) / 256, 256, 0, s>>>(out, init_bits, b->n);
    long long most = 0;
    for (const go_domain* d : b->members) most = std::max(most, (long long)d->k.nx * d->k.ny);
    // about 4 blocks per SM in all, spread over the members
    const int per_member = (int)std::max(1LL, std::min((most + 255) / 256, (148LL * 4 + b->n - 1) / b->n));
    k_batch_max_dt<<<dim3(per_member, b->n), 256, 0, s>>>(b->d_args, out);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

// Model-error descriptors of the members (their eta buffers, sizes,
// boundary kinds, member keys, scratch offsets) for filter radius W.R.
int grf_prepare(go_batch* b, const GrfWeights& W) {
    if (b->d_grf && b->grf_R == W.R) return GO_OK;
    std::vector<GrfMember> h(b->n);
    size_t off = 0;
    int mx = 0, my = 0;
    for (int m = 0; m < b->n; ++m) {
        const Scheme& k = b->members[m]->k;
        h[m].eta = const_cast<float*>(b->args[2 * m].eta_in);
        h[m].pitch = b->args[2 * m].pin;
        h[m].nx = k.nx;
        h[m].ny = k.ny;
        h[m].periodic_x = k.bcE == kPeriodic;
        h[m].periodic_y = k.bcN == kPeriodic;
        h[m].key1 = (uint32_t)m;
        h[m].tmp_off = off;
        off += grf_member_scratch(k.nx, k.ny, W.R);
        mx = max(mx, k.nx);
        my = max(my, k.ny);
    }
    if (!b->d_grf) GO_CUDA(cudaMalloc(&b->d_grf, sizeof(GrfMember) * b->n));
    GO_CUDA(cudaMemcpy(b->d_grf, h.data(), sizeof(GrfMember) * b->n, cudaMemcpyHostToDevice));
    b->grf_R = W.R;
    b->grf_scratch = off;
    b->grf_max_nx = mx;
    b->grf_max_ny = my;
    return GO_OK;
}

// ---- device-driven event loop ----------------------------------------------
// The step of the event that starts at t_now: the common dt, or the model
// time left in the event rounded to float32 when that is shorter, which
// makes it the event's last step (CDKLM16.py:508-517: local_dt =
// float32(min(dt, float32(t_end - t_now))), the whole-step loop stops at the
// first step shorter than dt).
__device__ __forceinline__ float event_step_dt(EventLoop* L) {
    const float rem = __double2float_rn(__dsub_rn(L->interval, L->t_now));
    const float local = fminf(L->dt, rem);
    if (local != L->dt) L->last = 1;
    return local;
}

// Start of an event: its first step's dt into every member's dt; the step
// loop's condition set.
__global__ void k_event_begin(EventLoop* L, float* __restrict__ dts, int n, cudaGraphConditionalHandle steps) {
    __shared__ float sdt;
    if (threadIdx.x == 0) {
        L->t_now = 0.0;
        L->last = 0;
        sdt = event_step_dt(L);
        cudaGraphSetConditional(steps, 1u);
    }
    __syncthreads();
    for (int m = threadIdx.x; m < n; m += blockDim.x) dts[m] = sdt;
}

// After a step: the members' model times advance by the dt they stepped
// with (float64 sums, as CDKLM16.step keeps t), then the next step's dt or
// the end of the event (the step loop's condition).
__global__ void k_step_done(EventLoop* L, float* __restrict__ dts, double* __restrict__ t, int n,
                            cudaGraphConditionalHandle steps) {
    __shared__ float snext;
    __shared__ int scont;
    for (int m = threadIdx.x; m < n; m += blockDim.x) t[m] = __dadd_rn(t[m], (double)dts[m]);
    __syncthreads();
    if (threadIdx.x == 0) {
        L->steps += 1;
        int cont = 0;
        float next = 0.0f;
        if (!L->last) {
            L->t_now = __dadd_rn(L->t_now, (double)L->dt);
            if (L->t_now < L->interval) {
                next = event_step_dt(L);
                cont = 1;
            }
        }
        snext = next;
        scont = cont;
        cudaGraphSetConditional(steps, (unsigned)cont);
    }
    __syncthreads();
    if (scont)
        for (int m = threadIdx.x; m < n; m += blockDim.x) dts[m] = snext;
}

// End of an event, after its model error and the members' CFL limits: the
// common dt = float32(courant x least limit) (float64 product, as the host
// computes it), the next event, the event loop's condition.
__global__ void k_event_end(EventLoop* L, const unsigned int* __restrict__ cfl, float* __restrict__ dts, int n,
                            cudaGraphConditionalHandle events) {
    __shared__ float red[256];
    float mn = kRefFltMax;
    for (int m = threadIdx.x; m < n; m += blockDim.x) mn = fminf(mn, __uint_as_float(cfl[m]));
    red[threadIdx.x] = mn;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] = fminf(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const float dt = __double2float_rn(__dmul_rn(L->courant, (double)red[0]));
        L->dt = dt;
        L->event += 1;
        L->events_left -= 1;
        cudaGraphSetConditional(events, L->events_left > 0 ? 1u : 0u);
        red[0] = dt;
    }
    __syncthreads();
    const float dt = red[0];
    for (int m = threadIdx.x; m < n; m += blockDim.x) dts[m] = dt;
}

// The graph of the event loop: WHILE (events left) { event begin; WHILE
// (steps left) { stage 0; stage 1; step done }; model error; CFL limits;
// event end }.  s captures the event body, b->loop_side the step body.
int build_event_graph(go_batch* b, cudaStream_t s, const GrfWeights& W, uint32_t key0, float std_dev,
                      float* scratch) {
    cudaGraph_t g = nullptr;
    GO_CUDA(cudaGraphCreate(&g, 0));
    int rc = GO_OK;
    bool capturing_s = false, capturing_side = false;
    auto fail = [&](cudaError_t e, const char* what) {
        if (rc == GO_OK) rc = go_fail(GO_ERR_CUDA, "event loop graph: %s: %s", what, cudaGetErrorString(e));
    };
    do {
        cudaGraphConditionalHandle h_events, h_steps;
        cudaError_t e = cudaGraphConditionalHandleCreate(&h_events, g, 1u, cudaGraphCondAssignDefault);
        if (e != cudaSuccess) { fail(e, "handle"); break; }
        cudaGraphNodeParams pe = {cudaGraphNodeTypeConditional};
        pe.conditional.handle = h_events;
        pe.conditional.type = cudaGraphCondTypeWhile;
        pe.conditional.size = 1;
        cudaGraphNode_t n_events;
        e = cudaGraphAddNode(&n_events, g, nullptr, 0, &pe);
        if (e != cudaSuccess) { fail(e, "event loop node"); break; }
        cudaGraph_t body_events = pe.conditional.phGraph_out[0];
        e = cudaGraphConditionalHandleCreate(&h_steps, body_events, 1u, 0);
        if (e != cudaSuccess) { fail(e, "step handle"); break; }

        e = cudaStreamBeginCaptureToGraph(s, body_events, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) { fail(e, "capture"); break; }
        capturing_s = true;
        k_event_begin<<<1, 256, 0, s>>>(b->d_loop, b->d_dt, b->n, h_steps);
        cudaStreamCaptureStatus st;
        cudaGraph_t cg = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t ndeps = 0;
        e = cudaStreamGetCaptureInfo(s, &st, nullptr, &cg, &deps, &ndeps);
        if (e != cudaSuccess) { fail(e, "capture info"); break; }
        cudaGraphNodeParams ps = {cudaGraphNodeTypeConditional};
        ps.conditional.handle = h_steps;
        ps.conditional.type = cudaGraphCondTypeWhile;
        ps.conditional.size = 1;
        cudaGraphNode_t n_steps;
        e = cudaGraphAddNode(&n_steps, cg, deps, ndeps, &ps);
        if (e != cudaSuccess) { fail(e, "step loop node"); break; }
        e = cudaStreamUpdateCaptureDependencies(s, &n_steps, 1, cudaStreamSetCaptureDependencies);
        if (e != cudaSuccess) { fail(e, "capture dependencies"); break; }

        e = cudaStreamBeginCaptureToGraph(b->loop_side, ps.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) { fail(e, "step body capture"); break; }
        capturing_side = true;
        rc = batch_launch(b, 0, b->loop_side);
        if (!rc) rc = batch_launch(b, 1, b->loop_side);
        if (rc) break;
        k_step_done<<<1, 256, 0, b->loop_side>>>(b->d_loop, b->d_dt, b->d_t, b->n, h_steps);
        cudaGraph_t done = nullptr;
        capturing_side = false;
        e = cudaStreamEndCapture(b->loop_side, &done);
        if (e != cudaSuccess) { fail(e, "step body capture end"); break; }

        GrfMember none;
        memset(&none, 0, sizeof(none));
        rc = grf_launch(b->d_grf, none, b->n, b->grf_max_nx, b->grf_max_ny, key0, 0u, std_dev, W, scratch, s,
                        &b->d_loop->event);
        if (!rc) rc = launch_max_dt(b, s, b->d_cfl);
        if (rc) break;
        k_event_end<<<1, 256, 0, s>>>(b->d_loop, b->d_cfl, b->d_dt, b->n, h_events);
        capturing_s = false;
        e = cudaStreamEndCapture(s, &done);
        if (e != cudaSuccess) { fail(e, "event body capture end"); break; }
        e = cudaGraphInstantiate(&b->loop_exec, g, 0);
        if (e != cudaSuccess) { fail(e, "instantiate"); break; }
    } while (false);
    if (capturing_side) {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(b->loop_side, &junk);
    }
    if (capturing_s) {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(s, &junk);
    }
    if (rc) {
        cudaGetLastError();
        if (b->loop_exec) cudaGraphExecDestroy(b->loop_exec);
        b->loop_exec = nullptr;
        cudaGraphDestroy(g);
        return rc;
    }
    b->loop_graph = g;
    return GO_OK;
}

}  // namespace

extern "C" {

int go_batch_create(go_domain* const* members, int n, go_batch** out) {
    if (!members || !out || n < 1) return go_fail(GO_ERR_INVALID, "need at least one member");
    *out = nullptr;
    go_batch* b = new go_batch();
    b->n = n;
    b->members.assign(members, members + n);
    for (int m = 0; m < n; ++m) {
        if (!members[m]) {
            delete b;
            return go_fail(GO_ERR_INVALID, "member %d is null", m);
        }
    }
    const go_domain* d0 = members[0];
    b->variant = go_variant(d0);
    b->arith = d0->arith;
    // 32-row strips (a batch launches enough blocks for long strips) and,
    // once the tiles need more than one wave of blocks, the read-ahead shape
    // with the less column work (measured on a B200, 100 members of 512^2:
    // 1597 us per step with 128 x 5 blocks of 16 rows and register prefetch,
    // 1532 with the ring, 1431 with 96-wide ring blocks and 32 rows).
    b->rows = 32;
    {
        long long work5 = 0, work6 = 0;
        for (int m = 0; m < n; ++m) {
            const Scheme& k = members[m]->k;
            work5 += shape_columns(5, k.nx) * k.ny;
            work6 += shape_columns(6, k.nx) * k.ny;
        }
        const int ring = ring_shape(work5, work6);
        long long tiles = 0;
        for (int m = 0; m < n; ++m) {
            const Scheme& k = members[m]->k;
            tiles += shape_columns(ring, k.nx) / shape_block_width(ring) * ((k.ny + b->rows - 1) / b->rows);
        }
        b->shape = tiles > 148LL * shape_blocks_per_sm(ring) ? ring : 4;
        // the column-pair kernel once the batch holds a few million cells
        // (measured on a B200, us per step with the ring shape / the pair
        // shape: 100 members of 512^2 1524 / 1145; 16 members 307 / 272;
        // 4 members 123 / 125)
        long long cells = 0;
        for (int m = 0; m < n; ++m) cells += (long long)members[m]->k.nx * members[m]->k.ny;
        if (cells >= kPairAutoBatchCells) b->shape = GO_SHAPE_PAIR;
    }
    for (int m = 0; m < n; ++m) {
        const go_domain* d = members[m];
        if (go_has_open_bc(d)) {
            delete b;
            return go_fail(GO_ERR_UNSUPPORTED, "member %d has open boundaries, which the batch does not run", m);
        }
        if (go_friction_mode(d) != b->variant.fric || go_general_north(d) != b->variant.gen_north) {
            delete b;
            return go_fail(GO_ERR_INVALID,
                           "member %d needs a different kernel variant (friction law or grid angle) than "
                           "member 0; use one batch per variant", m);
        }
    }
    b->args.resize(2 * n);
    b->member_set.assign(n, 0);
    b->dt.assign(n, 0.0f);
    cudaError_t e = cudaMalloc(&b->d_args, sizeof(StageArgs) * 2 * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_dt, sizeof(float) * n);
    if (e != cudaSuccess) {
        cudaFree(b->d_args);
        cudaFree(b->d_dt);
        delete b;
        return go_fail(GO_ERR_CUDA, "batch allocation failed: %s", cudaGetErrorString(e));
    }
    *out = b;
    return GO_OK;
}

int go_batch_destroy(go_batch* b) {
    if (!b) return GO_OK;
    drop_graph(b);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    cudaFree(b->d_tiles_frame);
    cudaFree(b->d_maps);
    cudaFree(b->d_args);
    cudaFree(b->d_dt);
    cudaFree(b->d_tiles);
    cudaFree(b->d_grf);
    cudaFree(b->d_loop);
    cudaFree(b->d_t);
    cudaFree(b->d_cfl);
    if (b->loop_side) cudaStreamDestroy(b->loop_side);
    delete b;
    return GO_OK;
}

int go_batch_set_member(go_batch* b, int m, float dt, float* eta0, float* hu0, float* hv0, int pitch0,
                        float* eta1, float* hu1, float* hv1, int pitch1, const float* Hi, int Hi_pitch,
                        float land_value, float wind_stress_t) {
    if (!b || m < 0 || m >= b->n) return go_fail(GO_ERR_INVALID, "bad batch or member index %d", m);
    if (!eta0 || !hu0 || !hv0 || !eta1 || !hu1 || !hv1 || !Hi) return go_fail(GO_ERR_INVALID, "null argument");
    const go_domain* d = b->members[m];
    int rc = go_check_pitch(pitch0, d->k.nx + 4, "h0");
    if (!rc) rc = go_check_pitch(pitch1, d->k.nx + 4, "h1");
    if (!rc) rc = go_check_pitch(Hi_pitch, d->k.nx + 5, "Hi");
    if (rc) return rc;
    b->args[2 * m] = go_stage_args(d, dt, 0, eta0, hu0, hv0, pitch0 / 4, eta1, hu1, hv1, pitch1 / 4, Hi,
                                   Hi_pitch / 4, land_value, wind_stress_t);
    b->args[2 * m + 1] = go_stage_args(d, dt, 1, eta1, hu1, hv1, pitch1 / 4, eta0, hu0, hv0, pitch0 / 4, Hi,
                                       Hi_pitch / 4, land_value, wind_stress_t);
    b->dt[m] = dt;
    b->member_set[m] = 1;
    b->dirty = true;
    b->grf_R = -1;          // model-error descriptors hold the state pointers
    drop_graph(b);
    return GO_OK;
}

int go_batch_set_launch(go_batch* b, int shape, int rows_per_block, int blocks) {
    if (!b) return go_fail(GO_ERR_INVALID, "null batch");
    if (shape < 0 || shape > GO_SHAPE_PAIR) return go_fail(GO_ERR_INVALID, "launch shape %d (0..8)", shape);
    if (rows_per_block == 0) rows_per_block = 32;
    if (rows_per_block < 1 || blocks < 0) return go_fail(GO_ERR_INVALID, "rows_per_block >= 1, blocks >= 0");
    b->shape = shape;
    b->rows = rows_per_block;
    b->blocks = blocks;
    b->dirty = true;
    drop_graph(b);
    return GO_OK;
}

int go_batch_set_arith(go_batch* b, int mode) {
    if (!b) return go_fail(GO_ERR_INVALID, "null batch");
    if (mode != GO_ARITH_EXACT && mode != GO_ARITH_RCP) return go_fail(GO_ERR_INVALID, "arith mode %d", mode);
    b->arith = mode;
    drop_graph(b);
    return GO_OK;
}

int go_batch_set_dt(go_batch* b, void* stream, const float* dt_host) {
    if (!b || !dt_host) return go_fail(GO_ERR_INVALID, "null argument");
    for (int m = 0; m < b->n; ++m) {
        b->dt[m] = dt_host[m];
        b->args[2 * m].dt = dt_host[m];
        b->args[2 * m + 1].dt = dt_host[m];
    }
    if (b->dirty) return GO_OK;  // uploaded by the next commit
    GO_CUDA(cudaMemcpyAsync(b->d_dt, b->dt.data(), sizeof(float) * b->n, cudaMemcpyHostToDevice,
                            (cudaStream_t)stream));
    GO_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    return GO_OK;
}

int go_batch_tiles(go_batch* b, int* ntiles) {
    if (!b || !ntiles) return go_fail(GO_ERR_INVALID, "null argument");
    int rc = batch_commit(b);
    if (rc) return rc;
    *ntiles = b->ntiles + b->ntiles_frame;
    return GO_OK;
}

int go_batch_step(go_batch* b, void* stream, int n_steps) {
    GO_TRACE("go_batch_step");
    if (!b || n_steps < 0) return go_fail(GO_ERR_INVALID, "bad arguments");
    int rc = batch_commit(b);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    for (int i = 0; i < n_steps; ++i) {
        rc = batch_launch(b, 0, s);
        if (rc) return rc;
        rc = batch_launch(b, 1, s);
        if (rc) return rc;
    }
    return GO_OK;
}

int go_batch_graph_capture(go_batch* b, void* stream, int n_steps) {
    if (!b || n_steps < 1) return go_fail(GO_ERR_INVALID, "bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (s == nullptr) return go_fail(GO_ERR_INVALID, "graph capture needs a non-default stream");
    int rc = batch_commit(b);
    if (rc) return rc;
    drop_graph(b);
    GO_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < n_steps && !rc; ++i) {
        rc = batch_launch(b, 0, s);
        if (!rc) rc = batch_launch(b, 1, s);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    b->graph = g;
    GO_CUDA(cudaGraphInstantiate(&b->graph_exec, g, 0));
    b->graph_steps = n_steps;
    return GO_OK;
}

int go_batch_graph_launch(go_batch* b, void* stream, int* steps_done) {
    GO_TRACE("go_batch_graph_launch");
    if (!b) return go_fail(GO_ERR_INVALID, "null batch");
    if (!b->graph_exec) return go_fail(GO_ERR_INVALID, "no captured graph (go_batch_graph_capture)");
    GO_CUDA(cudaGraphLaunch(b->graph_exec, (cudaStream_t)stream));
    if (steps_done) *steps_done = b->graph_steps;
    return GO_OK;
}

int go_batch_max_dt(go_batch* b, void* stream, float* dt_dev) {
    GO_TRACE("go_batch_max_dt");
    if (!b || !dt_dev) return go_fail(GO_ERR_INVALID, "null argument");
    int rc = batch_commit(b);
    if (rc) return rc;
    return launch_max_dt(b, (cudaStream_t)stream, reinterpret_cast<unsigned int*>(dt_dev));
}

int go_batch_status(go_batch* b, uint32_t* status_host, int clear) {
    if (!b || !status_host) return go_fail(GO_ERR_INVALID, "null argument");
    for (int m = 0; m < b->n; ++m) {
        int rc = go_domain_status(b->members[m], &status_host[m], clear);
        if (rc) return rc;
    }
    return GO_OK;
}

size_t go_batch_grf_scratch_floats(go_batch* b, float corr_cells) {
    GrfWeights W;
    if (!b || grf_weights(corr_cells, &W)) return 0;
    size_t total = 0;
    for (int m = 0; m < b->n; ++m) total += grf_member_scratch(b->members[m]->k.nx, b->members[m]->k.ny, W.R);
    return total;
}

int go_batch_grf_perturb(go_batch* b, void* stream, uint32_t key0, uint32_t event, float std_dev,
                         float corr_cells, float* scratch, size_t scratch_floats) {
    GO_TRACE("go_batch_grf_perturb");
    if (!b || !scratch) return go_fail(GO_ERR_INVALID, "null argument");
    int rc = batch_commit(b);
    if (rc) return rc;
    GrfWeights W;
    rc = grf_weights(corr_cells, &W);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    rc = grf_prepare(b, W);
    if (rc) return rc;
    if (scratch_floats < b->grf_scratch)
        return go_fail(GO_ERR_INVALID, "scratch holds %zu floats, the batch needs %zu", scratch_floats,
                       b->grf_scratch);
    GrfMember none;
    memset(&none, 0, sizeof(none));
    return grf_launch(b->d_grf, none, b->n, b->grf_max_nx, b->grf_max_ny, key0, event, std_dev, W, scratch, s);
}

int go_batch_run_events(go_batch* b, void* stream, uint32_t first_event, int n_events, double interval, float dt,
                        double courant, uint32_t key0, float std_dev, float corr_cells, float* scratch,
                        size_t scratch_floats, double* t_members, long long* steps_out, float* dt_out) {
    GO_TRACE("go_batch_run_events");
    if (!b || !scratch || !t_members) return go_fail(GO_ERR_INVALID, "null argument");
    if (n_events < 0 || !(interval > 0.0) || !(dt > 0.0f) || !(courant > 0.0))
        return go_fail(GO_ERR_INVALID, "n_events >= 0, interval > 0, dt > 0 and courant > 0");
    cudaStream_t s = (cudaStream_t)stream;
    if (s == nullptr) return go_fail(GO_ERR_INVALID, "the event loop needs a non-default stream");
    int rc = batch_commit(b);
    if (rc) return rc;
    GrfWeights W;
    rc = grf_weights(corr_cells, &W);
    if (rc) return rc;
    rc = grf_prepare(b, W);
    if (rc) return rc;
    if (scratch_floats < b->grf_scratch)
        return go_fail(GO_ERR_INVALID, "scratch holds %zu floats, the batch needs %zu", scratch_floats,
                       b->grf_scratch);
    if (steps_out) *steps_out = 0;
    if (dt_out) *dt_out = dt;
    if (n_events == 0) return GO_OK;
    if (!b->d_loop) {
        GO_CUDA(cudaMalloc(&b->d_loop, sizeof(EventLoop)));
        GO_CUDA(cudaMalloc(&b->d_t, sizeof(double) * b->n));
        GO_CUDA(cudaMalloc(&b->d_cfl, sizeof(unsigned int) * b->n));
        GO_CUDA(cudaStreamCreateWithFlags(&b->loop_side, cudaStreamNonBlocking));
    }
    EventLoopKey key;
    key.key0 = key0;
    key.std_dev = std_dev;
    key.corr_cells = corr_cells;
    key.scratch = scratch;
    key.valid = true;
    if (!(b->loop_key == key) || !b->loop_exec) {
        if (b->loop_exec) cudaGraphExecDestroy(b->loop_exec);
        if (b->loop_graph) cudaGraphDestroy(b->loop_graph);
        b->loop_exec = nullptr;
        b->loop_graph = nullptr;
        rc = build_event_graph(b, s, W, key0, std_dev, scratch);
        if (rc) return rc;
        b->loop_key = key;
    }
    EventLoop L;
    memset(&L, 0, sizeof(L));
    L.interval = interval;
    L.courant = courant;
    L.dt = dt;
    L.event = first_event;
    L.events_left = n_events;
    b->loop_t.assign(t_members, t_members + b->n);
    GO_CUDA(cudaMemcpyAsync(b->d_loop, &L, sizeof(L), cudaMemcpyHostToDevice, s));
    GO_CUDA(cudaMemcpyAsync(b->d_t, b->loop_t.data(), sizeof(double) * b->n, cudaMemcpyHostToDevice, s));
    GO_CUDA(cudaGraphLaunch(b->loop_exec, s));
    GO_CUDA(cudaMemcpyAsync(&L, b->d_loop, sizeof(L), cudaMemcpyDeviceToHost, s));
    GO_CUDA(cudaMemcpyAsync(b->loop_t.data(), b->d_t, sizeof(double) * b->n, cudaMemcpyDeviceToHost, s));
    GO_CUDA(cudaStreamSynchronize(s));
    std::copy(b->loop_t.begin(), b->loop_t.end(), t_members);
    for (int m = 0; m < b->n; ++m) {
        b->dt[m] = L.dt;
        b->args[2 * m].dt = L.dt;
        b->args[2 * m + 1].dt = L.dt;
    }
    if (steps_out) *steps_out = L.steps;
    if (dt_out) *dt_out = L.dt;
    return GO_OK;
}

}  // extern "C"
