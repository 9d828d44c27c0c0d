// go_cdklm_step_static: the RK2 step without any allocation.
//
// go_cdklm_step needs a go_domain handle, and go_domain_create allocates two
// small device buffers (the Coriolis row table and the status word) with
// cudaMalloc.  Some callers cannot allocate device memory: a host code that
// runs inside a pre-sized memory pool, a plugin that must not touch the
// allocator of the application that loaded it, a loop that may not block in
// cudaMalloc/cudaFree.  This entry point takes the scheme description
// directly and keeps both buffers in one file-scope __device__ array, so no
// call allocates anything: no cudaMalloc/cudaFree, no allocating library
// call, no torch.
//
// Limits and caveats:
//  * The array holds a Coriolis table of at most kNoAllocMaxRows = 16388
//    rows (ny <= 16384) plus the status word: 65,808 bytes per device,
//    resident for the life of the process.  Larger ny is rejected.
//  * The device address of the array comes from cudaGetSymbolAddress, looked
//    up on the first call made with each device current and then cached
//    together with the device's current context; a call that finds another
//    context current (after cudaDeviceReset, say) looks it up again.  That
//    lookup can load this library's device code into the context (lazy
//    module loading), which is not allowed inside stream capture: make the
//    first call on each device, and the first after a reset, outside any
//    capture (n_steps = 0 is enough).
//  * With a full Coriolis table (n_rows = ny + 4) the table is copied from
//    the caller's host memory with cudaMemcpyAsync on the call's stream;
//    from page-locked memory that copy runs after the call returns, so the
//    caller keeps the table unchanged until the stream has passed the call.
//  * The input's periodic ghost cells must be current: each stage refreshes
//    the ghosts of its own output, but nothing refreshes the input's before
//    the first stage (CDKLM16.step does that once at t = 0).
//  * Every call on one device shares the one array: calls that overlap in
//    time (different host threads, or different streams with no ordering
//    between them) race on the Coriolis table and the status word.  Order
//    them on one stream or serialise them on the host.
//  * Each call clears the status word and rewrites the whole table before
//    its launches, so nothing left by an earlier call is read.
#include <cudaTypedefs.h>

#include <mutex>

#include "pair_dispatch.cuh"

using namespace go;

namespace {

constexpr int kNoAllocMaxRows = 16388;  // ny + 4 for ny up to 16384
constexpr size_t kStatusOffset = 0;     // one uint32 status word
constexpr size_t kRowsOffset = 256;     // Coriolis table, ny + 4 floats
constexpr size_t kScratchBytes = kRowsOffset + sizeof(float) * kNoAllocMaxRows;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {nullptr};
CUcontext g_scratch_ctx[kMaxDevices] = {nullptr};   // context the cached address belongs to

// The calling thread's current context, through the driver entry point the
// runtime hands out (this library links the runtime only).
CUcontext current_context() {
    static PFN_cuCtxGetCurrent_v4000 get = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(fn);
    });
    CUcontext c = nullptr;
    if (get) get(&c);
    return c;
}

// Device address of the scratch array on the current device, looked up
// again when the device's context changed since the cached lookup.
int scratch_address(unsigned char** out) {
    int dev = -1;
    GO_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return go_fail(GO_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev] || g_scratch_ctx[dev] != current_context()) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);   // makes the context current
        if (e != cudaSuccess)
            return go_fail(GO_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch) failed: %s", cudaGetErrorString(e));
        g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
        g_scratch_ctx[dev] = current_context();
    }
    *out = g_scratch_ptr[dev];
    return GO_OK;
}

__global__ void k_fill_rows(float* rows, float value, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rows[i] = value;
}

// The checks and constants of go_domain_create, into a caller-owned
// go_domain (no allocation; the device pointers are set by the caller).
int fill_domain(const go_domain_desc& s, go_domain* d) {
    if (s.nx < 4 || s.ny < 4) return go_fail(GO_ERR_INVALID, "nx, ny must be >= 4 (got %d, %d)", s.nx, s.ny);
    if (!(s.dx > 0.0f) || !(s.dy > 0.0f) || !(s.g > 0.0f))
        return go_fail(GO_ERR_INVALID, "dx, dy, g must be positive");
    if (s.r < 0.0f) return go_fail(GO_ERR_INVALID, "friction r must be >= 0");
    if (s.rk_order != 2) return go_fail(GO_ERR_UNSUPPORTED, "rk_order %d: only 2 (Heun) is built", s.rk_order);
    const int bcs[4] = {s.bc_north, s.bc_east, s.bc_south, s.bc_west};
    for (int b : bcs)
        if (b != GO_BC_WALL && b != GO_BC_PERIODIC)
            return go_fail(GO_ERR_UNSUPPORTED, "boundary code %d: the allocation-free step takes wall (1) and "
                           "periodic (2) boundaries only", b);
    if ((s.bc_north == GO_BC_PERIODIC) != (s.bc_south == GO_BC_PERIODIC) ||
        (s.bc_east == GO_BC_PERIODIC) != (s.bc_west == GO_BC_PERIODIC))
        return go_fail(GO_ERR_INVALID, "periodic boundaries must be set on both opposite sides");
    if (s.friction_law != GO_FRICTION_QUADRATIC && s.friction_law != GO_FRICTION_LINEAR)
        return go_fail(GO_ERR_INVALID, "unknown friction law %d", s.friction_law);
    memset(d, 0, sizeof(*d));
    d->desc = s;
    Scheme& k = d->k;
    k.nx = s.nx; k.ny = s.ny;
    k.dx = s.dx; k.dy = s.dy; k.g = s.g; k.r = s.r; k.theta = s.theta;
    k.desing_eps = s.desing_eps; k.flux_slope_eps = s.flux_slope_eps; k.cutoff = s.depth_cutoff;
    k.land = 1.0e20f;
    k.nX = s.north_x; k.nY = s.north_y;
    k.bcN = s.bc_north; k.bcE = s.bc_east; k.bcS = s.bc_south; k.bcW = s.bc_west;
    volatile float g = s.g, two = 2.0f, half = 0.5f;  // folded in IEEE float32, as go_domain_create does
    k.two_g = two * g;
    k.half_g = half * g;
    k.theta_g = s.theta * g;
    k.V = s.dx / k.two_g;
    k.U = s.dy / k.two_g;
    k.two_r = two * s.r;
    d->shape = go_auto_shape(s.nx, s.ny);
    d->rows_per_block = go_auto_rows(s.nx, s.ny, d->shape);
    d->arith = GO_ARITH_RCP;
    d->has_land = 1;
    return GO_OK;
}

}  // namespace

extern "C" int go_cdklm_step_static(const go_domain_desc* desc, void* stream, const float* f_rows_host,
                                    int n_rows, float wind_x, float wind_y, int n_steps, float dt,
                                    float* eta0, float* hu0, float* hv0, int pitch0,
                                    float* eta1, float* hu1, float* hv1, int pitch1,
                                    const float* Hi, int Hi_pitch, float land_value, uint32_t* status_out) {
    if (!desc || !f_rows_host || !eta0 || !hu0 || !hv0 || !eta1 || !hu1 || !hv1 || !Hi)
        return go_fail(GO_ERR_INVALID, "null argument");
    go_domain d;
    int rc = fill_domain(*desc, &d);
    if (rc) return rc;
    if (desc->ny + 4 > kNoAllocMaxRows)
        return go_fail(GO_ERR_INVALID, "ny = %d exceeds the static scratch of the no-allocation step "
                       "(ny + 4 <= %d)", desc->ny, kNoAllocMaxRows);
    if (n_rows != 1 && n_rows != desc->ny + 4)
        return go_fail(GO_ERR_INVALID, "Coriolis table has %d rows, need 1 or ny+4 = %d", n_rows, desc->ny + 4);
    if (n_steps < 0) return go_fail(GO_ERR_INVALID, "n_steps < 0");
    rc = go_check_pitch(pitch0, desc->nx + 4, "h0");
    if (!rc) rc = go_check_pitch(pitch1, desc->nx + 4, "h1");
    if (!rc) rc = go_check_pitch(Hi_pitch, desc->nx + 5, "Hi");
    if (rc) return rc;

    unsigned char* scratch = nullptr;
    rc = scratch_address(&scratch);
    if (rc) return rc;
    unsigned int* status = reinterpret_cast<unsigned int*>(scratch + kStatusOffset);
    float* rows = reinterpret_cast<float*>(scratch + kRowsOffset);
    cudaStream_t s = (cudaStream_t)stream;

    GO_CUDA(cudaMemsetAsync(status, 0, sizeof(unsigned int), s));
    if (n_rows == 1) {
        k_fill_rows<<<(desc->ny + 4 + 255) / 256, 256, 0, s>>>(rows, f_rows_host[0], desc->ny + 4);
        GO_CUDA(cudaGetLastError());
    } else {
        GO_CUDA(cudaMemcpyAsync(rows, f_rows_host, sizeof(float) * n_rows, cudaMemcpyHostToDevice, s));
    }

    d.d_frows = rows;
    d.d_status = status;
    d.wxc = d.wxn = wind_x;
    d.wyc = d.wyn = wind_y;
    const StageArgs a0 = go_stage_args(&d, dt, 0, eta0, hu0, hv0, pitch0 / 4, eta1, hu1, hv1, pitch1 / 4, Hi,
                                       Hi_pitch / 4, land_value, 0.0f);
    const StageArgs a1 = go_stage_args(&d, dt, 1, eta1, hu1, hv1, pitch1 / 4, eta0, hu0, hv0, pitch0 / 4, Hi,
                                       Hi_pitch / 4, land_value, 0.0f);
    PreparedStage p0, p1;
    rc = go_prepare_stage(&d, a0, &p0);
    if (!rc) rc = go_prepare_stage(&d, a1, &p1);
    if (rc) return rc;
    for (int n = 0; n < n_steps; ++n) {
        rc = go_launch_prepared(&d, s, p0);
        if (rc) return rc;
        rc = go_launch_prepared(&d, s, p1);
        if (rc) return rc;
    }
    if (status_out) {
        GO_CUDA(cudaMemcpyAsync(status_out, status, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
        GO_CUDA(cudaStreamSynchronize(s));
    }
    return GO_OK;
}
