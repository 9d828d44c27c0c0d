// C ABI of the B200-native CDKLM16 step (declarations in include/gocean.h).
//
// Build: gpu-ocean_b200/build.py compiles every csrc/*.cu for sm_100a with
// the reference's floating-point flags (CDKLM16.py:196-200):
// --ftz=true --prec-div=false --prec-sqrt=false --fmad=false.
#include <string>

#include "pair_dispatch.cuh"
#include "trace.h"

using namespace go;

static thread_local std::string g_err;

int go_fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int go_check_pitch(int pitch_bytes, int min_floats, const char* what) {
    if (pitch_bytes <= 0 || (pitch_bytes % 4) != 0 || pitch_bytes / 4 < min_floats)
        return go_fail(GO_ERR_INVALID, "%s pitch %d bytes is invalid (need a multiple of 4, >= %d floats)",
                       what, pitch_bytes, min_floats);
    return GO_OK;
}

// Rows per block strip.  A block's cost is about (rows + 4) row steps: it
// recomputes the 4 rows above and below its strip before its first output
// row.  The strip height r in {2, 4, 8, 16, 24} minimises
//   ceil(blocks(r) / (148 SMs x resident blocks per SM)) x (r + 4),
// whole waves of blocks times the length of one block, taking the taller
// strip on a tie.  Measured on a B200 (us per RK2 step, default shape):
// 1024^2 picks 16 (66; 8 rows: 70), 4096^2 picks 24 (720; 16 rows: 727).
int go_auto_rows(int nx, int ny, int shape) {
    const int useful = go::shape_block_width(shape) - 4;
    const long long strips = (nx + useful - 1) / useful;
    const long long slots = 148LL * go::shape_blocks_per_sm(shape);
    static const int kRows[] = {2, 4, 8, 16, 24};
    // column-pair shapes: heights in whole ring chunks of 3 rows; priming a
    // strip costs about 2 rows
    static const int kPairRows[] = {3, 6, 12, 24, 36, 48, 72, 96};
    const bool pair = go_pair_shape(shape);
    const int* rows = pair ? kPairRows : kRows;
    const int n = pair ? 8 : 5;
    const int extra = pair ? 2 : 4;
    int best = rows[0];
    long long best_cost = -1;
    for (int i = 0; i < n; ++i) {
        const int r = rows[i];
        const long long blocks = strips * ((ny + r - 1) / r);
        const long long cost = ((blocks + slots - 1) / slots) * (r + extra);
        if (best_cost < 0 || cost <= best_cost) { best = r; best_cost = cost; }
    }
    return best;
}

// Default launch shape: the column-pair kernel (shape 8) from about 1500^2
// cells up (measured on a B200, us per step, shapes 4 / 5 / 8, walls N/S and
// periodic E/W: 1536^2 126 / 128 / 118, 2048^2 208 / 203 / 200, 2560^2
// 308 / 292 / 262, 3072^2 429 / 399 / 373, 4096^2 720 / 686 / 583; at
// 1024^2 and below the pair kernel's separate boundary-frame launch does not
// pay: 68 / 72 / 71 and 29 / 32 / 36 at 512^2).  Below that a read-ahead shape (5,
// or 6 for widths that 96-wide blocks cover with less waste) once the grid
// needs more than one wave of blocks, where the ring hides the load
// latency; in a single wave the register prefetch of 128 x 5 blocks
// (shape 4) is faster (1024^2 and below lose 6-9% with the ring).
int go_auto_shape(int nx, int ny) {
    if ((long long)nx * ny >= kPairAutoCells) return GO_SHAPE_PAIR;
    const int ring = go::ring_shape(go::shape_columns(5, nx), go::shape_columns(6, nx));
    const int rows = go_auto_rows(nx, ny, ring);
    const long long blocks = go::shape_columns(ring, nx) / go::shape_block_width(ring) * ((ny + rows - 1) / rows);
    return blocks > 148LL * go::shape_blocks_per_sm(ring) ? ring : 4;
}

int go_friction_mode(const go_domain* d) {
    if (d->desc.friction_law == GO_FRICTION_LINEAR) return kFricLinear;
    return (d->k.r > 0.0f) ? kFricQuad : kFricNone;
}

bool go_general_north(const go_domain* d) { return !(d->k.nX == 0.0f && d->k.nY == 1.0f); }


StageArgs go_stage_args(const go_domain* d, float dt, int rk_step, const float* e0, const float* u0,
                        const float* v0, int pin, float* e1, float* u1, float* v1, int pout,
                        const float* Hi, int phi, float land, float wind_t) {
    StageArgs a;
    memset(&a, 0, sizeof(a));
    a.k = d->k;
    a.k.land = land;
    a.dt = dt;
    a.rk_step = rk_step;
    a.eta_in = e0; a.hu_in = u0; a.hv_in = v0; a.pin = pin;
    a.eta_out = e1; a.hu_out = u1; a.hv_out = v1; a.pout = pout;
    a.qn_eta = e1; a.qn_hu = u1; a.qn_hv = v1; a.pqn = pout;
    a.Hi = Hi; a.phi = phi;
    a.f_rows = d->d_frows;
    a.wind_t = wind_t;
    a.wxc = d->wxc; a.wxn = d->wxn; a.wyc = d->wyc; a.wyn = d->wyn;
    a.wx_cur = d->wx_cur; a.wx_next = d->wx_next; a.wy_cur = d->wy_cur; a.wy_next = d->wy_next;
    a.pw = d->wpitch;
    a.rows_per_block = d->rows_per_block;
    a.status = d->d_status;
    a.debug = d->debug;
    a.neg_zero = -0.0f;
    a.fric = go_friction_mode(d);
    return a;
}

// ---------------------------------------------------------------------------
// Bathymetry set-up kernels (boundary_kernels.cu:121-246, initBm_kernel.cu:38)
// ---------------------------------------------------------------------------

__global__ void k_bi_corners_ns(float* Hi, int p, int nx, int ny, int periodic) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > nx + 4) return;
    if (periodic) {
        for (int j = 0; j < 2; ++j) Hi[(size_t)j * p + i] = Hi[(size_t)(j + ny) * p + i];
        for (int j = ny + 2; j <= ny + 4; ++j) Hi[(size_t)j * p + i] = Hi[(size_t)(j - ny) * p + i];
    } else {
        for (int j = 0; j < 2; ++j) Hi[(size_t)j * p + i] = Hi[(size_t)(4 - j) * p + i];
        for (int j = 0; j < 2; ++j) Hi[(size_t)(ny + 4 - j) * p + i] = Hi[(size_t)(ny + j) * p + i];
    }
}

__global__ void k_bi_corners_ew(float* Hi, int p, int nx, int ny, int periodic) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j > ny + 4) return;
    float* row = Hi + (size_t)j * p;
    if (periodic) {
        for (int i = 0; i < 2; ++i) row[i] = row[i + nx];
        for (int i = nx + 2; i <= nx + 4; ++i) row[i] = row[i - nx];
    } else {
        for (int i = 0; i < 2; ++i) row[i] = row[4 - i];
        for (int i = 0; i < 2; ++i) row[nx + 4 - i] = row[nx + i];
    }
}

__global__ void k_init_bm(const float* Hi, int ph, float* Bm, int pb, int nx, int ny, float land) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx + 4 || j >= ny + 4) return;
    Bm[(size_t)j * pb + i] = cell_mean_depth(Hi[(size_t)j * ph + i], Hi[(size_t)(j + 1) * ph + i],
                                             Hi[(size_t)j * ph + i + 1], Hi[(size_t)(j + 1) * ph + i + 1], land);
}

// ---------------------------------------------------------------------------
// Periodic ghost refresh (boundary_kernels.cu:35-110): NS, then EW.
// ---------------------------------------------------------------------------

__global__ void k_periodic_ns(float* e, float* u, float* v, int p, int nx, int ny) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;  // ghost row index 0..3
    if (i > nx + 3) return;
    const int j = (g < 2) ? g : ny + g;          // 0, 1, ny+2, ny+3
    const int src = (g < 2) ? j + ny : j - ny;
    const size_t o = (size_t)j * p + i, s = (size_t)src * p + i;
    e[o] = e[s]; u[o] = u[s]; v[o] = v[s];
}

__global__ void k_periodic_ew(float* e, float* u, float* v, int p, int nx, int ny) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;
    if (j > ny + 3) return;
    const int i = (g < 2) ? g : nx + g;
    const int src = (g < 2) ? i + nx : i - nx;
    const size_t o = (size_t)j * p + i, s = (size_t)j * p + src;
    e[o] = e[s]; u[o] = u[s]; v[o] = v[s];
}

// ---------------------------------------------------------------------------
// CFL limit (max_dt.cu:42-141), exact minimum over all interior cells.
// ---------------------------------------------------------------------------

__global__ void k_max_dt(const float* eta, const float* hu, const float* hv, int p,
                         const float* Bm, int pb, int nx, int ny, float dx, float dy, float g,
                         float land, unsigned int* out) {
    float best = kRefFltMax;
    const int n = nx * ny;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
        const int j = idx / nx + 2, i = idx % nx + 2;
        const size_t o = (size_t)j * p + i;
        best = fminf(best, cell_cfl_dt(eta[o], hu[o], hv[o], Bm[(size_t)j * pb + i], dx, dy, g, land, kRefFltMax));
    }
    block_min_to(best, out, kRefFltMax);
}

__global__ void k_fill_u32(unsigned int* p, unsigned int v) { *p = v; }

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

const char* go_last_error(void) { return g_err.c_str(); }
const char* go_version(void) { return "gocean-b200 0.1 (sm_100a)"; }

int go_domain_create(const go_domain_desc* desc, go_domain** out) {
    if (!desc || !out) return go_fail(GO_ERR_INVALID, "null argument");
    *out = nullptr;
    const go_domain_desc& s = *desc;
    if (s.nx < 4 || s.ny < 4) return go_fail(GO_ERR_INVALID, "nx, ny must be >= 4 (got %d, %d)", s.nx, s.ny);
    if (!(s.dx > 0.0f) || !(s.dy > 0.0f) || !(s.g > 0.0f))
        return go_fail(GO_ERR_INVALID, "dx, dy, g must be positive");
    if (s.r < 0.0f) return go_fail(GO_ERR_INVALID, "friction r must be >= 0");
    if (s.rk_order != 2) return go_fail(GO_ERR_UNSUPPORTED, "rk_order %d: only 2 (Heun) is built", s.rk_order);
    const int bcs[4] = {s.bc_north, s.bc_east, s.bc_south, s.bc_west};
    for (int b : bcs)
        if (b < GO_BC_WALL || b > GO_BC_LINEAR_SPONGE)
            return go_fail(GO_ERR_UNSUPPORTED, "boundary code %d: wall (1), periodic (2), flow relaxation (3) "
                           "and linear sponge (4) are built", b);
    if ((s.bc_north == GO_BC_PERIODIC) != (s.bc_south == GO_BC_PERIODIC) ||
        (s.bc_east == GO_BC_PERIODIC) != (s.bc_west == GO_BC_PERIODIC))
        return go_fail(GO_ERR_INVALID, "periodic boundaries must be set on both opposite sides");
    if (s.friction_law != GO_FRICTION_QUADRATIC && s.friction_law != GO_FRICTION_LINEAR)
        return go_fail(GO_ERR_INVALID, "unknown friction law %d", s.friction_law);

    go_domain* d = new go_domain();
    d->own_side = 1;
    d->desc = s;
    Scheme& k = d->k;
    k.nx = s.nx; k.ny = s.ny;
    k.dx = s.dx; k.dy = s.dy; k.g = s.g; k.r = s.r; k.theta = s.theta;
    k.desing_eps = s.desing_eps; k.flux_slope_eps = s.flux_slope_eps; k.cutoff = s.depth_cutoff;
    k.land = 1.0e20f;
    k.nX = s.north_x; k.nY = s.north_y;
    k.bcN = s.bc_north; k.bcE = s.bc_east; k.bcS = s.bc_south; k.bcW = s.bc_west;
    // constants the reference folds at compile time (IEEE float32 on the host)
    volatile float g = s.g, two = 2.0f, half = 0.5f;
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
    cudaError_t e = cudaGetDevice(&d->device);
    if (e == cudaSuccess) e = cudaMalloc(&d->d_frows, sizeof(float) * (s.ny + 4));
    if (e == cudaSuccess) e = cudaMemset(d->d_frows, 0, sizeof(float) * (s.ny + 4));
    if (e == cudaSuccess) e = cudaMalloc(&d->d_status, sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemset(d->d_status, 0, sizeof(unsigned int));
    if (e != cudaSuccess) {
        cudaFree(d->d_frows);
        cudaFree(d->d_status);
        delete d;
        return go_fail(GO_ERR_CUDA, "domain allocation failed: %s", cudaGetErrorString(e));
    }
    *out = d;
    return GO_OK;
}

int go_domain_destroy(go_domain* d) {
    if (!d) return GO_OK;
    if (d->side) cudaStreamDestroy(d->side);
    if (d->ev_fork) cudaEventDestroy(d->ev_fork);
    if (d->ev_join) cudaEventDestroy(d->ev_join);
    cudaFree(d->d_frows);
    cudaFree(d->d_status);
    delete d;
    return GO_OK;
}

int go_domain_set_coriolis(go_domain* d, const float* f_rows_host, int n) {
    if (!d || !f_rows_host) return go_fail(GO_ERR_INVALID, "null argument");
    const int rows = d->k.ny + 4;
    if (n == 1) {
        float* tmp = new float[rows];
        for (int j = 0; j < rows; ++j) tmp[j] = f_rows_host[0];
        cudaError_t e = cudaMemcpy(d->d_frows, tmp, sizeof(float) * rows, cudaMemcpyHostToDevice);
        delete[] tmp;
        GO_CUDA(e);
        return GO_OK;
    }
    if (n != rows) return go_fail(GO_ERR_INVALID, "Coriolis table has %d rows, need 1 or ny+4 = %d", n, rows);
    GO_CUDA(cudaMemcpy(d->d_frows, f_rows_host, sizeof(float) * rows, cudaMemcpyHostToDevice));
    return GO_OK;
}

int go_domain_set_wind_uniform(go_domain* d, float x_cur, float x_next, float y_cur, float y_next) {
    if (!d) return go_fail(GO_ERR_INVALID, "null domain");
    d->wxc = x_cur; d->wxn = x_next; d->wyc = y_cur; d->wyn = y_next;
    d->wx_cur = d->wx_next = d->wy_cur = d->wy_next = nullptr;
    return GO_OK;
}

int go_domain_set_wind_field(go_domain* d, const float* x_cur, const float* x_next,
                             const float* y_cur, const float* y_next, int pitch) {
    if (!d) return go_fail(GO_ERR_INVALID, "null domain");
    if (!x_cur && !x_next && !y_cur && !y_next) {
        d->wx_cur = d->wx_next = d->wy_cur = d->wy_next = nullptr;
        return GO_OK;
    }
    if (!x_cur || !x_next || !y_cur || !y_next) return go_fail(GO_ERR_INVALID, "wind field needs four arrays");
    int rc = go_check_pitch(pitch, d->k.nx, "wind");
    if (rc) return rc;
    d->wx_cur = x_cur; d->wx_next = x_next; d->wy_cur = y_cur; d->wy_next = y_next;
    d->wpitch = pitch / 4;
    return GO_OK;
}

int go_domain_set_launch(go_domain* d, int shape, int rows_per_block) {
    if (!d) return go_fail(GO_ERR_INVALID, "null domain");
    if (shape < 0 || shape > GO_SHAPE_PAIR) return go_fail(GO_ERR_INVALID, "launch shape %d (0..8)", shape);
    if (rows_per_block == 0) rows_per_block = go_auto_rows(d->k.nx, d->k.ny, shape);
    if (rows_per_block < 1) return go_fail(GO_ERR_INVALID, "rows_per_block must be >= 1");
    d->shape = shape;
    d->rows_per_block = rows_per_block;
    return GO_OK;
}

int go_domain_set_arith(go_domain* d, int mode) {
    if (!d) return go_fail(GO_ERR_INVALID, "null domain");
    if (mode != GO_ARITH_EXACT && mode != GO_ARITH_RCP) return go_fail(GO_ERR_INVALID, "arith mode %d", mode);
    d->arith = mode;
    return GO_OK;
}

int go_domain_set_land(go_domain* d, int may_have_land) {
    if (!d) return go_fail(GO_ERR_INVALID, "null domain");
    d->has_land = may_have_land ? 1 : 0;
    return GO_OK;
}

int go_init_bathymetry(go_domain* d, void* stream, float* Hi, int Hi_pitch, float* Bm, int Bm_pitch,
                       float land_value) {
    if (!d || !Hi || !Bm) return go_fail(GO_ERR_INVALID, "null argument");
    int rc = go_check_pitch(Hi_pitch, d->k.nx + 5, "Hi");
    if (rc) return rc;
    rc = go_check_pitch(Bm_pitch, d->k.nx + 4, "Bm");
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int nx = d->k.nx, ny = d->k.ny, ph = Hi_pitch / 4, pb = Bm_pitch / 4;
    k_bi_corners_ns<<<(nx + 5 + 127) / 128, 128, 0, s>>>(Hi, ph, nx, ny, d->k.bcN == GO_BC_PERIODIC);
    k_bi_corners_ew<<<(ny + 5 + 127) / 128, 128, 0, s>>>(Hi, ph, nx, ny, d->k.bcE == GO_BC_PERIODIC);
    dim3 b(32, 8), g((nx + 4 + 31) / 32, (ny + 4 + 7) / 8);
    k_init_bm<<<g, b, 0, s>>>(Hi, ph, Bm, pb, nx, ny, land_value);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

int go_boundary_condition(go_domain* d, void* stream, float* eta, float* hu, float* hv, int pitch) {
    if (!d || !eta || !hu || !hv) return go_fail(GO_ERR_INVALID, "null argument");
    int rc = go_check_pitch(pitch, d->k.nx + 4, "state");
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int nx = d->k.nx, ny = d->k.ny, p = pitch / 4;
    // north-south (periodic copy, or the open kinds), then east-west
    if (d->k.bcN == GO_BC_PERIODIC) {
        k_periodic_ns<<<dim3((nx + 4 + 127) / 128, 4), 128, 0, s>>>(eta, hu, hv, p, nx, ny);
    } else {
        rc = go_open_bc_ns(d, s, eta, hu, hv, p);
        if (rc) return rc;
    }
    if (d->k.bcE == GO_BC_PERIODIC) {
        k_periodic_ew<<<dim3((ny + 4 + 127) / 128, 4), 128, 0, s>>>(eta, hu, hv, p, nx, ny);
    } else {
        rc = go_open_bc_ew(d, s, eta, hu, hv, p);
        if (rc) return rc;
    }
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

static int pack_bc(const Scheme& k) { return (k.bcN << 24) | (k.bcS << 16) | (k.bcE << 8) | k.bcW; }

int go_cdklm_swe_2D(go_domain* d, void* stream, float dt, int rk_step,
                    const float* eta0, int eta0_pitch, const float* hu0, int hu0_pitch,
                    const float* hv0, int hv0_pitch,
                    float* eta1, int eta1_pitch, float* hu1, int hu1_pitch,
                    float* hv1, int hv1_pitch,
                    const float* Hi, int Hi_pitch, const float* Hm, int Hm_pitch,
                    float land_value, float wind_stress_t, int boundary_conditions) {
    GO_TRACE("go_cdklm_swe_2D");
    (void)Hm; (void)Hm_pitch;
    if (!d || !eta0 || !hu0 || !hv0 || !eta1 || !hu1 || !hv1 || !Hi)
        return go_fail(GO_ERR_INVALID, "null argument");
    if (rk_step != 0 && rk_step != 1) return go_fail(GO_ERR_INVALID, "rk_step %d (RK2 has 0 and 1)", rk_step);
    if (eta0_pitch != hu0_pitch || eta0_pitch != hv0_pitch || eta1_pitch != hu1_pitch ||
        eta1_pitch != hv1_pitch)
        return go_fail(GO_ERR_INVALID, "eta/hu/hv of one state must share a pitch");
    if (boundary_conditions != pack_bc(d->k))
        return go_fail(GO_ERR_INVALID, "packed boundary code 0x%08x does not match the domain's 0x%08x",
                    boundary_conditions, pack_bc(d->k));
    int rc = go_check_pitch(eta0_pitch, d->k.nx + 4, "input");
    if (!rc) rc = go_check_pitch(eta1_pitch, d->k.nx + 4, "output");
    if (!rc) rc = go_check_pitch(Hi_pitch, d->k.nx + 5, "Hi");
    if (rc) return rc;
    const StageArgs a = go_stage_args(d, dt, rk_step, eta0, hu0, hv0, eta0_pitch / 4, eta1, hu1, hv1,
                                      eta1_pitch / 4, Hi, Hi_pitch / 4, land_value, wind_stress_t);
    return go_launch_stage(d, (cudaStream_t)stream, a);
}

int go_cdklm_step(go_domain* d, void* stream, int n_steps, float dt, float wind_stress_t,
                  float* eta0, float* hu0, float* hv0, int pitch0,
                  float* eta1, float* hu1, float* hv1, int pitch1,
                  const float* Hi, int Hi_pitch, float land_value) {
    GO_TRACE("go_cdklm_step");
    if (!d || !eta0 || !hu0 || !hv0 || !eta1 || !hu1 || !hv1 || !Hi)
        return go_fail(GO_ERR_INVALID, "null argument");
    if (n_steps < 0) return go_fail(GO_ERR_INVALID, "n_steps < 0");
    int rc = go_check_pitch(pitch0, d->k.nx + 4, "h0");
    if (!rc) rc = go_check_pitch(pitch1, d->k.nx + 4, "h1");
    if (!rc) rc = go_check_pitch(Hi_pitch, d->k.nx + 5, "Hi");
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const StageArgs a0 = go_stage_args(d, dt, 0, eta0, hu0, hv0, pitch0 / 4, eta1, hu1, hv1, pitch1 / 4, Hi,
                                       Hi_pitch / 4, land_value, wind_stress_t);
    const StageArgs a1 = go_stage_args(d, dt, 1, eta1, hu1, hv1, pitch1 / 4, eta0, hu0, hv0, pitch0 / 4, Hi,
                                       Hi_pitch / 4, land_value, wind_stress_t);
    const bool open = go_has_open_bc(d);
    PreparedStage p0, p1;
    rc = go_prepare_stage(d, a0, &p0);
    if (!rc) rc = go_prepare_stage(d, a1, &p1);
    if (rc) return rc;
    for (int n = 0; n < n_steps; ++n) {
        rc = go_launch_prepared(d, s, p0);
        // open boundaries: the reference's ghost sequence after each stage
        // (CDKLM16.py:537-540, 585-586); the stage kernel's own periodic
        // images are redone in order after the open kinds of the other axis
        if (!rc && open) rc = go_boundary_condition(d, stream, eta1, hu1, hv1, pitch1);
        if (rc) return rc;
        rc = go_launch_prepared(d, s, p1);
        if (!rc && open) rc = go_boundary_condition(d, stream, eta0, hu0, hv0, pitch0);
        if (rc) return rc;
    }
    return GO_OK;
}

int go_max_dt(go_domain* d, void* stream, const float* eta, const float* hu, const float* hv, int pitch,
              const float* Bm, int Bm_pitch, float land_value, float* dt_dev) {
    GO_TRACE("go_max_dt");
    if (!d || !eta || !hu || !hv || !Bm || !dt_dev) return go_fail(GO_ERR_INVALID, "null argument");
    int rc = go_check_pitch(pitch, d->k.nx + 4, "state");
    if (!rc) rc = go_check_pitch(Bm_pitch, d->k.nx + 4, "Bm");
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned int* out = reinterpret_cast<unsigned int*>(dt_dev);
    unsigned int init_bits;
    memcpy(&init_bits, &kRefFltMax, sizeof(init_bits));
    k_fill_u32<<<1, 1, 0, s>>>(out, init_bits);
    const int n = d->k.nx * d->k.ny;
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_max_dt<<<blocks, 256, 0, s>>>(eta, hu, hv, pitch / 4, Bm, Bm_pitch / 4, d->k.nx, d->k.ny, d->k.dx,
                                     d->k.dy, d->k.g, land_value, out);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

int go_domain_status(go_domain* d, uint32_t* status, int clear) {
    if (!d || !status) return go_fail(GO_ERR_INVALID, "null argument");
    unsigned int v = 0;
    GO_CUDA(cudaMemcpy(&v, d->d_status, sizeof(v), cudaMemcpyDeviceToHost));
    *status = v;
    if (clear) GO_CUDA(cudaMemset(d->d_status, 0, sizeof(unsigned int)));
    return GO_OK;
}

int go_domain_set_debug(go_domain* d, unsigned flags) {
    if (!d) return go_fail(GO_ERR_INVALID, "null domain");
    if (flags & ~GO_DEBUG_SKIP_TMA) return go_fail(GO_ERR_INVALID, "unknown debug flags 0x%x", flags);
    d->debug = flags;
    return GO_OK;
}

int go_domain_stage_launches(go_domain* d, int* launches) {
    if (!d || !launches) return go_fail(GO_ERR_INVALID, "null argument");
    *launches = d->stage_launches;
    return GO_OK;
}

}  // extern "C"
