// Additive model error: seeded Gaussian random fields added to eta.
//
// The batched-ensemble workload perturbs every member's surface elevation by
// a correlated Gaussian field every 60 s of model time (and once at t = 0).
// The field is built from counter-based normals, so that member m's field at
// event e is the same number whether the members are stepped one by one or in
// one batched launch:
//
//   * Philox4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers:
//     as easy as 1, 2, 3", SC'11): key (key0, key1), counter (group, event,
//     0, 0) where group = linear index / 4 on the noise grid; its four 32-bit
//     words give four normals by the Box-Muller transform on 23-bit uniforms
//     u = (2 floor(x / 2^9) + 1) / 2^24, which lie strictly inside (0, 1).
//   * A separable Gaussian filter exp(-d^2 / (2 s^2)), s = L / sqrt(2) for a
//     field correlation exp(-r^2 / (2 L^2)), truncated at R = ceil(3 s) and
//     scaled so that the sum of squared weights is 1 (unit variance in 2-D).
//   * The noise grid is nx wide (the field is periodic in x) and ny + 2R high;
//     with periodic north/south boundaries its rows wrap too.
//
// No counterpart kernel in the reference (its OceanStateNoise draws its model
// error differently); the generator is this project's model-error term.
#include "grf.cuh"

using namespace go;

namespace {

constexpr uint32_t kPhiloxM0 = 0xD2511F53u, kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u, kPhiloxW1 = 0xBB67AE85u;
constexpr int kChunk = 1024;            // x-filter columns per block

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = kPhiloxM0 * c.x, hi0 = __umulhi(kPhiloxM0, c.x);
        const uint32_t lo1 = kPhiloxM1 * c.z, hi1 = __umulhi(kPhiloxM1, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += kPhiloxW0;
        k.y += kPhiloxW1;
    }
    return c;
}

__device__ __forceinline__ float unit_open(uint32_t x) {
    return (float)(2u * (x >> 9) + 1u) * 5.9604644775390625e-8f;   // 2^-24
}

// Normal number at linear index l of the noise grid.
__device__ __forceinline__ float grf_normal(uint32_t l, uint32_t event, uint2 key) {
    const uint4 r = philox4x32_10(make_uint4(l >> 2, event, 0u, 0u), key);
    const int lane = l & 3;
    const uint32_t a = (lane < 2) ? r.x : r.z;
    const uint32_t b = (lane < 2) ? r.y : r.w;
    const float rad = sqrtf(-2.0f * logf(unit_open(a)));
    float s, c;
    sincospif(2.0f * unit_open(b), &s, &c);
    return rad * ((lane & 1) ? s : c);
}

// x pass: one block per (noise row, chunk of kChunk columns); the normals of
// the chunk plus R columns either side (periodic in x) in shared memory.
__global__ void k_grf_xpass(const GrfMember* __restrict__ members, const GrfMember single, uint32_t key0,
                            uint32_t event_arg, const uint32_t* __restrict__ event_dev, float* __restrict__ scratch,
                            const GrfWeights W) {
    __shared__ float row[kChunk + kGrfMaxTaps];
    const GrfMember M = members ? members[blockIdx.z] : single;
    const uint32_t event = event_dev ? *event_dev : event_arg;
    const int R = W.R;
    const int yext = blockIdx.y;
    const int x0 = blockIdx.x * kChunk;
    if (yext >= M.ny + 2 * R || x0 >= M.nx) return;
    const int grow = M.periodic_y ? R + ((yext - R) % M.ny + M.ny) % M.ny : yext;
    const uint2 key = make_uint2(key0, M.key1);
    const int w = min(kChunk, M.nx - x0);
    for (int t = threadIdx.x; t < w + 2 * R; t += blockDim.x) {
        const int x = ((x0 - R + t) % M.nx + M.nx) % M.nx;
        row[t] = grf_normal((uint32_t)grow * (uint32_t)M.nx + (uint32_t)x, event, key);
    }
    __syncthreads();
    float* tmp = scratch + M.tmp_off;
    for (int t = threadIdx.x; t < w; t += blockDim.x) {
        float acc = 0.0f;
        for (int d = 0; d <= 2 * R; ++d) acc += W.w[d] * row[t + d];
        tmp[(size_t)yext * M.nx + x0 + t] = acc;
    }
}

// y pass: eta += std * field at each interior cell; the periodic ghost
// images of the changed cells are rewritten.  One block per 32 columns x
// kYTile rows: the block's x-filtered noise column strip (kYTile + 2R rows)
// is staged in shared memory once, instead of each output reading its 2R+1
// taps from global memory.
constexpr int kYTile = 64;
__global__ void k_grf_ypass(const GrfMember* __restrict__ members, const GrfMember single, float std_dev,
                            const float* __restrict__ scratch, const GrfWeights W) {
    __shared__ float strip[(kYTile + kGrfMaxTaps - 1) * 32];
    const GrfMember M = members ? members[blockIdx.z] : single;
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y0 = blockIdx.y * kYTile;
    if (y0 >= M.ny || (int)blockIdx.x * 32 >= M.nx) return;      // whole block
    const float* tmp = scratch + M.tmp_off;
    const int rows = min(kYTile, M.ny - y0) + 2 * W.R;             // <= ny + 2R - y0
    for (int r = threadIdx.y; r < rows; r += blockDim.y)
        strip[r * 32 + threadIdx.x] = (x < M.nx) ? tmp[(size_t)(y0 + r) * M.nx + x] : 0.0f;
    __syncthreads();
    if (x >= M.nx) return;
    for (int yy = threadIdx.y; yy < kYTile && y0 + yy < M.ny; yy += blockDim.y) {
        float acc = 0.0f;
        for (int d = 0; d <= 2 * W.R; ++d) acc += W.w[d] * strip[(yy + d) * 32 + threadIdx.x];
        const int j = y0 + yy + 2, i = x + 2;
        const float v = M.eta[(size_t)j * M.pitch + i] + std_dev * acc;
        M.eta[(size_t)j * M.pitch + i] = v;
        const int rows_img[2] = {j, M.periodic_y ? ((j < 4) ? j + M.ny : (j >= M.ny ? j - M.ny : -1)) : -1};
        const int cols_img[2] = {i, M.periodic_x ? ((i < 4) ? i + M.nx : (i >= M.nx ? i - M.nx : -1)) : -1};
        for (int a2 = 0; a2 < 2; ++a2)
            for (int b2 = 0; b2 < 2; ++b2)
                if ((a2 || b2) && rows_img[a2] >= 0 && cols_img[b2] >= 0)
                    M.eta[(size_t)rows_img[a2] * M.pitch + cols_img[b2]] = v;
    }
}

}  // namespace

namespace go {

int grf_weights(float corr_cells, GrfWeights* W) {
    if (!(corr_cells > 0.0f)) return go_fail(GO_ERR_INVALID, "correlation length must be positive");
    const double s = (double)corr_cells / sqrt(2.0);
    const int R = (int)ceil(3.0 * s);
    if (2 * R + 1 > kGrfMaxTaps)
        return go_fail(GO_ERR_INVALID, "correlation length %g cells exceeds the filter limit (R <= %d)",
                       (double)corr_cells, (kGrfMaxTaps - 1) / 2);
    double w[kGrfMaxTaps], ss = 0.0;
    for (int d = -R; d <= R; ++d) {
        w[d + R] = exp(-(double)d * d / (2.0 * s * s));
        ss += w[d + R] * w[d + R];
    }
    const double scale = 1.0 / sqrt(ss);
    memset(W, 0, sizeof(*W));
    W->R = R;
    for (int t = 0; t < 2 * R + 1; ++t) W->w[t] = (float)(w[t] * scale);
    return GO_OK;
}

int grf_launch(const GrfMember* d_members, const GrfMember& single, int n_members, int max_nx, int max_ny,
               uint32_t key0, uint32_t event, float std_dev, const GrfWeights& W, float* scratch,
               cudaStream_t s, const uint32_t* event_dev) {
    if (n_members < 1) return GO_OK;
    const dim3 gx((max_nx + kChunk - 1) / kChunk, max_ny + 2 * W.R, n_members);
    k_grf_xpass<<<gx, 256, 0, s>>>(d_members, single, key0, event, event_dev, scratch, W);
    const dim3 b(32, 8), gy((max_nx + 31) / 32, (max_ny + kYTile - 1) / kYTile, n_members);
    k_grf_ypass<<<gy, b, 0, s>>>(d_members, single, std_dev, scratch, W);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

}  // namespace go

extern "C" {

size_t go_grf_scratch_floats(int nx, int ny, float corr_cells) {
    GrfWeights W;
    if (nx < 1 || ny < 1 || grf_weights(corr_cells, &W)) return 0;
    return grf_member_scratch(nx, ny, W.R);
}

int go_grf_perturb(go_domain* d, void* stream, float* eta, int pitch, uint32_t key0, uint32_t key1,
                   uint32_t event, float std_dev, float corr_cells, float* scratch, size_t scratch_floats) {
    if (!d || !eta || !scratch) return go_fail(GO_ERR_INVALID, "null argument");
    int rc = go_check_pitch(pitch, d->k.nx + 4, "eta");
    if (rc) return rc;
    GrfWeights W;
    rc = grf_weights(corr_cells, &W);
    if (rc) return rc;
    const size_t need = grf_member_scratch(d->k.nx, d->k.ny, W.R);
    if (scratch_floats < need)
        return go_fail(GO_ERR_INVALID, "scratch holds %zu floats, need %zu", scratch_floats, need);
    GrfMember m;
    m.eta = eta;
    m.pitch = pitch / 4;
    m.nx = d->k.nx;
    m.ny = d->k.ny;
    m.periodic_x = d->k.bcE == kPeriodic;
    m.periodic_y = d->k.bcN == kPeriodic;
    m.key1 = key1;
    m.tmp_off = 0;
    return grf_launch(nullptr, m, 1, m.nx, m.ny, key0, event, std_dev, W, scratch, (cudaStream_t)stream);
}

}  // extern "C"
