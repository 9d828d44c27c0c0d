// Stochastic model error of OceanStateNoise: random fields (LCG or XORWOW),
// SOAR-correlated perturbation of eta on a coarse grid, and the
// geostrophically balanced perturbation of (eta, hu, hv) on the model grid,
// directly (interpolation factor 1) or through bicubic interpolation.
//
// Restates, kernel by kernel:
//   gpu_ocean/SWESimulators/gpu_kernels/ocean_noise.cu:81-118   (ansic_lcg, boxMuller)
//   gpu_ocean/SWESimulators/gpu_kernels/ocean_noise.cu:121-200  (uniformDistribution, normalDistribution)
//   gpu_ocean/SWESimulators/gpu_kernels/ocean_noise.cu:206-241  (makePerpendicular)
//   gpu_ocean/SWESimulators/gpu_kernels/ocean_noise.cu:249-372  (soar_covariance, SOAR)
//   gpu_ocean/SWESimulators/gpu_kernels/ocean_noise.cu:379-508  (geostrophicBalance)
//   gpu_ocean/SWESimulators/gpu_kernels/ocean_noise.cu:522-772  (bicubicInterpolation)
//   gpu_ocean/SWESimulators/gpu_kernels/common.cu:696-819       (bicubic coefficients, evaluation)
//   gpu_ocean/SWESimulators/gpu_kernels/reductions.cu           (squareSum, squareSumDouble)
// The reference compiles ocean_noise.cu with --use_fast_math
// (OceanStateNoise.py:222-227), so this unit is built with the same option
// (build.py UNIT_FLAGS) and writes each expression with the reference's
// operand order: approximate logf/expf/sqrtf/division and FMA contraction
// then round the same way.
//
// What differs from the reference's kernels, by design:
//  * SOAR: the 25 covariance weights depend only on the tap offset, so each
//    block evaluates them once (the reference's expression, per offset) into
//    shared memory instead of once per tap per cell; the sum runs in the
//    reference's tap order with the same fused multiply-adds.
//  * Per-cell indexing: every kernel computes each cell's sources from its
//    own global index (clamped or wrapped as the reference's shared tiles
//    are filled), so the launch shape is free and no thread reads past the
//    arrays (the reference's tiles read one row past the random buffer, and
//    its bicubic tile origin depends on the block).
//  * Reductions: many blocks with double accumulators and a fixed-order
//    finish by the last block, instead of one 128-thread block in float.
//  * XORWOW: curand's XORWOW device generator with one persistent state per
//    generator (pycuda's XORWOWRandomNumberGenerator uses the same
//    generator; its seeds and stream layout are its own, so the XORWOW path
//    matches the reference in distribution, not draw for draw).
#include "internal.h"
#include "trace.h"

#include <curand_kernel.h>

#include <algorithm>

namespace {

constexpr int kCutoff = 2;             // OceanStateNoise.py:96 (config.soar_cutoff)
constexpr int kBW = 32, kBH = 8;       // 2-D blocks of the per-cell kernels

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }
__device__ __forceinline__ int wrap(int v, int n) { return ((v % n) + n) % n; }

// ---- random numbers ---------------------------------------------------------

// One LCG step, (seed a + c) mod m with m = 2^31 - 1, the product wrapping
// at 2^64 as the reference's unsigned long long arithmetic does.  For seeds
// below 2^32 the sum is below 2^63 and m is a Mersenne prime, so the
// remainder folds with shifts and adds (x = h 2^31 + l = h + l mod m);
// larger seeds take the division.
__device__ __forceinline__ unsigned long long lcg_next(unsigned long long seed) {
    const unsigned long long m = 2147483647ULL;
    const unsigned long long x = seed * 1103515245ULL + 12345ULL;
    if (seed >> 32) return x % m;
    unsigned long long r = (x & m) + (x >> 31);
    r = (r & m) + (r >> 31);
    return r >= m ? r - m : r;
}

// ANSI C LCG, two draws (ocean_noise.cu:81-99): u = seed / 2^31 rounded to
// float (the quotient by a power of two is exact in double).
__device__ __forceinline__ float2 lcg_pair(unsigned long long& seed) {
    seed = lcg_next(seed);
    const float u1 = (float)((double)seed / 2147483648.0);
    seed = lcg_next(seed);
    const float u2 = (float)((double)seed / 2147483648.0);
    return make_float2(u1, u2);
}

// Box-Muller (ocean_noise.cu:106-116).
__device__ __forceinline__ float2 box_muller(float2 u) {
    const float r = sqrtf(-2.0f * logf(u.x));
    float s, c;
    sincospif(2 * u.y, &s, &c);
    return make_float2(r * c, r * s);
}

// One thread per seed; writes its pair into columns 2i, 2i+1 of its row
// (ocean_noise.cu:121-200).  The reference's branch for a lone last column
// (2i == random_nx) is met by no thread, so an odd width keeps its last
// column unwritten; kept as it is for parity.
__device__ __forceinline__ void lcg_body(int normal, int seed_nx, int seed_ny, int random_nx,
                                         unsigned long long* __restrict__ seed, int sp, float* __restrict__ rnd,
                                         int rp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= seed_nx || j >= seed_ny) return;
    unsigned long long s = seed[(size_t)j * sp + i];
    float2 u = lcg_pair(s);
    if (normal) u = box_muller(u);
    seed[(size_t)j * sp + i] = s;
    float* row = rnd + (size_t)j * rp;
    if (2 * i + 1 < random_nx) {
        row[2 * i] = u.x;
        row[2 * i + 1] = u.y;
    } else if (2 * i == random_nx) {
        row[2 * i] = u.x;
    }
}

__global__ void k_lcg(int normal, int seed_nx, int seed_ny, int random_nx, unsigned long long* __restrict__ seed,
                      int sp, float* __restrict__ rnd, int rp) {
    lcg_body(normal, seed_nx, seed_ny, random_nx, seed, sp, rnd, rp);
}

__global__ void k_xorwow_init(unsigned long long seed, int n, curandStateXORWOW_t* __restrict__ states) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    curandStateXORWOW_t st;
    curand_init(seed, (unsigned long long)g, 0ULL, &st);
    states[g] = st;
}

// Generator g fills the element pairs g, g + n, g + 2n, ... of the row-major
// nx x ny field (pitched rows).
__device__ __forceinline__ void xorwow_body(int normal, int n, curandStateXORWOW_t* __restrict__ states, int nx,
                                            int ny, float* __restrict__ out, int op) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    curandStateXORWOW_t st = states[g];
    const long long total = (long long)nx * ny;
    for (long long e = 2LL * g; e < total; e += 2LL * n) {
        float2 v;
        if (normal) {
            v = curand_normal2(&st);
        } else {
            v.x = curand_uniform(&st);
            v.y = curand_uniform(&st);
        }
        const int j0 = (int)(e / nx), i0 = (int)(e % nx);
        out[(size_t)j0 * op + i0] = v.x;
        if (e + 1 < total) {
            const int j1 = (int)((e + 1) / nx), i1 = (int)((e + 1) % nx);
            out[(size_t)j1 * op + i1] = v.y;
        }
    }
    states[g] = st;
}

__global__ void k_xorwow_fill(int normal, int n, curandStateXORWOW_t* __restrict__ states, int nx, int ny,
                              float* __restrict__ out, int op) {
    xorwow_body(normal, n, states, nx, ny, out, op);
}

// ---- SOAR covariance on the coarse grid ---------------------------------------

// soar_covariance of ocean_noise.cu:249-255 for the tap offset (ox, oy) =
// (a_x - b_x, a_y - b_y).
__device__ __forceinline__ float soar_weight(int ox, int oy, float dx, float dy, float q0, float L) {
    const float dist = sqrtf(dx * dx * ox * ox + dy * dy * oy * oy);
    return q0 * (1.0f + dist / L) * expf(-dist / L);
}

constexpr int kTaps = 2 * kCutoff + 1;
constexpr int kSoarRows = 8;                  // coarse rows per thread
constexpr int kSoarTY = 4;                    // thread rows per block
constexpr int kSoarBH = kSoarRows * kSoarTY;  // 32 coarse rows per block

// Index into the random buffer behind tile position c (coarse index plus
// tap) along one axis (ocean_noise.cu:300-330): wrapped over the n interior
// values when periodic (c - 4), else c itself in a buffer with 4 extra
// values on each side.  -1 for positions no written cell reads (beyond
// c - 4 = n + 3, or c = n + 7).
__device__ __forceinline__ int random_src(int c, int n, int periodic) {
    if (periodic) {
        int v = c - 2 * kCutoff;
        if (v > n + 3) return -1;
        if (n < 2 * kCutoff) return wrap(v, n);
        return v < 0 ? v + n : (v >= n ? v - n : v);
    }
    return c > n + 4 * kCutoff - 1 ? -1 : c;
}

// Coarse cells, ghost cells included ((nx+4) x (ny+4)): coarse = scale *
// sum_taps Q(tap) xi(tap), or += when additive (ocean_noise.cu:264-372).
// A block covers 32 x 32 cells; the random values behind them (36 x 36) sit
// in shared memory and each thread sums a strip of 8 cells down one column
// from registers, taps in the reference's order (rows outer, columns inner).
__device__ __forceinline__ void soar_body(int nx, int ny, float dx, float dy, float q0, float L, float scale, int pns,
                                          int pew, const float* __restrict__ rnd, int rp, float* __restrict__ coarse,
                                          int cp, int additive, int aligned16) {
    constexpr int TW = kBW + 2 * kCutoff, TH = kSoarBH + 2 * kCutoff;
    static_assert(TW % 4 == 0 && (2 * kCutoff) % 4 == 0, "float4 tile rows");
    __shared__ float xi[TH][TW];
    __shared__ float w[kTaps * kTaps];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int t = ty * kBW + tx;
    const int bx = blockIdx.x * kBW, by = blockIdx.y * kSoarBH;
    if (t < kTaps * kTaps) w[t] = soar_weight(kCutoff - t % kTaps, kCutoff - t / kTaps, dx, dy, q0, L);
    // First random row and column behind the tile, and whether the whole
    // tile lies inside the random buffer without wrapping: then its rows are
    // read as 9 aligned float4 each (the first column is a multiple of 4;
    // aligned16 says the buffer and pitch are 16-byte aligned).
    const int row0 = pns ? by - 2 * kCutoff : by;
    const int col0 = pew ? bx - 2 * kCutoff : bx;
    const int rows_avail = pns ? ny : ny + 4 * kCutoff;
    const int cols_avail = pew ? nx : nx + 4 * kCutoff;
    if (aligned16 && row0 >= 0 && col0 >= 0 && row0 + TH <= rows_avail && col0 + TW <= cols_avail) {
        constexpr int V = TW / 4;
        for (int k = t; k < TH * V; k += kBW * kSoarTY) {
            const int j = k / V, v = k % V;
            const float4 q = __ldg(reinterpret_cast<const float4*>(rnd + (size_t)(row0 + j) * rp + col0) + v);
            xi[j][4 * v] = q.x;
            xi[j][4 * v + 1] = q.y;
            xi[j][4 * v + 2] = q.z;
            xi[j][4 * v + 3] = q.w;
        }
    } else {
        // edge tiles: each thread fills tile columns tx and tx + 32 (tx < 4)
        const int gi0 = random_src(bx + tx, nx, pew);
        const int gi1 = tx < TW - kBW ? random_src(bx + kBW + tx, nx, pew) : -1;
        for (int j = ty; j < TH; j += kSoarTY) {
            const int gj = random_src(by + j, ny, pns);
            const float* row = rnd + (size_t)max(gj, 0) * rp;
            xi[j][tx] = (gj >= 0 && gi0 >= 0) ? __ldg(row + gi0) : 0.0f;
            if (tx < TW - kBW) xi[j][kBW + tx] = (gj >= 0 && gi1 >= 0) ? __ldg(row + gi1) : 0.0f;
        }
    }
    __syncthreads();
    float wr[kTaps * kTaps];
#pragma unroll
    for (int k = 0; k < kTaps * kTaps; ++k) wr[k] = w[k];
    const int ti = bx + tx;
    const int r0 = ty * kSoarRows;
    // The tile rows q = r0 .. r0 + 11 are read once each, in order; row q
    // is tap row ky = q - r of cell r, so every cell still receives its taps
    // rows first, columns second, as the reference sums them.
    float acc[kSoarRows];
#pragma unroll
    for (int r = 0; r < kSoarRows; ++r) acc[r] = 0.0f;
#pragma unroll
    for (int q = 0; q < kSoarRows + kTaps - 1; ++q) {
        float x[kTaps];
#pragma unroll
        for (int kx = 0; kx < kTaps; ++kx) x[kx] = xi[r0 + q][tx + kx];
#pragma unroll
        for (int r = 0; r < kSoarRows; ++r) {
            const int ky = q - r;
            if (ky < 0 || ky >= kTaps) continue;
#pragma unroll
            for (int kx = 0; kx < kTaps; ++kx) acc[r] = __fmaf_rn(wr[ky * kTaps + kx], x[kx], acc[r]);
        }
    }
    if (ti >= nx + 4) return;
#pragma unroll
    for (int r = 0; r < kSoarRows; ++r) {
        const int tj = by + r0 + r;
        if (tj < ny + 4) {
            float* out = coarse + (size_t)tj * cp + ti;
            *out = additive > 0 ? __fmaf_rn(scale, acc[r], *out) : scale * acc[r];
        }
    }
}

__global__ void __launch_bounds__(kBW* kSoarTY) k_soar(int nx, int ny, float dx, float dy, float q0, float L,
                                                       float scale, int pns, int pew,
                                                       const float* __restrict__ rnd, int rp,
                                                       float* __restrict__ coarse, int cp, int additive,
                                                       int aligned16) {
    soar_body(nx, ny, dx, dy, q0, L, scale, pns, pew, rnd, rp, coarse, cp, additive, aligned16);
}

// ---- geostrophic balance -------------------------------------------------------

struct BalanceArgs {
    int nx, ny, gx, gy;
    float dx, dy, g, f, beta;
    const float* coarse;
    // interior cells perturbed: [i_lo, i_hi) x [j_lo, j_hi)
    int i_lo, i_hi, j_lo, j_hi;
    int cp;
    float *eta, *hu, *hv;
    int pe, pu, pv;
    const float* Hi;
    int ph;
    float land;
    cudaTextureObject_t angle, coriolis;
};

// H at the cell centre and whether a corner is land (ocean_noise.cu:418-438).
__device__ __forceinline__ void cell_depth(const BalanceArgs& a, int ti, int tj, float& H_mid, bool& dry) {
    const int j0 = clampi(tj, 0, a.ny + 4), j1 = clampi(tj + 1, 0, a.ny + 4);
    const int i0 = clampi(ti, 0, a.nx + 4), i1 = clampi(ti + 1, 0, a.nx + 4);
    const float h00 = __ldg(a.Hi + (size_t)j0 * a.ph + i0), h01 = __ldg(a.Hi + (size_t)j0 * a.ph + i1);
    const float h10 = __ldg(a.Hi + (size_t)j1 * a.ph + i0), h11 = __ldg(a.Hi + (size_t)j1 * a.ph + i1);
    dry = (h00 == a.land) || (h01 == a.land) || (h10 == a.land) || (h11 == a.land);
    H_mid = 0.25f * (h00 + h01 + h10 + h11);
}

// How the Coriolis parameter of a cell is found (ocean_noise.cu:471-476):
// the reference evaluates f + beta (north . x) with the north vector from
// the angle texture, then takes the Coriolis texture instead when f == 0.
// With beta == 0 and f != 0 that is f + 0 * (finite) = f exactly, so the
// texture and trigonometry are only needed in the two other cases.
enum CoriolisMode { kCorF = 0, kCorBeta = 1, kCorTexture = 2 };

__host__ __device__ __forceinline__ int coriolis_mode(float f, float beta) {
    return f == 0.0f ? kCorTexture : (beta == 0.0f ? kCorF : kCorBeta);
}

__device__ __forceinline__ float cell_coriolis(const BalanceArgs& a, int mode, int ti, int tj) {
    if (mode == kCorF) return a.f;
    const float s = (ti + 0.5f) / (a.nx + 4.0f);
    const float t = (tj + 0.5f) / (a.ny + 4.0f);
    if (mode == kCorTexture) return tex2D<float>(a.coriolis, s, t);
    const float angle = tex2D<float>(a.angle, s, t);
    const float2 north = make_float2(sinf(angle), cosf(angle));
    return a.f + a.beta * ((ti + 0.5f) * a.dx * north.x + (tj + 0.5f) * a.dy * north.y);
}

constexpr int kBalRows = 4;                   // cells per thread, down a column

// One interior cell's balance (ocean_noise.cu:418-508): corner depths
// h00..h11 (rows tj, tj+1 x columns ti, ti+1), the coarse perturbation d at
// the cell and its neighbours (cl, cr west and east, cdn, cup south and
// north), the cell's (e, u, v); returns the new (eta, hu, hv).
__device__ __forceinline__ float3 balance_cell(const BalanceArgs& a, int mode, int ti, int tj, float h00, float h01,
                                               float h10, float h11, float d, float cl, float cr, float cdn,
                                               float cup, float e, float u, float v) {
    const bool dry = (h00 == a.land) || (h01 == a.land) || (h10 == a.land) || (h11 == a.land);
    if (dry) return make_float3(0.0f, 0.0f, 0.0f);
    const float H_mid = 0.25f * (h00 + h01 + h10 + h11);
    const float coriolis = cell_coriolis(a, mode, ti, tj);
    const float h_mid = d + H_mid + e;
    const float eta_diff_x = (cr - cl) / (2.0f * a.dx);
    const float eta_diff_y = (cup - cdn) / (2.0f * a.dy);
    // d_hu = -(g / f) h_mid d_y eta and d_hv = (g / f) h_mid d_x eta; the
    // reference's hu += d_hu contracts into one fused multiply-add with the
    // last product (ocean_noise.cu:480-493 under --use_fast_math), written
    // out here so the rounding does not depend on the compiler.
    return make_float3(e + d, __fmaf_rn(-(a.g / coriolis) * h_mid, eta_diff_y, u),
                       __fmaf_rn((a.g / coriolis) * h_mid, eta_diff_x, v));
}

// Interior cells of the model grid; the coarse grid is the model grid
// (ocean_noise.cu:379-508).  Each thread marches kBalRows cells down one
// column, carrying the coarse values of the rows above and below and the
// lower corner pair of Hi from one cell to the next.
__device__ __forceinline__ void balance_body(const BalanceArgs& a, int mode) {
    const int ti = blockIdx.x * kBW + threadIdx.x + a.i_lo;
    const int tj0 = (blockIdx.y * kBH + threadIdx.y) * kBalRows + a.j_lo;
    if (ti >= a.i_hi) return;
    const float* __restrict__ coarse = a.coarse;
    const float* __restrict__ Hi = a.Hi;
    float* __restrict__ eta_p = a.eta;
    float* __restrict__ hu_p = a.hu;
    float* __restrict__ hv_p = a.hv;
    auto c = [&](int i, int j) {
        return __ldg(coarse + (size_t)clampi(j, 0, a.ny + 3) * a.cp + clampi(i, 0, a.nx + 3));
    };
    auto h = [&](int i, int j) { return __ldg(Hi + (size_t)clampi(j, 0, a.ny + 4) * a.ph + clampi(i, 0, a.nx + 4)); };
    // every input of the column strip first (independent loads in flight),
    // then the cells; rows past the grid load clamped values and are skipped
    float cc[kBalRows + 2], cl[kBalRows], cr[kBalRows], hl[kBalRows + 1], hr[kBalRows + 1];
    float e[kBalRows], u[kBalRows], v[kBalRows];
#pragma unroll
    for (int k = 0; k < kBalRows + 2; ++k) cc[k] = c(ti, tj0 - 1 + k);
#pragma unroll
    for (int k = 0; k < kBalRows + 1; ++k) {
        hl[k] = h(ti, tj0 + k);
        hr[k] = h(ti + 1, tj0 + k);
    }
#pragma unroll
    for (int r = 0; r < kBalRows; ++r) {
        const int tj = min(tj0 + r, a.ny + 3);
        cl[r] = c(ti - 1, tj);
        cr[r] = c(ti + 1, tj);
        e[r] = eta_p[(size_t)tj * a.pe + ti];
        u[r] = hu_p[(size_t)tj * a.pu + ti];
        v[r] = hv_p[(size_t)tj * a.pv + ti];
    }
#pragma unroll
    for (int r = 0; r < kBalRows; ++r) {
        const int tj = tj0 + r;
        if (tj >= a.j_hi) continue;
        const float3 q = balance_cell(a, mode, ti, tj, hl[r], hr[r], hl[r + 1], hr[r + 1], cc[r + 1], cl[r], cr[r],
                                      cc[r], cc[r + 2], e[r], u[r], v[r]);
        eta_p[(size_t)tj * a.pe + ti] = q.x;
        hu_p[(size_t)tj * a.pu + ti] = q.y;
        hv_p[(size_t)tj * a.pv + ti] = q.z;
    }
}

__global__ void __launch_bounds__(kBW* kBH) k_balance(const BalanceArgs a, int mode) { balance_body(a, mode); }

// ---- bicubic interpolation from the coarse grid ---------------------------------

struct M4 {
    float4 r0, r1, r2, r3;
};

__device__ __forceinline__ float dot4(const float4 a, const float4 b) {
    return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}

// Coefficients B F B^T of the bicubic patch for corner values and
// derivatives F (common.cu:723-801; B = [[1,0,0,0],[0,0,1,0],[-3,3,-2,-1],
// [2,-2,1,1]]), as dot products of F's rows with B's rows, then B's rows
// with those.
__device__ __forceinline__ M4 bicubic_coefficients(const M4 f) {
    const float4 b0 = make_float4(1.0f, 0.0f, 0.0f, 0.0f);
    const float4 b1 = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
    const float4 b2 = make_float4(-3.0f, 3.0f, -2.0f, -1.0f);
    const float4 b3 = make_float4(2.0f, -2.0f, 1.0f, 1.0f);
    M4 ft;   // (F B^T)^T
    ft.r0 = make_float4(dot4(f.r0, b0), dot4(f.r1, b0), dot4(f.r2, b0), dot4(f.r3, b0));
    ft.r1 = make_float4(dot4(f.r0, b1), dot4(f.r1, b1), dot4(f.r2, b1), dot4(f.r3, b1));
    ft.r2 = make_float4(dot4(f.r0, b2), dot4(f.r1, b2), dot4(f.r2, b2), dot4(f.r3, b2));
    ft.r3 = make_float4(dot4(f.r0, b3), dot4(f.r1, b3), dot4(f.r2, b3), dot4(f.r3, b3));
    M4 o;
    o.r0 = make_float4(dot4(b0, ft.r0), dot4(b0, ft.r1), dot4(b0, ft.r2), dot4(b0, ft.r3));
    o.r1 = make_float4(dot4(b1, ft.r0), dot4(b1, ft.r1), dot4(b1, ft.r2), dot4(b1, ft.r3));
    o.r2 = make_float4(dot4(b2, ft.r0), dot4(b2, ft.r1), dot4(b2, ft.r2), dot4(b2, ft.r3));
    o.r3 = make_float4(dot4(b3, ft.r0), dot4(b3, ft.r1), dot4(b3, ft.r2), dot4(b3, ft.r3));
    return o;
}

// x^T C y (common.cu:803-819).
__device__ __forceinline__ float bicubic_eval(const float4 x, const float4 y, const M4 c) {
    const float4 tmp = make_float4(dot4(c.r0, y), dot4(c.r1, y), dot4(c.r2, y), dot4(c.r3, y));
    return dot4(x, tmp);
}

struct InterpArgs {
    BalanceArgs b;
    int cnx, cny, cgx, cgy;
    float cdx, cdy;
    int off_i, off_j;
};

// d_eta at ghost-inclusive model cell (ti, tj): the coarse cell below-left
// of the cell centre, its 4x4 neighbourhood (clamped to the coarse array),
// central differences for the derivatives and the bicubic patch
// (ocean_noise.cu:610-705).
__device__ float interpolate(const InterpArgs& a, int ti, int tj) {
    const float x = (ti - a.b.gx + 0.5f + a.off_i) * a.b.dx;
    const float y = (tj - a.b.gy + 0.5f + a.off_j) * a.b.dy;
    int ci = (int)(floorf((x / a.cdx) + a.cgx - 0.5f));
    int cj = (int)(floorf((y / a.cdy) + a.cgy - 0.5f));
    if (ci > a.cnx + 1) ci -= 1;
    if (cj > a.cny + 1) cj -= 1;
    const float coarse_x = (ci - a.cgx + 0.5f) * a.cdx;
    const float coarse_y = (cj - a.cgy + 0.5f) * a.cdy;
    auto c = [&](int di, int dj) {
        return __ldg(a.b.coarse + (size_t)clampi(cj + dj, 0, a.cny + 3) * a.b.cp + clampi(ci + di, 0, a.cnx + 3));
    };
    M4 f;
    f.r0.x = c(0, 0);
    f.r0.y = c(0, 1);
    f.r1.x = c(1, 0);
    f.r1.y = c(1, 1);
    f.r2.x = (c(1, 0) - c(-1, 0)) / 2.0f;
    f.r2.y = (c(1, 1) - c(-1, 1)) / 2.0f;
    f.r3.x = (c(2, 0) - c(0, 0)) / 2.0f;
    f.r3.y = (c(2, 1) - c(0, 1)) / 2.0f;
    f.r0.z = (c(0, 1) - c(0, -1)) / 2.0f;
    f.r0.w = (c(0, 2) - c(0, 0)) / 2.0f;
    f.r1.z = (c(1, 1) - c(1, -1)) / 2.0f;
    f.r1.w = (c(1, 2) - c(1, 0)) / 2.0f;
    const float fy_10 = (c(-1, 1) - c(-1, -1)) / 2.0f;
    const float fy_11 = (c(-1, 2) - c(-1, 0)) / 2.0f;
    const float fy20 = (c(2, 1) - c(2, -1)) / 2.0f;
    const float fy21 = (c(2, 2) - c(2, 0)) / 2.0f;
    f.r2.z = (f.r1.z - fy_10) / 2.0f;
    f.r2.w = (f.r1.w - fy_11) / 2.0f;
    f.r3.z = (fy20 - f.r0.z) / 2.0f;
    f.r3.w = (fy21 - f.r0.w) / 2.0f;
    const float rel_x = (x - coarse_x) / a.cdx;
    const float rel_y = (y - coarse_y) / a.cdy;
    const M4 coef = bicubic_coefficients(f);
    const float4 xv = make_float4(1.0f, rel_x, rel_x * rel_x, rel_x * rel_x * rel_x);
    const float4 yv = make_float4(1.0f, rel_y, rel_y * rel_y, rel_y * rel_y * rel_y);
    return bicubic_eval(xv, yv, coef);
}

// Interior cells: d_eta interpolated on the block and a one-cell halo into
// shared memory, then the geostrophic balance from its central differences
// (ocean_noise.cu:522-772).
__global__ void __launch_bounds__(kBW* kBH) k_interp_balance(const InterpArgs a) {
    __shared__ float d_eta[kBH + 2][kBW + 2];
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int bx = blockIdx.x * kBW + a.b.i_lo, by = blockIdx.y * kBH + a.b.j_lo;
    for (int j = ty; j < kBH + 2; j += kBH)
        for (int i = tx; i < kBW + 2; i += kBW) d_eta[j][i] = interpolate(a, bx + i - 1, by + j - 1);
    __syncthreads();
    const int ti = bx + tx, tj = by + ty;
    if (ti >= a.b.i_hi || tj >= a.b.j_hi) return;
    float H_mid;
    bool dry;
    cell_depth(a.b, ti, tj, H_mid, dry);
    const float coriolis = cell_coriolis(a.b, coriolis_mode(a.b.f, a.b.beta), ti, tj);
    const int ex = tx + 1, ey = ty + 1;
    const float eta_diff_x = (d_eta[ey][ex + 1] - d_eta[ey][ex - 1]) / (2.0f * a.b.dx);
    const float eta_diff_y = (d_eta[ey + 1][ex] - d_eta[ey - 1][ex]) / (2.0f * a.b.dy);
    float d = d_eta[ey][ex];
    float d_hu = -(a.b.g / coriolis) * (H_mid + d) * eta_diff_y;
    float d_hv = (a.b.g / coriolis) * (H_mid + d) * eta_diff_x;
    if (dry) {
        d = 0.0f;
        d_hu = 0.0f;
        d_hv = 0.0f;
    }
    // here the land test selects d_hu before the sum, so the reference adds
    // the rounded product (no contraction, ocean_noise.cu:758-770)
    float* eta = a.b.eta + (size_t)tj * a.b.pe + ti;
    float* hu = a.b.hu + (size_t)tj * a.b.pu + ti;
    float* hv = a.b.hv + (size_t)tj * a.b.pv + ti;
    *eta = __fadd_rn(*eta, d);
    *hu = __fadd_rn(*hu, d_hu);
    *hv = __fadd_rn(*hv, d_hv);
}

// ---- reductions and the perpendicular field ------------------------------------

constexpr int kRedThreads = 256;
constexpr int kRedBlocksMax = 1184;    // 148 SMs x 8

struct RedScratch {
    unsigned int ticket;
    unsigned int pad;
    double part[kRedBlocksMax][3];
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block sums of a^2 (and b^2, a b when b is given) over an nx x ny pitched
// field; the last block to finish adds the partials in block order and
// writes the floats (reductions.cu: squareSum, squareSumDouble).
__global__ void __launch_bounds__(kRedThreads) k_square_sums(int nx, int ny, const float* __restrict__ a, int pa,
                                                             const float* __restrict__ b, int pb,
                                                             float* __restrict__ result, RedScratch* s) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    const long long total = (long long)nx * ny;
    for (long long e = (long long)blockIdx.x * kRedThreads + threadIdx.x; e < total;
         e += (long long)gridDim.x * kRedThreads) {
        const int j = (int)(e / nx), i = (int)(e % nx);
        const double x = __ldg(a + (size_t)j * pa + i);
        s0 += x * x;
        if (b) {
            const double y = __ldg(b + (size_t)j * pb + i);
            s1 += y * y;
            s2 += x * y;
        }
    }
    __shared__ double red[3][kRedThreads / 32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    if (lane == 0) {
        red[0][warp] = s0;
        red[1][warp] = s1;
        red[2][warp] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0, t2 = 0.0;
        for (int w = 0; w < kRedThreads / 32; ++w) {
            t0 += red[0][w];
            t1 += red[1][w];
            t2 += red[2][w];
        }
        s->part[blockIdx.x][0] = t0;
        s->part[blockIdx.x][1] = t1;
        s->part[blockIdx.x][2] = t2;
        __threadfence();
        last = (atomicAdd(&s->ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double t0 = 0.0, t1 = 0.0, t2 = 0.0;
    for (unsigned int k = 0; k < gridDim.x; ++k) {
        t0 += ((volatile double*)s->part[k])[0];
        t1 += ((volatile double*)s->part[k])[1];
        t2 += ((volatile double*)s->part[k])[2];
    }
    result[0] = (float)t0;
    if (b) {
        result[1] = (float)t1;
        result[2] = (float)t2;
    }
    s->ticket = 0;
}

// nu <- sqrt(|nu|^2 / |nu_perp|^2) (nu - (xi.nu / |xi|^2) xi)
// (ocean_noise.cu:206-241), from the three sums in red.
__global__ void k_make_perpendicular(int nx, int ny, const float* __restrict__ xi, int px, float* __restrict__ nu,
                                     int pn, const float* __restrict__ red) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= nx || j >= ny) return;
    const float xi_norm = red[0];
    const float nu_norm = red[1];
    const float dot_product = red[2];
    const float parallel_factor = dot_product / xi_norm;
    const float perpendicular_norm = nu_norm - parallel_factor * dot_product;
    float* n = nu + (size_t)j * pn + i;
    *n = sqrtf(nu_norm / perpendicular_norm) * (*n - (parallel_factor * xi[(size_t)j * px + i]));
}

int check_field(int pitch_bytes, int width, const char* what) { return go_check_pitch(pitch_bytes, width, what); }

}  // namespace

extern "C" {

int go_noise_lcg(void* stream, int normal, int seed_nx, int seed_ny, int random_nx, uint64_t* seed,
                 int seed_pitch, float* random, int random_pitch) {
    if (!seed || !random) return go_fail(GO_ERR_INVALID, "null argument");
    if (seed_nx < 1 || seed_ny < 1 || random_nx < 1 || (random_nx + 1) / 2 > seed_nx)
        return go_fail(GO_ERR_INVALID, "seed grid %d x %d cannot fill %d random columns", seed_nx, seed_ny,
                       random_nx);
    if (seed_pitch < 8 * seed_nx || seed_pitch % 8)
        return go_fail(GO_ERR_INVALID, "seed pitch %d for %d seeds", seed_pitch, seed_nx);
    int rc = check_field(random_pitch, random_nx, "random");
    if (rc) return rc;
    const dim3 block(64, 4);
    const dim3 grid((seed_nx + 63) / 64, (seed_ny + 3) / 4);
    k_lcg<<<grid, block, 0, (cudaStream_t)stream>>>(normal, seed_nx, seed_ny, random_nx,
                                                    (unsigned long long*)seed, seed_pitch / 8, random,
                                                    random_pitch / 4);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

size_t go_noise_xorwow_state_bytes(void) { return sizeof(curandStateXORWOW_t); }

int go_noise_xorwow_init(void* stream, uint64_t seed, int n_generators, void* states) {
    if (!states || n_generators < 1) return go_fail(GO_ERR_INVALID, "no generator states");
    k_xorwow_init<<<(n_generators + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
        (unsigned long long)seed, n_generators, (curandStateXORWOW_t*)states);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

int go_noise_xorwow_fill(void* stream, int normal, int n_generators, void* states, int nx, int ny, float* out,
                         int out_pitch) {
    if (!states || !out || n_generators < 1) return go_fail(GO_ERR_INVALID, "null argument");
    if (nx < 1 || ny < 1) return go_fail(GO_ERR_INVALID, "empty field");
    int rc = check_field(out_pitch, nx, "random");
    if (rc) return rc;
    k_xorwow_fill<<<(n_generators + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
        normal, n_generators, (curandStateXORWOW_t*)states, nx, ny, out, out_pitch / 4);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

int go_noise_soar(void* stream, int coarse_nx, int coarse_ny, float coarse_dx, float coarse_dy, float soar_q0,
                  float soar_L, float perturbation_scale, int periodic_north_south, int periodic_east_west,
                  const float* random, int random_pitch, float* coarse, int coarse_pitch, int additive) {
    if (!random || !coarse) return go_fail(GO_ERR_INVALID, "null argument");
    if (coarse_nx < 1 || coarse_ny < 1) return go_fail(GO_ERR_INVALID, "empty coarse grid");
    const int rnx = periodic_east_west ? coarse_nx : coarse_nx + 4 * kCutoff;
    int rc = check_field(random_pitch, rnx, "random");
    if (!rc) rc = check_field(coarse_pitch, coarse_nx + 4, "coarse");
    if (rc) return rc;
    const dim3 grid((coarse_nx + 4 + kBW - 1) / kBW, (coarse_ny + 4 + kSoarBH - 1) / kSoarBH);
    k_soar<<<grid, dim3(kBW, kSoarTY), 0, (cudaStream_t)stream>>>(
        coarse_nx, coarse_ny, coarse_dx, coarse_dy, soar_q0, soar_L, perturbation_scale, periodic_north_south,
        periodic_east_west, random, random_pitch / 4, coarse, coarse_pitch / 4, additive,
        (((uintptr_t)random | (uintptr_t)random_pitch) & 15) == 0);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

static int fill_balance(BalanceArgs& a, int nx, int ny, float dx, float dy, int ghost_x, int ghost_y, float g, float f,
                        float beta, const float* coarse, int coarse_pitch, int coarse_width, float* eta,
                        int eta_pitch, float* hu, int hu_pitch, float* hv, int hv_pitch, const float* Hi,
                        int Hi_pitch, float land_value, uint64_t angle_texture, uint64_t coriolis_texture) {
    if (!coarse || !eta || !hu || !hv || !Hi) return go_fail(GO_ERR_INVALID, "null argument");
    if (nx < 1 || ny < 1) return go_fail(GO_ERR_INVALID, "empty grid");
    if (!angle_texture || !coriolis_texture) return go_fail(GO_ERR_INVALID, "angle and Coriolis textures needed");
    int rc = check_field(coarse_pitch, coarse_width, "coarse");
    if (!rc) rc = check_field(eta_pitch, nx + 4, "eta");
    if (!rc) rc = check_field(hu_pitch, nx + 4, "hu");
    if (!rc) rc = check_field(hv_pitch, nx + 4, "hv");
    if (!rc) rc = check_field(Hi_pitch, nx + 5, "Hi");
    if (rc) return rc;
    a.nx = nx; a.ny = ny; a.gx = ghost_x; a.gy = ghost_y;
    a.dx = dx; a.dy = dy; a.g = g; a.f = f; a.beta = beta;
    a.coarse = coarse; a.cp = coarse_pitch / 4;
    a.eta = eta; a.hu = hu; a.hv = hv;
    a.pe = eta_pitch / 4; a.pu = hu_pitch / 4; a.pv = hv_pitch / 4;
    a.Hi = Hi; a.ph = Hi_pitch / 4; a.land = land_value;
    // The reference launches one 16 x 16 block per 16 x 16 cells from the
    // ghost offset and perturbs the interior cells its threads reach
    // (OceanStateNoise.py:279-282, ocean_noise.cu:462): with offsets 0 or
    // 1 that can stop short of the last interior cells.  Same cells here.
    constexpr int kRefBlock = 16;
    a.i_lo = ghost_x > 2 ? ghost_x : 2;
    a.j_lo = ghost_y > 2 ? ghost_y : 2;
    a.i_hi = std::min(nx + 2, ghost_x + kRefBlock * ((nx + kRefBlock - 1) / kRefBlock));
    a.j_hi = std::min(ny + 2, ghost_y + kRefBlock * ((ny + kRefBlock - 1) / kRefBlock));
    a.angle = (cudaTextureObject_t)angle_texture;
    a.coriolis = (cudaTextureObject_t)coriolis_texture;
    return GO_OK;
}

int go_noise_geostrophic(void* stream, int nx, int ny, float dx, float dy, int ghost_x, int ghost_y, float g,
                         float f, float beta, float y0_reference_cell, const float* coarse, int coarse_pitch,
                         float* eta, int eta_pitch, float* hu, int hu_pitch, float* hv, int hv_pitch,
                         const float* Hi, int Hi_pitch, float land_value, uint64_t angle_texture,
                         uint64_t coriolis_texture) {
    (void)y0_reference_cell;   // accepted and unused, as in the reference kernel
    BalanceArgs a;
    int rc = fill_balance(a, nx, ny, dx, dy, ghost_x, ghost_y, g, f, beta, coarse, coarse_pitch, nx + 4, eta,
                          eta_pitch, hu, hu_pitch, hv, hv_pitch, Hi, Hi_pitch, land_value, angle_texture,
                          coriolis_texture);
    if (rc) return rc;
    const int ci = a.i_hi - a.i_lo, cj = a.j_hi - a.j_lo;
    if (ci <= 0 || cj <= 0) return GO_OK;
    const dim3 grid((ci + kBW - 1) / kBW, (cj + kBH * kBalRows - 1) / (kBH * kBalRows));
    k_balance<<<grid, dim3(kBW, kBH), 0, (cudaStream_t)stream>>>(a, coriolis_mode(f, beta));
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

int go_noise_bicubic(void* stream, int nx, int ny, int ghost_x, int ghost_y, float dx, float dy, int coarse_nx,
                     int coarse_ny, int coarse_ghost_x, int coarse_ghost_y, float coarse_dx, float coarse_dy,
                     int offset_i, int offset_j, float g, float f, float beta, float y0_reference_cell,
                     const float* coarse, int coarse_pitch, float* eta, int eta_pitch, float* hu, int hu_pitch,
                     float* hv, int hv_pitch, const float* Hi, int Hi_pitch, float land_value,
                     uint64_t angle_texture, uint64_t coriolis_texture) {
    (void)y0_reference_cell;
    if (coarse_nx < 1 || coarse_ny < 1) return go_fail(GO_ERR_INVALID, "empty coarse grid");
    InterpArgs a;
    int rc = fill_balance(a.b, nx, ny, dx, dy, ghost_x, ghost_y, g, f, beta, coarse, coarse_pitch, coarse_nx + 4,
                          eta, eta_pitch, hu, hu_pitch, hv, hv_pitch, Hi, Hi_pitch, land_value, angle_texture,
                          coriolis_texture);
    if (rc) return rc;
    a.cnx = coarse_nx; a.cny = coarse_ny; a.cgx = coarse_ghost_x; a.cgy = coarse_ghost_y;
    a.cdx = coarse_dx; a.cdy = coarse_dy; a.off_i = offset_i; a.off_j = offset_j;
    const int ci = a.b.i_hi - a.b.i_lo, cj = a.b.j_hi - a.b.j_lo;
    if (ci <= 0 || cj <= 0) return GO_OK;
    const dim3 grid((ci + kBW - 1) / kBW, (cj + kBH - 1) / kBH);
    k_interp_balance<<<grid, dim3(kBW, kBH), 0, (cudaStream_t)stream>>>(a);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

size_t go_noise_reduce_scratch_bytes(void) { return sizeof(RedScratch); }

int go_noise_square_sums(void* stream, int nx, int ny, const float* a, int a_pitch, const float* b, int b_pitch,
                         float* result, void* scratch, size_t scratch_bytes) {
    if (!a || !result || !scratch) return go_fail(GO_ERR_INVALID, "null argument");
    if (nx < 1 || ny < 1) return go_fail(GO_ERR_INVALID, "empty field");
    if (scratch_bytes < sizeof(RedScratch))
        return go_fail(GO_ERR_INVALID, "reduction scratch of %zu bytes, %zu needed", scratch_bytes,
                       sizeof(RedScratch));
    int rc = check_field(a_pitch, nx, "a");
    if (!rc && b) rc = check_field(b_pitch, nx, "b");
    if (rc) return rc;
    const long long total = (long long)nx * ny;
    const int blocks = (int)std::min<long long>(kRedBlocksMax, (total + kRedThreads - 1) / kRedThreads);
    k_square_sums<<<blocks, kRedThreads, 0, (cudaStream_t)stream>>>(nx, ny, a, a_pitch / 4, b, b ? b_pitch / 4 : 0,
                                                                    result, (RedScratch*)scratch);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

int go_noise_make_perpendicular(void* stream, int nx, int ny, const float* xi, int xi_pitch, float* nu,
                                int nu_pitch, const float* reduction) {
    if (!xi || !nu || !reduction) return go_fail(GO_ERR_INVALID, "null argument");
    if (nx < 1 || ny < 1) return go_fail(GO_ERR_INVALID, "empty field");
    int rc = check_field(xi_pitch, nx, "xi");
    if (!rc) rc = check_field(nu_pitch, nx, "nu");
    if (rc) return rc;
    const dim3 grid((nx + kBW - 1) / kBW, (ny + kBH - 1) / kBH);
    k_make_perpendicular<<<grid, dim3(kBW, kBH), 0, (cudaStream_t)stream>>>(nx, ny, xi, xi_pitch / 4, nu,
                                                                            nu_pitch / 4, reduction);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

}  // extern "C"

// ---- the model error of an ensemble, batched across members ---------------------
//
// One launch per kernel over all members (blockIdx.z = member); each block
// runs the single-member kernel's body on its member's buffers and
// parameters, so each member gets exactly its own perturbation.

namespace {

__global__ void k_lcg_batch(const go_noise_member* __restrict__ m, int seed_nx, int seed_ny, int random_nx) {
    const go_noise_member& a = m[blockIdx.z];
    lcg_body(1, seed_nx, seed_ny, random_nx, reinterpret_cast<unsigned long long*>(a.seed), a.seed_pitch / 8,
             a.random, a.random_pitch / 4);
}

__global__ void k_xorwow_batch(const go_noise_member* __restrict__ m, int nx, int ny) {
    const go_noise_member& a = m[blockIdx.z];
    xorwow_body(1, a.n_generators, reinterpret_cast<curandStateXORWOW_t*>(a.xorwow_states), nx, ny, a.random,
                a.random_pitch / 4);
}

__global__ void __launch_bounds__(kBW* kSoarTY) k_soar_batch(const go_noise_member* __restrict__ m, int nx, int ny,
                                                             float dx, float dy, float L, double q0_scale,
                                                             float scale, int pns, int pew, int aligned16) {
    const go_noise_member& a = m[blockIdx.z];
    const float q0 = (float)((double)a.soar_q0 * q0_scale);
    soar_body(nx, ny, dx, dy, q0, L, scale, pns, pew, a.random, a.random_pitch / 4, a.coarse, a.coarse_pitch / 4, 0,
              aligned16);
}

__global__ void __launch_bounds__(kBW* kBH) k_balance_batch(const go_noise_member* __restrict__ m,
                                                            const BalanceArgs geom) {
    const go_noise_member& mm = m[blockIdx.z];
    BalanceArgs a = geom;
    a.g = mm.g;
    a.f = mm.f;
    a.beta = mm.beta;
    a.coarse = mm.coarse;
    a.cp = mm.coarse_pitch / 4;
    a.eta = mm.eta;
    a.hu = mm.hu;
    a.hv = mm.hv;
    a.pe = mm.eta_pitch / 4;
    a.pu = mm.hu_pitch / 4;
    a.pv = mm.hv_pitch / 4;
    a.Hi = mm.Hi;
    a.ph = mm.Hi_pitch / 4;
    a.land = mm.land_value;
    a.angle = (cudaTextureObject_t)mm.angle_texture;
    a.coriolis = (cudaTextureObject_t)mm.coriolis_texture;
    balance_body(a, coriolis_mode(a.f, a.beta));
}

}  // namespace

struct go_noise_batch {
    int n, nx, ny, pns, pew, use_lcg, n_gen, aligned16;
    int seed_nx, seed_ny, rand_nx, rand_ny;
    float dx, dy, L;
    BalanceArgs geom;                 // shared geometry of the balance (cells, dx, dy)
    go_noise_member* d_members;
};

extern "C" {

int go_noise_batch_create(const go_noise_member* members, int n, int nx, int ny, float dx, float dy, int ghost_x,
                          int ghost_y, float soar_L, int periodic_north_south, int periodic_east_west, int use_lcg,
                          go_noise_batch** out) {
    if (!members || !out || n < 1) return go_fail(GO_ERR_INVALID, "no members");
    if (n > 65535) return go_fail(GO_ERR_INVALID, "%d members, at most 65535", n);
    if (nx < 1 || ny < 1) return go_fail(GO_ERR_INVALID, "empty grid");
    *out = nullptr;
    const int rnx = periodic_east_west ? nx : nx + 4 * kCutoff;
    const int rny = periodic_north_south ? ny : ny + 4 * kCutoff;
    const int snx = (rnx + 1) / 2;
    int aligned = 1;
    for (int k = 0; k < n; ++k) {
        const go_noise_member& m = members[k];
        if (!m.random || !m.coarse || !m.eta || !m.hu || !m.hv || !m.Hi)
            return go_fail(GO_ERR_INVALID, "member %d: null buffer", k);
        if (!m.angle_texture || !m.coriolis_texture)
            return go_fail(GO_ERR_INVALID, "member %d: angle and Coriolis textures needed", k);
        if (use_lcg) {
            if (!m.seed || m.seed_pitch < 8 * snx || m.seed_pitch % 8)
                return go_fail(GO_ERR_INVALID, "member %d: seeds", k);
        } else if (!m.xorwow_states || m.n_generators < 1 || m.n_generators != members[0].n_generators) {
            return go_fail(GO_ERR_INVALID, "member %d: XORWOW states", k);
        }
        int rc = check_field(m.random_pitch, rnx, "random");
        if (!rc) rc = check_field(m.coarse_pitch, nx + 4, "coarse");
        if (!rc) rc = check_field(m.eta_pitch, nx + 4, "eta");
        if (!rc) rc = check_field(m.hu_pitch, nx + 4, "hu");
        if (!rc) rc = check_field(m.hv_pitch, nx + 4, "hv");
        if (!rc) rc = check_field(m.Hi_pitch, nx + 5, "Hi");
        if (rc) return rc;
        if (((uintptr_t)m.random | (uintptr_t)m.random_pitch) & 15) aligned = 0;
    }
    go_noise_batch* b = new go_noise_batch();
    b->n = n; b->nx = nx; b->ny = ny; b->pns = periodic_north_south; b->pew = periodic_east_west;
    b->use_lcg = use_lcg; b->n_gen = members[0].n_generators; b->aligned16 = aligned;
    b->seed_nx = snx; b->seed_ny = rny; b->rand_nx = rnx; b->rand_ny = rny;
    b->dx = dx; b->dy = dy; b->L = soar_L;
    const go_noise_member& m0 = members[0];
    int rc = fill_balance(b->geom, nx, ny, dx, dy, ghost_x, ghost_y, m0.g, m0.f, m0.beta, m0.coarse,
                          m0.coarse_pitch, nx + 4, m0.eta, m0.eta_pitch, m0.hu, m0.hu_pitch, m0.hv, m0.hv_pitch,
                          m0.Hi, m0.Hi_pitch, m0.land_value, m0.angle_texture, m0.coriolis_texture);
    cudaError_t e = cudaSuccess;
    if (!rc) e = cudaMalloc(&b->d_members, sizeof(go_noise_member) * n);
    if (!rc && e == cudaSuccess)
        e = cudaMemcpy(b->d_members, members, sizeof(go_noise_member) * n, cudaMemcpyHostToDevice);
    if (rc || e != cudaSuccess) {
        if (b->d_members) cudaFree(b->d_members);
        delete b;
        return rc ? rc : go_fail(GO_ERR_CUDA, "noise batch: %s", cudaGetErrorString(e));
    }
    *out = b;
    return GO_OK;
}

int go_noise_batch_destroy(go_noise_batch* b) {
    if (!b) return GO_OK;
    cudaFree(b->d_members);
    delete b;
    return GO_OK;
}

int go_noise_batch_perturb(go_noise_batch* b, void* stream, double q0_scale, float perturbation_scale,
                           int update_random_field) {
    GO_TRACE("go_noise_batch_perturb");
    if (!b) return go_fail(GO_ERR_INVALID, "null batch");
    cudaStream_t s = (cudaStream_t)stream;
    if (update_random_field) {
        if (b->use_lcg) {
            const dim3 grid((b->seed_nx + 63) / 64, (b->seed_ny + 3) / 4, b->n);
            k_lcg_batch<<<grid, dim3(64, 4), 0, s>>>(b->d_members, b->seed_nx, b->seed_ny, b->rand_nx);
        } else {
            const dim3 grid((b->n_gen + 127) / 128, 1, b->n);
            k_xorwow_batch<<<grid, 128, 0, s>>>(b->d_members, b->rand_nx, b->rand_ny);
        }
        GO_CUDA(cudaGetLastError());
    }
    const dim3 gs((b->nx + 4 + kBW - 1) / kBW, (b->ny + 4 + kSoarBH - 1) / kSoarBH, b->n);
    k_soar_batch<<<gs, dim3(kBW, kSoarTY), 0, s>>>(b->d_members, b->nx, b->ny, b->dx, b->dy, b->L, q0_scale,
                                                   perturbation_scale, b->pns, b->pew, b->aligned16);
    GO_CUDA(cudaGetLastError());
    const int ci = b->geom.i_hi - b->geom.i_lo, cj = b->geom.j_hi - b->geom.j_lo;
    if (ci > 0 && cj > 0) {
        const dim3 gb((ci + kBW - 1) / kBW, (cj + kBH * kBalRows - 1) / (kBH * kBalRows), b->n);
        k_balance_batch<<<gb, dim3(kBW, kBH), 0, s>>>(b->d_members, b->geom);
        GO_CUDA(cudaGetLastError());
    }
    return GO_OK;
}

}  // extern "C"
