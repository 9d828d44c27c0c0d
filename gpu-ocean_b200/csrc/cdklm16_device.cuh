// Device arithmetic of the CDKLM16 scheme (Chertock, Dudzinski, Kurganov &
// Lukacova-Medvidova 2016), restated from gpu-ocean's kernel:
//   gpu_ocean/SWESimulators/gpu_kernels/CDKLM16_kernel.cu  (flux, slopes, sources)
//   gpu_ocean/SWESimulators/gpu_kernels/common.cu          (minmod, desingularize)
// Every expression keeps the reference's operand order so that, compiled
// with the reference's flags (--ftz=true --prec-div=false --prec-sqrt=false
// --fmad=false), each operation rounds as the reference's does.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace go {

constexpr float kDryFlag = 1.0e-30f;  // CDKLM16_kernel.cu:38
constexpr float kDryEps = 1.0e-3f;    // CDKLM16_kernel.cu:39
constexpr int kWall = 1;
constexpr int kPeriodic = 2;

// Scheme constants of one domain.  Products the reference folds at compile
// time from its #defines (THETA*GRAV, DX/(2*GRAV), ...) are folded on the
// host in IEEE float32, which is what constant folding produces.
struct Scheme {
    int nx, ny;
    float dx, dy, g, r, theta;
    float desing_eps, flux_slope_eps, cutoff, land;
    float nX, nY;          // north vector (sin a, cos a)
    int bcN, bcE, bcS, bcW;
    // host-folded constants
    float two_g;           // 2.0f*GRAV
    float half_g;          // 0.5f*GRAV
    float theta_g;         // THETA*GRAV
    float V;               // DX/(2.0f*GRAV)   (CDKLM16_kernel.cu:654)
    float U;               // DY/(2.0f*GRAV)   (CDKLM16_kernel.cu:760)
    float two_r;           // 2.0f*FRIC (linear friction)
};

struct Prim { float e, u, v; };     // reconstruction state (eta, u, v)
struct Slp { float du, dv, K; };    // (u', v', K) slopes along one axis
struct F3 { float a, b, c; };

// minmod of three differences, common.cu:544-551.  The reference writes it
// as 0.25*s(b)*(s(b)+s(c))*(s(c)+s(f))*min(|b|,|c|,|f|) with s = copysign(1,.)
// which equals s(b)*min(...) when the three signs agree and zero otherwise
// (the two forms differ at most in the sign of a zero result).
__device__ __forceinline__ float minmod_raw(float b, float c, float f) {
    const float m = fminf(fminf(fabsf(b), fabsf(c)), fabsf(f));
    const uint32_t sb = __float_as_uint(b), sc = __float_as_uint(c), sf = __float_as_uint(f);
    const bool same = (((sb ^ sc) | (sc ^ sf)) & 0x80000000u) == 0u;
    return same ? copysignf(m, b) : 0.0f;
}

// common.cu:532-542
__device__ __forceinline__ float minmod_slope(float l, float c, float r, float theta) {
    const float backward = (c - l) * theta;
    const float central = (r - l) * 0.5f;
    const float forward = (r - c) * theta;
    return minmod_raw(backward, central, forward);
}

// common.cu:822-824.  0.5*eps is a double literal there; keep the promotion.
__device__ __forceinline__ float desingularize(float h, float hu, float eps) {
    const float a = (float)((double)(h * h / (2.0f * eps)) + 0.5 * (double)eps);
    return hu / fmaxf(fminf(a, eps), fabsf(h));
}

__device__ __forceinline__ float rcp_approx_f(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// CDKLM16_flux, CDKLM16_kernel.cu:80-140.  Face states are (h, u, v).  RCP:
// the two quotients by (ap - am) share one reciprocal.
template <bool RCP>
__device__ __forceinline__ F3 central_upwind(float hm, float um, float vm,
                                             float hp, float up, float vp,
                                             const Scheme& k) {
    float Fp0 = 0.0f, Fp1 = 0.0f, Fp2 = 0.0f, upw = 0.0f, cp = 0.0f;
    if (hp > k.cutoff) {
        Fp0 = hp * up;
        Fp1 = hp * up * up + k.half_g * hp * hp;
        Fp2 = hp * up * vp;
        upw = up;
        cp = sqrtf(k.g * hp);
    }
    float Fm0 = 0.0f, Fm1 = 0.0f, Fm2 = 0.0f, umw = 0.0f, cm = 0.0f;
    if (hm > k.cutoff) {
        Fm0 = hm * um;
        Fm1 = hm * um * um + k.half_g * hm * hm;
        Fm2 = hm * um * vm;
        umw = um;
        cm = sqrtf(k.g * hm);
    }
    const float am = fminf(fminf(umw - cm, upw - cp), 0.0f);
    const float ap = fmaxf(fmaxf(umw + cm, upw + cp), 0.0f);
    if (fabsf(ap - am) < k.flux_slope_eps) return F3{0.0f, 0.0f, 0.0f};
    F3 F;
    if (RCP) {
        const float rd = rcp_approx_f(ap - am);
        F.a = ((ap * Fm0 - am * Fp0) + ap * am * (hp - hm)) * rd;
        F.b = ((ap * Fm1 - am * Fp1) + ap * am * (Fp0 - Fm0)) * rd;
    } else {
        F.a = ((ap * Fm0 - am * Fp0) + ap * am * (hp - hm)) / (ap - am);
        F.b = ((ap * Fm1 - am * Fp1) + ap * am * (Fp0 - Fm0)) / (ap - am);
    }
    F.c = (um + up > 0.0f) ? Fm2 : Fp2;
    return F;
}

// Cell state from conserved variables, CDKLM16_kernel.cu:551-593.  Bm is
// the cell's mean bathymetry (initBm), used for the land and dry tests.
__device__ __forceinline__ Prim to_prim(float eta, float hu, float hv, float Bm,
                                        const Scheme& k) {
    Prim p;
    const float h = eta + Bm;
    if (fabsf(Bm - k.land) <= kDryEps) {
        p.e = kDryFlag; p.u = 0.0f; p.v = 0.0f;
    } else if (h < k.desing_eps) {
        if (h <= k.cutoff) {
            p.e = -Bm + k.cutoff; p.u = 0.0f; p.v = 0.0f;
        } else {
            p.e = eta;
            p.u = desingularize(h, hu, k.desing_eps);
            p.v = desingularize(h, hv, k.desing_eps);
        }
    } else {
        p.e = eta; p.u = hu / h; p.v = hv / h;
    }
    return p;
}

// Corner bathymetry with land replaced by the dry flag (CDKLM16_kernel.cu:520).
__device__ __forceinline__ float corner(float H, const Scheme& k) {
    return (fabsf(H - k.land) < kDryEps) ? kDryFlag : H;
}

// initBm (initBm_kernel.cu:87-104) for corners a=(j,i) b=(j+1,i) c=(j,i+1)
// d=(j+1,i+1), already dry-flagged, and s = ((a + b) + c) + d, the plain
// corner sum whose quarter is the kernel's own-cell Hm (CDKLM16_kernel.cu:547).
// The reference builds initBm_kernel.cu with nvcc's default options
// (Common.py:1376 passes no compile flags), so its s / wet is the IEEE
// round-to-nearest quotient, not the approximate division the CDKLM16
// kernel's --prec-div=false gives: __fdiv_rn keeps that rounding (they
// differ by an ulp for some sums over 3 wet corners).
__device__ __forceinline__ float cell_bm(float a, float b, float c, float d, float s,
                                         const Scheme& k) {
    const float wet = 4.0f - (float)(a == kDryFlag) - (float)(b == kDryFlag)
                    - (float)(c == kDryFlag) - (float)(d == kDryFlag);
    if (wet == 4.0f) return s * 0.25f;   // s/4 is exact scaling
    if (wet == 0.0f) return k.land;
    return __fdiv_rn(s, wet);
}

// Cell-mean bathymetry of one cell from its four corners (initBm_kernel.cu:
// 87-104): land corners are dry, the mean over the wet ones, the land value
// when all four are land.  Shared by the bathymetry set-up and the batched
// CFL reduction, so both give the same float.
__device__ __forceinline__ float cell_mean_depth(float a, float b, float c, float d, float land) {
    auto dry = [&](float v) { return (fabsf(v - land) <= kDryEps) ? kDryFlag : v; };
    a = dry(a); b = dry(b); c = dry(c); d = dry(d);
    const float wet = 4.0f - (float)(a == kDryFlag) - (float)(b == kDryFlag) - (float)(c == kDryFlag) -
                      (float)(d == kDryFlag);
    return (wet == 0.0f) ? land : __fdiv_rn(a + b + c + d, wet);   // IEEE quotient, as cell_bm
}

constexpr float kRefFltMax = 100000.0f;   // max_dt.cu:30 redefines FLT_MAX

// CFL limit of one interior cell (max_dt.cu:42-107): min of 0.25 dx/|u +- c|
// and 0.25 dy/|v +- c|; `none` for a dry or land cell.  The reference builds
// max_dt.cu with nvcc's default options (CDKLM16.py:221 passes no compile
// flags): its quotients and square root are IEEE round-to-nearest, kept here
// with __fdiv_rn / __fsqrt_rn whatever this library's own flags are.
__device__ __forceinline__ float cell_cfl_dt(float e, float hu, float hv, float H, float dx, float dy, float g,
                                             float land, float none) {
    const float h = e + H;
    if (h <= 0.0f || fabsf(H - land) < kDryEps) return none;
    const float u = __fdiv_rn(hu, h);
    const float v = __fdiv_rn(hv, h);
    const float c = __fsqrt_rn(g * h);
    float d = __fdiv_rn(0.25f * dx, fabsf(u + c));
    d = fminf(d, __fdiv_rn(0.25f * dx, fabsf(u - c)));
    d = fminf(d, __fdiv_rn(0.25f * dy, fabsf(v + c)));
    d = fminf(d, __fdiv_rn(0.25f * dy, fabsf(v - c)));
    return d;
}

// Block minimum of a positive float, then atomicMin on its bit pattern
// (positive floats order like their bits).  Every thread of the block calls.
__device__ __forceinline__ void block_min_to(float best, unsigned int* out, float none) {
    for (int off = 16; off > 0; off >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, off));
    __shared__ float warp_min[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_min[w] = best;
    __syncthreads();
    if (w == 0) {
        best = (lane < (int)(blockDim.x >> 5)) ? warp_min[lane] : none;
        for (int off = 16; off > 0; off >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, off));
        if (lane == 0) atomicMin(out, __float_as_uint(best));
    }
}

}  // namespace go
