// One Runge-Kutta sub-step of CDKLM16 on column pairs with packed FP32x2
// arithmetic and TMA-staged input tiles.
//
// Restates cdklm_swe_2D (gpu_ocean/SWESimulators/gpu_kernels/CDKLM16_kernel.cu:429-1006)
// followed by the periodic ghost refresh the host issues after it
// (Common.py:1219-1239 -> boundary_kernels.cu:35-110), with the same
// per-operation rounding as the reference's --ftz=true --fmad=false build.
//
// Work layout.  A block of T threads covers 2T consecutive ghost-inclusive
// columns cl0 .. cl0+2T-1 and writes the 2T-4 interior columns among them;
// thread t owns the column pair (cl0+2t, cl0+2t+1).  Every per-cell value
// is a float2 over that pair, and every add, subtract and multiply of the
// scheme issues as one sm_100 add/sub/mul.rn.ftz.f32x2 for both cells (per
// lane the same IEEE round-to-nearest, flush-to-zero result as the scalar
// instruction; no FMA contraction).  The y direction is per column, so its
// stencil (slopes, slope adjustment, G flux) works on pairs with no data
// movement; threads walk a strip of rows with the y window in registers.
// The x stencil needs the neighbouring pairs (c-1, c) and (c+1, c+2):
// cell states, slopes and face fluxes are exchanged through shared-memory
// rows stored one column to the right (slot k holds columns 2k-1 and 2k),
// so both shifted pairs load as aligned float2 without register moves.
// Each face flux is evaluated once.
//
// Inputs.  Boundary-free blocks (EDGE = false) of a TMA launch stage their
// inputs through a ring of shared-memory chunks of 3 rows: one elected
// thread issues cp.async.bulk.tensor 2-D tile loads (eta, hu, hv of rows
// j+2, corner row j+3, and Q^n of row j for stage 1) completing on an
// mbarrier per slot, kSlots-1 chunks ahead of the rows being computed.  The
// row loop is unrolled by the chunk height, so ring addresses are
// compile-time offsets and the register window rotates without moves.
// Other blocks load per lane from global memory, with wall mirroring in the
// load addresses, one row ahead.
#pragma once

#include <cuda.h>

#include "cdklm16_stage.cuh"
#include "checked.cuh"
#include "gocean.h"

namespace go {

// ---- packed FP32x2 arithmetic ---------------------------------------------
// Sums issue as FADD2 (add.rn.ftz.f32x2 under --ftz=true), differences as
// FFMA2(b, -1, a) = round(a - b), products as FFMA2(a, b, nz) with nz = -0
// taken from the kernel arguments: round(a b + (-0)) = round(a b) for every
// a, b (a zero product keeps its sign), so each lane rounds exactly as the
// scalar add/sub/mul.rn.ftz of the reference's build.  A packed multiply
// is not used because ptxas contracts mul.f32x2 followed by add.f32x2 into
// one FFMA2 (measured on a B200: 7% of a*b+c and half of 16-step x*b+c
// chains differ from the separately rounded scalar operations, with
// --fmad=false and explicit .rn), while an FMA whose addend it cannot see
// leaves nothing to contract.
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 psub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 pmul_nz(float2 a, float2 b, float2 nz) { return __ffma2_rn(a, b, nz); }
__device__ __forceinline__ float2 pb(float s) { return make_float2(s, s); }
// x * s per lane for a scalar s: two scalar multiplies that take s as an
// operand, instead of a packed one that needs s copied into a register pair
// (measured on a B200 at 4096^2 with 24-row strips: 624 -> 583 us per RK2
// step, and the region kernel no longer spills at 128 registers)
__device__ __forceinline__ float2 pscale(float2 x, float s) { return make_float2(x.x * s, x.y * s); }
__device__ __forceinline__ float2 psel(bool cx, bool cy, float2 a, float2 b) {
    return make_float2(cx ? a.x : b.x, cy ? a.y : b.y);
}

// Three-input minimum and maximum (sm_100).
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float d;
    asm("min.ftz.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float d;
    asm("max.ftz.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// minmodRaw (common.cu:544-551) per lane as max(min(b,c,f), 0) +
// min(max(b,c,f), 0): with three positive arguments the smallest, with three
// negative ones the largest, otherwise zero.  Equal to the reference's
// 0.25 s(b) (s(b)+s(c)) (s(c)+s(f)) min(|b|,|c|,|f|) up to the sign of a zero
// result; the sum adds a zero to the other term, so it is exact.
__device__ __forceinline__ float2 pminmod(float2 b, float2 c, float2 f) {
    const float2 lo = make_float2(fmaxf(fmin3(b.x, c.x, f.x), 0.0f), fmaxf(fmin3(b.y, c.y, f.y), 0.0f));
    const float2 hi = make_float2(fminf(fmax3(b.x, c.x, f.x), 0.0f), fminf(fmax3(b.y, c.y, f.y), 0.0f));
    return padd(lo, hi);
}

// minmodSlope (common.cu:532-542) per lane.
__device__ __forceinline__ float2 pslope(float2 l, float2 c, float2 r, float theta, float2 nz) {
    return pminmod(pscale(psub(c, l), theta), pscale(psub(r, l), 0.5f), pscale(psub(r, c), theta));
}

template <bool RCP>
__device__ __forceinline__ float2 prcp_or_div(float2 a, float2 b, float2 nz) {
    if (RCP) return pmul_nz(a, make_float2(rcp_approx(b.x), rcp_approx(b.y)), nz);
    return make_float2(a.x / b.x, a.y / b.y);
}

// Division by a domain constant c per lane: a / c, or a * (1/c) with 1/c hoisted.
template <bool RCP>
struct PDiv {
    float c, inv;
    float2 nz;
    __device__ __forceinline__ PDiv(float c_, float2 nz_) : c(c_), inv(RCP ? rcp_approx(c_) : 0.0f), nz(nz_) {}
    __device__ __forceinline__ float2 operator()(float2 a) const {
        if (RCP) return pscale(a, inv);
        return make_float2(a.x / c, a.y / c);
    }
};

// CDKLM16_flux (CDKLM16_kernel.cu:80-140) on two faces: per lane the face
// states (h, un, ut), un normal to the face; returns (mass, normal
// momentum, tangential momentum) fluxes.
template <bool RCP>
__device__ __forceinline__ void pflux(float2 hm, float2 um, float2 vm, float2 hp, float2 up, float2 vp,
                                      const Scheme& k, float2 nz, float2& F0, float2& F1, float2& F2) {
    auto pmul = [&](float2 x, float2 y) { return pmul_nz(x, y, nz); };
    const bool wpx = hp.x > k.cutoff, wpy = hp.y > k.cutoff;
    const bool wmx = hm.x > k.cutoff, wmy = hm.y > k.cutoff;
    const float2 z = pb(0.0f);
    const float2 hpu = pmul(hp, up);
    const float2 hmu = pmul(hm, um);
    float2 Fp0 = hpu, Fp1 = padd(pmul(hpu, up), pmul(pscale(hp, k.half_g), hp)), Fp2 = pmul(hpu, vp), upw = up;
    float2 Fm0 = hmu, Fm1 = padd(pmul(hmu, um), pmul(pscale(hm, k.half_g), hm)), Fm2 = pmul(hmu, vm), umw = um;
    const float2 gp = pscale(hp, k.g), gm = pscale(hm, k.g);
    float2 cp, cm;
    if (wpx && wpy && wmx && wmy) {
        cp = make_float2(sqrtf(gp.x), sqrtf(gp.y));
        cm = make_float2(sqrtf(gm.x), sqrtf(gm.y));
    } else {   // a dry side contributes nothing (:108-123)
        Fp0 = psel(wpx, wpy, Fp0, z); Fp1 = psel(wpx, wpy, Fp1, z); Fp2 = psel(wpx, wpy, Fp2, z);
        upw = psel(wpx, wpy, upw, z);
        Fm0 = psel(wmx, wmy, Fm0, z); Fm1 = psel(wmx, wmy, Fm1, z); Fm2 = psel(wmx, wmy, Fm2, z);
        umw = psel(wmx, wmy, umw, z);
        cp = make_float2(wpx ? sqrtf(gp.x) : 0.0f, wpy ? sqrtf(gp.y) : 0.0f);
        cm = make_float2(wmx ? sqrtf(gm.x) : 0.0f, wmy ? sqrtf(gm.y) : 0.0f);
    }
    const float2 a1 = psub(umw, cm), a2 = psub(upw, cp);
    const float2 b1 = padd(umw, cm), b2 = padd(upw, cp);
    const float2 am = make_float2(fmin3(a1.x, a2.x, 0.0f), fmin3(a1.y, a2.y, 0.0f));
    const float2 ap = make_float2(fmax3(b1.x, b2.x, 0.0f), fmax3(b1.y, b2.y, 0.0f));
    const float2 d = psub(ap, am);
    const float2 apam = pmul(ap, am);
    const float2 n0 = padd(psub(pmul(ap, Fm0), pmul(am, Fp0)), pmul(apam, psub(hp, hm)));
    const float2 n1 = padd(psub(pmul(ap, Fm1), pmul(am, Fp1)), pmul(apam, psub(Fp0, Fm0)));
    if (RCP) {
        const float2 rd = make_float2(rcp_approx(d.x), rcp_approx(d.y));
        F0 = pmul(n0, rd);
        F1 = pmul(n1, rd);
    } else {
        F0 = make_float2(n0.x / d.x, n0.y / d.y);
        F1 = make_float2(n1.x / d.x, n1.y / d.y);
    }
    const float2 s = padd(um, up);
    F2 = make_float2(s.x > 0.0f ? Fm2.x : Fp2.x, s.y > 0.0f ? Fm2.y : Fp2.y);   // upwinded tangential flux
    const bool zx = fabsf(d.x) < k.flux_slope_eps, zy = fabsf(d.y) < k.flux_slope_eps;
    if (zx || zy) {   // symmetric Riemann fan: zero flux (:128-131)
        F0 = psel(zx, zy, z, F0); F1 = psel(zx, zy, z, F1); F2 = psel(zx, zy, z, F2);
    }
}

// Face states of two faces (one float2 lane each): minus side (hm, um, vm),
// plus side (hp, up, vp); un normal, ut tangential.
struct PFace {
    float2 hm, um, vm, hp, up, vp;
};

// Cell state of one lane from conserved variables (CDKLM16_kernel.cu:551-593).
template <bool RCP, bool LAND>
__device__ __forceinline__ void cell_lane(float e, float hu, float hv, float Bm, const Scheme& k, float& pe,
                                          float& pu, float& pv) {
    const float h = e + Bm;
    if (LAND && fabsf(Bm - k.land) <= kDryEps) {
        pe = kDryFlag; pu = 0.0f; pv = 0.0f;
    } else if (h < k.desing_eps) {
        if (h <= k.cutoff) {
            pe = -Bm + k.cutoff; pu = 0.0f; pv = 0.0f;
        } else {
            pe = e;
            pu = desingularize(h, hu, k.desing_eps);
            pv = desingularize(h, hv, k.desing_eps);
        }
    } else {
        pe = e;
        pu = quot<RCP>(hu, h);
        pv = quot<RCP>(hv, h);
    }
}

// Per-row state of the register window (one column pair).
struct PRow {
    float2 e, u, v;    // reconstruction state (eta, u, v)
    float2 fu;         // Coriolis part of L_y: (east . (u', v)) f, u' flipped in wall ghost rows
    float2 Hm;         // 0.25 x corner sum of the cell (CDKLM16_kernel.cu:547)
    float2 Ha, Hb;     // corners of the corner row at (cl, cl+1) and (cl+1, cl+2)
    float2 Hy;         // y-face depth of the corner row: 0.5 (Ha + Hb)
    float f;           // Coriolis parameter of the row
};

// y-direction state carried from row j to row j+1.
struct PY {
    float2 uy, vy, Ly;     // y slopes of the row
    float2 G0, G1, G2;     // G flux (mass, hu, hv) on the face south of the row
};

// Shared memory of one block: the exchange rows and the TMA ring.
constexpr int kPairRingRows = 3;   // rows per ring chunk (= the row loop's unroll)

template <int T>
struct PairX {
    float4 st[2][T + 1];   // slot k: (e, e, u, u), (v, v, fv, fv) of columns 2k-1, 2k
    float4 sl[T + 1];      // (du, du, dv, dv)
    float2 sk[T + 1];      // (K, K)
    float4 fl[T + 1];      // (F0, F0, F1, F1) of the faces west of columns 2k-1, 2k
    float2 f2[T + 1];      // (F2, F2)
    int abort_flag;
};

// Ring chunk: 3 rows of eta, hu, hv (rows j+2), corner rows j+3 and, for
// stage 1, Q^n rows j; each array 128-byte aligned as TMA needs.
template <int T>
struct PairChunk {
    static constexpr int kQ = 3 * 2 * T;                                    // floats per field
    static constexpr int kQpad = (kQ * 4 + 127) / 128 * 128 / 4;
    static constexpr int kH = 3 * (2 * T + 4);
    static constexpr int kHpad = (kH * 4 + 127) / 128 * 128 / 4;
    static constexpr int kFloats0 = 3 * kQpad + kHpad;                       // stage 0
    static constexpr int kFloats1 = 6 * kQpad + kHpad;                       // stage 1
    static constexpr unsigned kBytes0 = (3u * kQ + kH) * 4u;                 // bytes a stage-0 chunk receives
    static constexpr unsigned kBytes1 = (6u * kQ + kH) * 4u;
};

// Tensor maps of one stage launch: eta, hu, hv of the input; Q^n (stage 1);
// the corners.  Generic addresses (kernel parameter or global memory).
struct PairMaps {
    const CUtensorMap* q[3];
    const CUtensorMap* qn[3];
    const CUtensorMap* h;
};

// Kernel-parameter copy of the maps for the single-domain launch.
struct alignas(64) PairMapParams {
    CUtensorMap q[3];
    CUtensorMap qn[3];
    CUtensorMap h;
};

// ---- mbarrier and TMA -------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// One bounded test of the phase with parity `phase`; true once it completed.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned phase) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase), "r"(1000u)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Waits are bounded: about a second of polling, after which the block sets
// GO_STATUS_TIMEOUT in the status word and abandons its strip.
constexpr int kWaitPolls = 1 << 20;
constexpr unsigned kStatusTimeout = GO_STATUS_TIMEOUT;

template <int T>
__device__ __forceinline__ void pair_sync() {
    if (T == 32) __syncwarp();
    else __syncthreads();
}

template <int T>
struct PairSmem {
    PairX<T> x;
    uint64_t bar[4];
};

// True when the column block from cl0 (2T columns) needs no wall logic: it
// reaches no ghost column of a wall side (periodic and open sides are read
// as they are; the periodic images of its cells are written after the
// stage).  Rows [4, ny) need none either.  Such strips run the TMA path.
template <int T>
__host__ __device__ __forceinline__ bool pair_fast_cols(const Scheme& k, int cl0) {
    return (k.bcW != kWall || cl0 >= 4) && (k.bcE != kWall || cl0 + 2 * T - 1 <= k.nx - 1);
}
__host__ __device__ __forceinline__ bool pair_fast_rows(const Scheme& k, int r0, int r1) {
    return r0 >= 4 && r1 <= k.ny;
}

// One block strip of the column-pair stage.
//   ring: dynamic shared memory for NS chunks (TMA launches), else null
//   chunk_base: running chunk counter of this block (mbarrier phases)
// FRIC: kFric* or -1 for the law in StageArgs::fric; WIND: 0 uniform wind,
// 1 per-cell wind field, -1 whichever StageArgs holds.  The boundary-free
// kernels fix both at compile time: deciding them at run time costs that
// kernel 10% (measured at 4096^2: 586 against 524 us per step).
template <int T, int NS, int UNR, int FRIC, int WIND, bool GEN_NORTH, bool RCP, bool LAND, bool EDGE, bool TMA>
__device__ __forceinline__ void pair_strip(const StageArgs& a, const PairMaps& maps, const float dt, const int bx,
                                           const int r0, const int r1, PairSmem<T>& sm, float* ring,
                                           unsigned& chunk_base) {
    const Scheme& k = a.k;
    const int t = threadIdx.x;
    const int cl0 = bx * (2 * T - 4);
    const int cl = cl0 + 2 * t;            // lane x column; lane y is cl + 1
    const bool stage1 = (a.rk_step == 1);
    const int fric = FRIC >= 0 ? FRIC : a.fric;                         // friction law
    const bool wind_field = WIND >= 0 ? (WIND == 1) : (a.wx_cur != nullptr);

    const float2 NZ = pb(a.neg_zero);      // -0, opaque to the compiler
    // array extents of the checked-index build (unused otherwise)
    const long long xin = ext_in(a), xout = ext_out(a), xqn = ext_qn(a), xhi = ext_hi(a), xf = ext_f(a),
                    xw = ext_w(a);
    auto pmul = [&](float2 x, float2 y) { return pmul_nz(x, y, NZ); };
    const PDiv<RCP> by2g(k.two_g, NZ);
    const PDiv<RCP> bydx(k.dx, NZ);
    const PDiv<RCP> bydy(k.dy, NZ);
    const float eX = k.nY, eY = -k.nX;      // east = (north.y, -north.x), :681

    // ---- per-lane column addressing (EDGE blocks) --------------------------
    int qcx = cl, qcy = cl + 1;
    float husx = 1.0f, husy = 1.0f;
    int hc0 = cl, hc1 = cl + 1, hc2 = cl + 2;
    // TMA path: the last column block at a periodic or open east side
    // reaches past the array.  Its prime reads those columns past the end of
    // the row, into the following rows of the same allocation (the prime
    // reads Q rows up to ny and corner rows up to ny+1, and go_prepare_pair
    // takes the TMA path only when the 4 rows below them hold the overflow);
    // the values feed only lanes that are never written nor read by a
    // written cell.  The ring's tile loads fill such columns with zeros.
    if (EDGE) {
        auto mirror_col = [&](int c, int& qc, float& s) {
            qc = min(c, k.nx + 3);
            s = 1.0f;
            if (k.bcW == kWall && c < 2) { qc = 3 - c; s = -1.0f; }
            if (k.bcE == kWall && c > k.nx + 1 && c <= k.nx + 3) { qc = 2 * k.nx + 3 - c; s = -1.0f; }
        };
        mirror_col(cl, qcx, husx);
        mirror_col(cl + 1, qcy, husy);
        hc0 = min(cl, k.nx + 4); hc1 = min(cl + 1, k.nx + 4); hc2 = min(cl + 2, k.nx + 4);
    }
    auto wallW = [&](int c) { return EDGE && k.bcW == kWall && c < 2; };
    auto wallE = [&](int c, int lim) { return EDGE && k.bcE == kWall && c > lim; };
    // Wall sign flips the reference applies by global index, per lane.
    const bool flipKx_x = wallW(cl) || wallE(cl, k.nx + 1), flipKx_y = wallW(cl + 1) || wallE(cl + 1, k.nx + 1);
    const bool flipAdjX_x = wallW(cl) || wallE(cl, k.nx + 2), flipAdjX_y = wallW(cl + 1) || wallE(cl + 1, k.nx + 2);
    const bool flipFm_x = EDGE && k.bcW == kWall && cl == 2, flipFm_y = EDGE && k.bcW == kWall && cl + 1 == 2;
    const bool flipFp_x = EDGE && k.bcE == kWall && cl == k.nx + 2, flipFp_y = EDGE && k.bcE == kWall && cl + 1 == k.nx + 2;
    auto flipLy = [&](int r) { return EDGE && ((k.bcS == kWall && r < 2) || (k.bcN == kWall && r > k.ny + 1)); };
    auto flipAdjY = [&](int r) { return EDGE && ((k.bcS == kWall && r < 2) || (k.bcN == kWall && r > k.ny + 2)); };
    const bool wr_x = (t >= 1) && (t < T - 1) && cl <= k.nx + 1;          // lane writes its cell
    const bool wr_y = (t >= 1) && (t < T - 1) && cl + 1 <= k.nx + 1;
    const bool writer = wr_x || wr_y;


    const float* __restrict__ frow = a.f_rows;

    auto mirror_row = [&](int r, float& hv_sgn) {
        hv_sgn = 1.0f;
        int rr = r;
        if (EDGE) {
            if (k.bcS == kWall && r < 2) { hv_sgn = -1.0f; rr = 3 - r; }
            else if (k.bcN == kWall && r > k.ny + 1) { hv_sgn = -1.0f; rr = 2 * k.ny + 3 - r; }
        }
        return rr;
    };
    // Q of row r for the pair, from global memory (mirrored at walls)
    auto load_q = [&](int r, float2& e, float2& hu, float2& hv) {
        float hv_sgn;
        const int rr = mirror_row(r, hv_sgn);
        const size_t o = (size_t)rr * a.pin;
        if (!EDGE && TMA) {   // 8-byte aligned pairs
            e = ldg2(a.eta_in, o + cl, xin, a.status);
            hu = ldg2(a.hu_in, o + cl, xin, a.status);
            hv = ldg2(a.hv_in, o + cl, xin, a.status);
        } else {
            e = make_float2(ldg1(a.eta_in, o + qcx, xin, a.status), ldg1(a.eta_in, o + qcy, xin, a.status));
            hu = make_float2(ldg1(a.hu_in, o + qcx, xin, a.status), ldg1(a.hu_in, o + qcy, xin, a.status));
            hv = make_float2(ldg1(a.hv_in, o + qcx, xin, a.status), ldg1(a.hv_in, o + qcy, xin, a.status));
        }
        if (EDGE) {
            hu = make_float2(hu.x * husx, hu.y * husy);
            hv = make_float2(hv.x * hv_sgn, hv.y * hv_sgn);
        }
    };
    auto land_corner = [&](float2 h) {
        if (LAND) return make_float2(corner(h.x, k), corner(h.y, k));
        return h;
    };
    // corners of corner row r: Ha = (cl, cl+1), Hb = (cl+1, cl+2)
    auto load_h = [&](int r, float2& Ha, float2& Hb) {
        const long long o = (long long)r * a.phi;
        float h2;
        if (!EDGE && TMA) {
            Ha = ldg2(a.Hi, o + cl, xhi, a.status);
            h2 = ldg1(a.Hi, o + cl + 2, xhi, a.status);
        } else {
            Ha = make_float2(ldg1(a.Hi, o + hc0, xhi, a.status), ldg1(a.Hi, o + hc1, xhi, a.status));
            h2 = ldg1(a.Hi, o + hc2, xhi, a.status);
        }
        Hb = make_float2(Ha.y, h2);
        Ha = land_corner(Ha);
        Hb = land_corner(Hb);
    };
    // cell state of a row from Q and its two corner rows
    auto to_cell = [&](float2 e, float2 hu, float2 hv, PRow& R, const PRow& Rc) {
        // R holds the corner row of the cell's south side, Rc the north one
        const float2 s = padd(padd(padd(R.Ha, Rc.Ha), R.Hb), Rc.Hb);
        R.Hm = pscale(s, 0.25f);
        float2 Bm = R.Hm;
        if (LAND) Bm = make_float2(cell_bm(R.Ha.x, Rc.Ha.x, R.Hb.x, Rc.Hb.x, s.x, k),
                                   cell_bm(R.Ha.y, Rc.Ha.y, R.Hb.y, Rc.Hb.y, s.y, k));
        const float2 h = padd(e, Bm);
        bool fast = h.x >= k.desing_eps && h.y >= k.desing_eps;
        if (LAND) fast = fast && !(fabsf(Bm.x - k.land) <= kDryEps) && !(fabsf(Bm.y - k.land) <= kDryEps);
        if (fast) {
            R.e = e;
            if (RCP) {
                const float2 rh = make_float2(rcp_approx(h.x), rcp_approx(h.y));
                R.u = pmul(hu, rh);
                R.v = pmul(hv, rh);
            } else {
                R.u = make_float2(hu.x / h.x, hu.y / h.y);
                R.v = make_float2(hv.x / h.x, hv.y / h.y);
            }
        } else {
            cell_lane<RCP, LAND>(e.x, hu.x, hv.x, Bm.x, k, R.e.x, R.u.x, R.v.x);
            cell_lane<RCP, LAND>(e.y, hu.y, hv.y, Bm.y, k, R.e.y, R.u.y, R.v.y);
        }
    };
    // Coriolis part of L_y of row r's cells (:738-758)
    auto fu_of = [&](PRow& R, int r) {
        float2 uu = R.u;
        if (EDGE && flipLy(r)) uu = make_float2(-uu.x, -uu.y);
        if (GEN_NORTH) R.fu = pscale(padd(pscale(uu, eX), pscale(R.v, eY)), R.f);
        else R.fu = pscale(uu, R.f);
    };
    // y slope (u_y, v_y, L_y) of the cells of row r = c, with neighbours lo
    // (r-1) and up (r+1); adjustSlopes_y (:198-241) with the face depths of
    // the corner rows r (south) and r+1 (north)
    auto y_slope = [&](const PRow& lo, const PRow& c, const PRow& up, const PRow& cn, int r, float2& du,
                       float2& dv, float2& L) {
        du = pslope(lo.u, c.u, up.u, k.theta, NZ);
        dv = pslope(lo.v, c.v, up.v, k.theta, NZ);
        const float2 backward = pscale(padd(psub(c.e, lo.e), pscale(padd(c.fu, lo.fu), k.U)), k.theta_g);
        const float2 central =
            pscale(padd(psub(up.e, lo.e), pscale(padd(padd(up.fu, pscale(c.fu, 2.0f)), lo.fu), k.U)), k.half_g);
        const float2 forward = pscale(padd(psub(up.e, c.e), pscale(padd(c.fu, up.fu), k.U)), k.theta_g);
        L = pminmod(backward, central, forward);
        float2 uu = c.u;
        if (EDGE && flipAdjY(r)) uu = make_float2(-uu.x, -uu.y);
        const float2 dyfu = pscale(uu, k.dy * c.f);
        const float2 q = by2g(psub(L, dyfu));
        const float2 hs = psub(padd(c.e, c.Hy), q);
        const float2 hn = padd(padd(c.e, cn.Hy), q);
        if (!(hs.x > 0.0f && hs.y > 0.0f && hn.x > 0.0f && hn.y > 0.0f)) {
            auto fix = [&](float Lv, float dyfu1, float ce, float Hs, float Hn, float hs1, float hn1) {
                Lv = (hs1 > 0.0f) ? Lv : dyfu1 + k.two_g * (ce + Hs);
                Lv = (hn1 > 0.0f) ? Lv : dyfu1 - k.two_g * (ce + Hn);
                return Lv;
            };
            L = make_float2(fix(L.x, dyfu.x, c.e.x, c.Hy.x, cn.Hy.x, hs.x, hn.x),
                            fix(L.y, dyfu.y, c.e.y, c.Hy.y, cn.Hy.y, hs.y, hn.y));
        }
    };
    // G flux on the face between rows r (lo) and r+1 (hi), corner row r+1;
    // slopes of the two rows; returns (mass, hu, hv) fluxes
    auto y_face = [&](const PRow& lo, const PRow& hi, const PRow& face_row, int r, float2 uy_lo, float2 vy_lo,
                      float2 Ly_lo, float2 uy_hi, float2 vy_hi, float2 Ly_hi, float2& G0, float2& G1, float2& G2) {
        float2 um = lo.u, up = hi.u;
        if (EDGE && k.bcS == kWall && r + 1 == 2) um = make_float2(-um.x, -um.y);
        if (EDGE && k.bcN == kWall && r + 1 == k.ny + 2) up = make_float2(-up.x, -up.y);
        if (GEN_NORTH) {
            um = padd(pscale(um, eX), pscale(lo.v, eY));
            up = padd(pscale(up, eX), pscale(hi.v, eY));
        }
        const float2 hp = psub(padd(hi.e, face_row.Hy), by2g(psub(Ly_hi, pscale(up, k.dy * hi.f))));
        const float2 hm = padd(padd(lo.e, face_row.Hy), by2g(psub(Ly_lo, pscale(um, k.dy * lo.f))));
        const float2 hp0 = make_float2(fmaxf(0.0f, hp.x), fmaxf(0.0f, hp.y));
        const float2 hm0 = make_float2(fmaxf(0.0f, hm.x), fmaxf(0.0f, hm.y));
        float2 F0, F1, F2;
        pflux<RCP>(hm0, padd(lo.v, pscale(vy_lo, 0.5f)), padd(lo.u, pscale(uy_lo, 0.5f)), hp0,
                   psub(hi.v, pscale(vy_hi, 0.5f)), psub(hi.u, pscale(uy_hi, 0.5f)), k, NZ, F0, F1, F2);
        {   // a land (dry-flag) cell on either side: zero flux (:271-273)
            const bool dx_ = hi.e.x == kDryFlag || lo.e.x == kDryFlag;
            const bool dy_ = hi.e.y == kDryFlag || lo.e.y == kDryFlag;
            if (dx_ || dy_) {
                const float2 z = pb(0.0f);
                F0 = psel(dx_, dy_, z, F0); F1 = psel(dx_, dy_, z, F1); F2 = psel(dx_, dy_, z, F2);
            }
        }
        G0 = F0; G1 = F2; G2 = F1;   // normal is v: (mass, hu tangential, hv normal)
    };

    // face states of the G flux on the face between rows r (lo) and r+1
    // (hi), corner row r+1 (face_row): lane = column, un = v, ut = u
    auto y_face_in = [&](const PRow& lo, const PRow& hi, const PRow& face_row, int r, float2 uy_lo, float2 vy_lo,
                         float2 Ly_lo, float2 uy_hi, float2 vy_hi, float2 Ly_hi) {
        float2 um = lo.u, up = hi.u;
        if (EDGE && k.bcS == kWall && r + 1 == 2) um = make_float2(-um.x, -um.y);
        if (EDGE && k.bcN == kWall && r + 1 == k.ny + 2) up = make_float2(-up.x, -up.y);
        if (GEN_NORTH) {
            um = padd(pscale(um, eX), pscale(lo.v, eY));
            up = padd(pscale(up, eX), pscale(hi.v, eY));
        }
        const float2 hp = psub(padd(hi.e, face_row.Hy), by2g(psub(Ly_hi, pscale(up, k.dy * hi.f))));
        const float2 hm = padd(padd(lo.e, face_row.Hy), by2g(psub(Ly_lo, pscale(um, k.dy * lo.f))));
        PFace F;
        F.hm = make_float2(fmaxf(0.0f, hm.x), fmaxf(0.0f, hm.y));
        F.hp = make_float2(fmaxf(0.0f, hp.x), fmaxf(0.0f, hp.y));
        F.um = padd(lo.v, pscale(vy_lo, 0.5f));
        F.vm = padd(lo.u, pscale(uy_lo, 0.5f));
        F.up = psub(hi.v, pscale(vy_hi, 0.5f));
        F.vp = psub(hi.u, pscale(uy_hi, 0.5f));
        return F;
    };
    // raw y slopes (u_y, v_y, L_y before adjustSlopes_y) of row r = c and the
    // terms of its adjustment: dyfu = dy f u', the face depths hs, hn
    auto y_slope_raw = [&](const PRow& lo, const PRow& c, const PRow& up, const PRow& cn, int r, float2& du,
                           float2& dv, float2& L, float2& dyfu, float2& hs, float2& hn) {
        du = pslope(lo.u, c.u, up.u, k.theta, NZ);
        dv = pslope(lo.v, c.v, up.v, k.theta, NZ);
        const float2 backward = pscale(padd(psub(c.e, lo.e), pscale(padd(c.fu, lo.fu), k.U)), k.theta_g);
        const float2 central =
            pscale(padd(psub(up.e, lo.e), pscale(padd(padd(up.fu, pscale(c.fu, 2.0f)), lo.fu), k.U)), k.half_g);
        const float2 forward = pscale(padd(psub(up.e, c.e), pscale(padd(c.fu, up.fu), k.U)), k.theta_g);
        L = pminmod(backward, central, forward);
        float2 uu = c.u;
        if (EDGE && flipAdjY(r)) uu = make_float2(-uu.x, -uu.y);
        dyfu = pscale(uu, k.dy * c.f);
        const float2 q = by2g(psub(L, dyfu));
        hs = psub(padd(c.e, c.Hy), q);
        hn = padd(padd(c.e, cn.Hy), q);
    };

    // ---- prime: rows r0-2 .. r0+1 and the G flux on the face (r0-1 | r0) ----
    PRow A, B, C;   // window: rows r0, r0+1, and the corner row r0+2
    PY Y;
    {
        PRow Pm2, Pm1;
        float2 e, hu, hv;
        load_h(r0 - 2, Pm2.Ha, Pm2.Hb);
        load_h(r0 - 1, Pm1.Ha, Pm1.Hb);
        load_h(r0, A.Ha, A.Hb);
        load_h(r0 + 1, B.Ha, B.Hb);
        load_h(r0 + 2, C.Ha, C.Hb);
        Pm2.f = ldg1(frow, r0 - 2, xf, a.status); Pm1.f = ldg1(frow, r0 - 1, xf, a.status);
        A.f = ldg1(frow, r0, xf, a.status); B.f = ldg1(frow, r0 + 1, xf, a.status);
        load_q(r0 - 2, e, hu, hv); to_cell(e, hu, hv, Pm2, Pm1);
        load_q(r0 - 1, e, hu, hv); to_cell(e, hu, hv, Pm1, A);
        load_q(r0, e, hu, hv);     to_cell(e, hu, hv, A, B);
        load_q(r0 + 1, e, hu, hv); to_cell(e, hu, hv, B, C);
        fu_of(Pm2, r0 - 2); fu_of(Pm1, r0 - 1); fu_of(A, r0); fu_of(B, r0 + 1);
        Pm1.Hy = pscale(padd(Pm1.Ha, Pm1.Hb), 0.5f);
        A.Hy = pscale(padd(A.Ha, A.Hb), 0.5f);
        B.Hy = pscale(padd(B.Ha, B.Hb), 0.5f);
        float2 uym1, vym1, Lym1;
        y_slope(Pm2, Pm1, A, A, r0 - 1, uym1, vym1, Lym1);
        y_slope(Pm1, A, B, B, r0, Y.uy, Y.vy, Y.Ly);
        y_face(Pm1, A, A, r0 - 1, uym1, vym1, Lym1, Y.uy, Y.vy, Y.Ly, Y.G0, Y.G1, Y.G2);
    }

    // shared-memory exchange rows; slot 0's left half and slot T's right
    // half belong to no column and hold zeros
    PairX<T>& X = sm.x;

    // ---- inputs of output row j: Q row j+2, corner row j+3, Q^n row j, f(j+2)
    float2 nq_e = pb(0.0f), nq_hu = pb(0.0f), nq_hv = pb(0.0f), nHa = pb(0.0f), nHb = pb(0.0f);
    float2 nqn_e = pb(0.0f), nqn_hu = pb(0.0f), nqn_hv = pb(0.0f);
    float nf = ldg1(frow, r0 + 2, xf, a.status);
    const bool use_ring = TMA && !EDGE;
    auto gload_row = [&](int jj) {   // global loads of the inputs of output row jj (one row ahead)
        if (jj < r1) {
            load_q(jj + 2, nq_e, nq_hu, nq_hv);
            load_h(jj + 3, nHa, nHb);
            if (stage1 && writer) {
                const size_t o = (size_t)jj * a.pqn;
                nqn_e = make_float2(ld1(a.qn_eta, o + cl, xqn, a.status), wr_y ? ld1(a.qn_eta, o + cl + 1, xqn, a.status) : 0.0f);
                nqn_hu = make_float2(ld1(a.qn_hu, o + cl, xqn, a.status), wr_y ? ld1(a.qn_hu, o + cl + 1, xqn, a.status) : 0.0f);
                nqn_hv = make_float2(ld1(a.qn_hv, o + cl, xqn, a.status), wr_y ? ld1(a.qn_hv, o + cl + 1, xqn, a.status) : 0.0f);
            }
        }
    };
    constexpr int Q_ = PairChunk<T>::kQpad, H_ = PairChunk<T>::kHpad;
    auto chunk_ptr = [&](unsigned g) { return ring + (size_t)(g % NS) * (stage1 ? PairChunk<T>::kFloats1 : PairChunk<T>::kFloats0); };
    const int nchunks = (r1 - r0 + kPairRingRows - 1) / kPairRingRows;
    int n_issued = 0;                 // thread 0: chunks of this strip whose loads are issued
    const bool skip_tma = (a.debug & GO_DEBUG_SKIP_TMA) != 0u;   // test hook: the waits run out
    auto issue_chunk = [&](int c) {   // thread 0: TMA loads of chunk c of this strip
        if (skip_tma) return;
        n_issued = c + 1;
        const unsigned g = chunk_base + (unsigned)c;
        float* base = chunk_ptr(g);
        uint64_t* bar = &sm.bar[g % NS];
        const int j0 = r0 + kPairRingRows * c;
        fence_proxy_async_smem();
        mbar_expect_tx(bar, stage1 ? PairChunk<T>::kBytes1 : PairChunk<T>::kBytes0);
        for (int f = 0; f < 3; ++f) tma_load_2d(base + f * Q_, maps.q[f], cl0, j0 + 2, bar);
        tma_load_2d(base + 3 * Q_, maps.h, cl0, j0 + 3, bar);
        if (stage1)
            for (int f = 0; f < 3; ++f) tma_load_2d(base + 3 * Q_ + H_ + f * Q_, maps.qn[f], cl0, j0, bar);
    };
    auto wait_chunk = [&](int c) {
        const unsigned g = chunk_base + (unsigned)c;
        uint64_t* bar = &sm.bar[g % NS];
        const unsigned phase = (g / NS) & 1u;
        int it = 0;
        while (!mbar_try_wait(bar, phase)) {
            if (++it >= kWaitPolls) {
                X.abort_flag = 1;
                if (a.status) atomicOr(a.status, kStatusTimeout);
                break;
            }
        }
    };
    // after a timeout, before the block leaves: thread 0 waits (bounded
    // again) for the chunks from c on whose loads it issued, so that no copy
    // lands in the shared memory of a block that has exited
    auto drain = [&](int c) {
        if (t != 0) return;
        for (int cc = c; cc < n_issued; ++cc) {
            const unsigned g = chunk_base + (unsigned)cc;
            for (int it = 0; it < kWaitPolls && !mbar_try_wait(&sm.bar[g % NS], (g / NS) & 1u); ++it) {
            }
        }
    };
    if (use_ring) {
        if (t == 0)
            for (int c = 0; c < NS - 1 && c < nchunks; ++c) issue_chunk(c);
    } else {
        gload_row(r0);
    }

    // per-launch constants of the update
    float Xw = 0.0f, Yw = 0.0f;
    if (!wind_field) {
        Xw = a.wind_t * a.wxn + (1.0f - a.wind_t) * a.wxc;
        Yw = a.wind_t * a.wyn + (1.0f - a.wind_t) * a.wyc;
    }
    const float dtr = dt * k.r;
    const float tr_dt = k.two_r * dt;

    // ---- one output row: j, window rows R0 = j, R1 = j+1, R2 <- j+2 ---------
    // ri: row of the ring chunk (0..2) for ring launches
    auto body = [&](int j, PRow& R0, PRow& R1, PRow& R2, const int ri, const int c) {
        // inputs of the row
        float2 q_e, q_hu, q_hv, qn_e = pb(0.0f), qn_hu = pb(0.0f), qn_hv = pb(0.0f);
        float2 Ha3, Hb3;
        R2.f = nf;
        if (use_ring) {
            if (ri == 0) wait_chunk(c);
            const float* base = chunk_ptr(chunk_base + (unsigned)c);
            const int o = ri * 2 * T + 2 * t;
            // shared reads of the chunk: Q rows of Q_ floats, the corner row of H_
            auto sld2 = [&](const float* p, int i, int extent) {
                return idx_ok(i, 2, extent, a.status) ? *reinterpret_cast<const float2*>(p + i)
                                                      : make_float2(0.0f, 0.0f);
            };
            q_e = sld2(base, o, Q_);
            q_hu = sld2(base + Q_, o, Q_);
            q_hv = sld2(base + 2 * Q_, o, Q_);
            const int oh = ri * (2 * T + 4) + 2 * t;
            Ha3 = sld2(base + 3 * Q_, oh, H_);
            Hb3 = make_float2(Ha3.y, idx_ok(oh + 2, 1, H_, a.status) ? base[3 * Q_ + oh + 2] : 0.0f);
            Ha3 = land_corner(Ha3);
            Hb3 = land_corner(Hb3);
            if (stage1) {
                const float* nb = base + 3 * Q_ + H_;
                qn_e = sld2(nb, o, Q_);
                qn_hu = sld2(nb + Q_, o, Q_);
                qn_hv = sld2(nb + 2 * Q_, o, Q_);
            }
            nf = ldg1(frow, min(j + 3, k.ny + 3), xf, a.status);
        } else {
            q_e = nq_e; q_hu = nq_hu; q_hv = nq_hv;
            Ha3 = nHa; Hb3 = nHb;
            qn_e = nqn_e; qn_hu = nqn_hu; qn_hv = nqn_hv;
            nf = ldg1(frow, min(j + 3, k.ny + 3), xf, a.status);
            gload_row(j + 1);
        }
        // corner row j+3 goes into the slot of row j+2's north corners: R2
        // holds corner row j+2 (loaded earlier), and the new row is kept in
        // the temporary until the next iteration makes it R0's successor
        PRow N;    // corner row j+3 (its cell data is filled two rows later)
        N.Ha = Ha3; N.Hb = Hb3;
        to_cell(q_e, q_hu, q_hv, R2, N);
        fu_of(R2, j + 2);
        R2.Hy = pscale(padd(R2.Ha, R2.Hb), 0.5f);

        // ---- publish row j's cell state for the x neighbours ----------------
        float2 vK = R0.v;
        if (EDGE) vK = make_float2(flipKx_x ? -vK.x : vK.x, flipKx_y ? -vK.y : vK.y);
        float2 fv;
        if (GEN_NORTH) fv = pscale(padd(pscale(R0.u, k.nX), pscale(vK, k.nY)), R0.f);
        else fv = pscale(vK, R0.f);
        {
            float* s0 = reinterpret_cast<float*>(&X.st[0][0]);
            float* s1 = reinterpret_cast<float*>(&X.st[1][0]);
            // column 2t -> slot t, second lanes; column 2t+1 -> slot t+1, first lanes
            s0[4 * t + 1] = R0.e.x; s0[4 * t + 3] = R0.u.x;
            s0[4 * t + 4] = R0.e.y; s0[4 * t + 6] = R0.u.y;
            s1[4 * t + 1] = R0.v.x; s1[4 * t + 3] = fv.x;
            s1[4 * t + 4] = R0.v.y; s1[4 * t + 6] = fv.y;
        }
        pair_sync<T>();
        if (use_ring && ri == 0) {
            if (X.abort_flag) {
                drain(c);
                return false;
            }
            if (t == 0 && c + NS - 1 < nchunks) issue_chunk(c + NS - 1);
        }
        const float4 L01 = X.st[0][t], L23 = X.st[1][t];          // columns (2t-1, 2t)
        const float4 R01 = X.st[0][t + 1], R23 = X.st[1][t + 1];  // columns (2t+1, 2t+2)
        const float2 Le = make_float2(L01.x, L01.y), Lu = make_float2(L01.z, L01.w);
        const float2 Lv = make_float2(L23.x, L23.y), Lfv = make_float2(L23.z, L23.w);
        const float2 Re = make_float2(R01.x, R01.y), Ru = make_float2(R01.z, R01.w);
        const float2 Rv = make_float2(R23.x, R23.y), Rfv = make_float2(R23.z, R23.w);

        // ---- x slopes of row j and y slopes of row j+1 -------------------------
        const float2 du = pslope(Lu, R0.u, Ru, k.theta, NZ);
        const float2 dv = pslope(Lv, R0.v, Rv, k.theta, NZ);
        float2 K;
        {
            const float2 backward = pscale(psub(psub(R0.e, Le), pscale(padd(fv, Lfv), k.V)), k.theta_g);
            const float2 central =
                pscale(psub(psub(Re, Le), pscale(padd(padd(Rfv, pscale(fv, 2.0f)), Lfv), k.V)), k.half_g);
            const float2 forward = pscale(psub(psub(Re, R0.e), pscale(padd(fv, Rfv), k.V)), k.theta_g);
            K = pminmod(backward, central, forward);
        }
        const float2 Hw = pscale(padd(R0.Ha, R1.Ha), 0.5f);   // x-face depth west of the cells
        const float2 He = pscale(padd(R0.Hb, R1.Hb), 0.5f);   // east
        const float dxf = k.dx * R0.f;
        // adjustSlopes_x (:148-191): K + dx f v, fallbacks 2g(..) - dx f v;
        // adjustSlopes_y (:198-241) of row j+1: L - dy f u, fallbacks dy f u +- 2g(..)
        float2 vv = R0.v;
        if (EDGE) vv = make_float2(flipAdjX_x ? -vv.x : vv.x, flipAdjX_y ? -vv.y : vv.y);
        const float2 nw = pscale(vv, dxf);
        const float2 qx = by2g(padd(K, nw));
        const float2 hw = psub(padd(R0.e, Hw), qx);
        const float2 he = padd(padd(R0.e, He), qx);
        float2 uy1, vy1, Ly1, dyfu1, hs1, hn1;
        y_slope_raw(R0, R1, R2, R2, j + 1, uy1, vy1, Ly1, dyfu1, hs1, hn1);
        if (!(hw.x > 0.0f && hw.y > 0.0f && he.x > 0.0f && he.y > 0.0f && hs1.x > 0.0f && hs1.y > 0.0f &&
              hn1.x > 0.0f && hn1.y > 0.0f)) {
            auto fixx = [&](float Kv, float nw1, float ce, float Hlo, float Hhi, float hlo, float hhi) {
                Kv = (hlo > 0.0f) ? Kv : -nw1 + k.two_g * (ce + Hlo);
                Kv = (hhi > 0.0f) ? Kv : -nw1 - k.two_g * (ce + Hhi);
                return Kv;
            };
            K = make_float2(fixx(K.x, nw.x, R0.e.x, Hw.x, He.x, hw.x, he.x),
                            fixx(K.y, nw.y, R0.e.y, Hw.y, He.y, hw.y, he.y));
            auto fixy = [&](float Lv, float dyfu, float ce, float Hs, float Hn, float hs, float hn) {
                Lv = (hs > 0.0f) ? Lv : dyfu + k.two_g * (ce + Hs);
                Lv = (hn > 0.0f) ? Lv : dyfu - k.two_g * (ce + Hn);
                return Lv;
            };
            Ly1 = make_float2(fixy(Ly1.x, dyfu1.x, R1.e.x, R1.Hy.x, R2.Hy.x, hs1.x, hn1.x),
                              fixy(Ly1.y, dyfu1.y, R1.e.y, R1.Hy.y, R2.Hy.y, hs1.y, hn1.y));
        }

        // ---- publish the x slopes of row j ------------------------------------
        {
            float* sl = reinterpret_cast<float*>(&X.sl[0]);
            float* sk = reinterpret_cast<float*>(&X.sk[0]);
            sl[4 * t + 1] = du.x; sl[4 * t + 3] = dv.x;
            sl[4 * t + 4] = du.y; sl[4 * t + 6] = dv.y;
            sk[2 * t + 1] = K.x; sk[2 * t + 2] = K.y;
        }
        pair_sync<T>();
        const float4 SL = X.sl[t];
        const float2 SK = X.sk[t];
        const float2 Ldu = make_float2(SL.x, SL.y), Ldv = make_float2(SL.z, SL.w);

        // ---- F on the faces west of the two columns (minus: (c-1, c), plus: (c, c+1))
        //      and G on the face (j | j+1), evaluated side by side
        float2 F0, F1, F2, G0, G1, G2;
        {
            float2 vmx = Lv, vpx = R0.v;
            if (EDGE) {
                vmx = make_float2(flipFm_x ? -vmx.x : vmx.x, flipFm_y ? -vmx.y : vmx.y);
                vpx = make_float2(flipFp_x ? -vpx.x : vpx.x, flipFp_y ? -vpx.y : vpx.y);
            }
            if (GEN_NORTH) {
                vmx = padd(pscale(Lu, k.nX), pscale(vmx, k.nY));
                vpx = padd(pscale(R0.u, k.nX), pscale(vpx, k.nY));
            }
            const float2 hp = psub(padd(R0.e, Hw), by2g(padd(K, pscale(vpx, dxf))));
            const float2 hm = padd(padd(Le, Hw), by2g(padd(SK, pscale(vmx, dxf))));
            PFace FX;
            FX.hp = make_float2(fmaxf(0.0f, hp.x), fmaxf(0.0f, hp.y));
            FX.hm = make_float2(fmaxf(0.0f, hm.x), fmaxf(0.0f, hm.y));
            FX.um = padd(Lu, pscale(Ldu, 0.5f));
            FX.vm = padd(Lv, pscale(Ldv, 0.5f));
            FX.up = psub(R0.u, pscale(du, 0.5f));
            FX.vp = psub(R0.v, pscale(dv, 0.5f));
            const PFace FY = y_face_in(R0, R1, R1, j, Y.uy, Y.vy, Y.Ly, uy1, vy1, Ly1);
            float2 Gn, Gt;
            // one face pair after the other: evaluated side by side the two
            // keep more values live than 128 registers hold (ptxas spills;
            // measured 672 against 635 us per 4096^2 step)
            pflux<RCP>(FX.hm, FX.um, FX.vm, FX.hp, FX.up, FX.vp, k, NZ, F0, F1, F2);
            pflux<RCP>(FY.hm, FY.um, FY.vm, FY.hp, FY.up, FY.vp, k, NZ, G0, Gn, Gt);
            G1 = Gt; G2 = Gn;   // G (mass, hu, hv): the normal momentum of a y face is hv
            // a land (dry-flag) cell on either side: zero flux (:271-273)
            const bool ax = R0.e.x == kDryFlag || Le.x == kDryFlag, ay = R0.e.y == kDryFlag || Le.y == kDryFlag;
            const bool bx_ = R1.e.x == kDryFlag || R0.e.x == kDryFlag, by_ = R1.e.y == kDryFlag || R0.e.y == kDryFlag;
            if (ax || ay || bx_ || by_) {
                const float2 z = pb(0.0f);
                F0 = psel(ax, ay, z, F0); F1 = psel(ax, ay, z, F1); F2 = psel(ax, ay, z, F2);
                G0 = psel(bx_, by_, z, G0); G1 = psel(bx_, by_, z, G1); G2 = psel(bx_, by_, z, G2);
            }
        }

        // ---- publish F, read the fluxes on the east faces --------------------------
        {
            float* fl = reinterpret_cast<float*>(&X.fl[0]);
            float* f2 = reinterpret_cast<float*>(&X.f2[0]);
            fl[4 * t + 1] = F0.x; fl[4 * t + 3] = F1.x;
            fl[4 * t + 4] = F0.y; fl[4 * t + 6] = F1.y;
            f2[2 * t + 1] = F2.x; f2[2 * t + 2] = F2.y;
        }
        pair_sync<T>();
        const float4 FE01 = X.fl[t + 1];
        const float2 FE2 = X.f2[t + 1];
        const float2 Fe0 = make_float2(FE01.x, FE01.y), Fe1 = make_float2(FE01.z, FE01.w);

        // ---- update the cells of row j (:807-1004) ------------------------------
        if (writer) {
            const float2 Hm = R0.Hm;
            const float2 fd0 = padd(bydx(psub(Fe0, F0)), bydy(psub(G0, Y.G0)));
            const float2 fd1 = padd(bydx(psub(Fe1, F1)), bydy(psub(G1, Y.G1)));
            const float2 fd2 = padd(bydx(psub(FE2, F2)), bydy(psub(G2, Y.G2)));
            // face values of eta for the bathymetry source (:706-707, :803-804)
            const float2 ttx = by2g(padd(K, pscale(R0.v, dxf)));
            const float2 tty = by2g(psub(Y.Ly, pscale(R0.u, k.dy * R0.f)));
            const float2 h = padd(R0.e, Hm);
            // (u h, v h) where the cell is deeper than the cut-off, else zero
            const float2 hu = psel(h.x > k.cutoff, h.y > k.cutoff, pmul(R0.u, h), pb(0.0f));
            const float2 hv = psel(h.x > k.cutoff, h.y > k.cutoff, pmul(R0.v, h), pb(0.0f));
            float2 stx, sty;
            const bool srcx = h.x >= k.cutoff && R0.e.x != kDryFlag;
            const bool srcy = h.y >= k.cutoff && R0.e.y != kDryFlag;
            {
                float2 Xv = pb(Xw), Yv = pb(Yw);
                if (wind_field) {
                    const size_t o = (size_t)(j - 2) * a.pw + (cl - 2);
                    auto wl = [&](const float* cur, const float* nxt, size_t oo) {
                        const float xn = ldg1(nxt, oo, xw, a.status);
                        const float xc = (cur == nxt) ? xn : ldg1(cur, oo, xw, a.status);
                        return a.wind_t * xn + (1.0f - a.wind_t) * xc;
                    };
                    Xv = make_float2(wl(a.wx_cur, a.wx_next, o), wr_y ? wl(a.wx_cur, a.wx_next, o + 1) : 0.0f);
                    Yv = make_float2(wl(a.wy_cur, a.wy_next, o), wr_y ? wl(a.wy_cur, a.wy_next, o + 1) : 0.0f);
                }
                const float2 ew = psub(R0.e, ttx), ee = padd(R0.e, ttx);
                const float2 es = psub(R0.e, tty), en = padd(R0.e, tty);
                const float2 bbx = pmul(pscale(padd(pscale(padd(ew, ee), 0.5f), Hm), k.g), psub(He, Hw));
                const float2 bby = pmul(pscale(padd(pscale(padd(es, en), 0.5f), Hm), k.g), psub(R1.Hy, R0.Hy));
                float2 corx, cory;
                if (GEN_NORTH) {
                    const float2 hu_east = padd(pscale(hu, eX), pscale(hv, eY));
                    const float2 hv_north = padd(pscale(hu, k.nX), pscale(hv, k.nY));
                    const float2 hu_east_cor = pscale(hv_north, R0.f);
                    const float2 hv_north_cor = pscale(hu_east, -R0.f);
                    const float upx = -k.nX, upy = k.nY;
                    const float rx = upy, ry = -upx;
                    corx = padd(pscale(hu_east_cor, rx), pscale(hv_north_cor, ry));
                    cory = padd(pscale(hu_east_cor, upx), pscale(hv_north_cor, upy));
                } else {
                    corx = pscale(hv, R0.f);
                    cory = pscale(hu, -R0.f);
                }
                const float2 sx = padd(padd(Xv, corx), bydx(bbx));
                const float2 sy = padd(padd(Yv, cory), bydy(bby));
                stx = psel(srcx, srcy, sx, pb(0.0f));
                sty = psel(srcx, srcy, sy, pb(0.0f));
            }
            const float2 L2 = psub(stx, fd1);
            const float2 L3 = psub(sty, fd2);

            float2 C = pb(0.0f);
            if (fric == kFricLinear) {
                C = prcp_or_div<RCP>(pb(tr_dt), h, NZ);
            } else if (fric == kFricQuad) {
                auto slow = [&](float h1, float hu1, float hv1) {
                    const float u = desingularize(h1, hu1, k.desing_eps);
                    const float v = desingularize(h1, hv1, k.desing_eps);
                    return dt * k.r * desingularize(h1, sqrtf(u * u + v * v), k.desing_eps);
                };
                if (h.x >= k.desing_eps && h.y >= k.desing_eps) {
                    float2 rh;
                    if (RCP) rh = make_float2(rcp_approx(h.x), rcp_approx(h.y));
                    float2 u, v;
                    if (RCP) { u = pmul(hu, rh); v = pmul(hv, rh); }
                    else { u = make_float2(hu.x / h.x, hu.y / h.y); v = make_float2(hv.x / h.x, hv.y / h.y); }
                    const float2 ss = padd(pmul(u, u), pmul(v, v));
                    const float2 num = pscale(make_float2(sqrtf(ss.x), sqrtf(ss.y)), dtr);
                    C = RCP ? pmul(num, rh) : make_float2(num.x / h.x, num.y / h.y);
                } else {
                    auto fast1 = [&](float h1, float hu1, float hv1) {
                        const float u = quot<RCP>(hu1, h1), v = quot<RCP>(hv1, h1);
                        return quot<RCP>(dtr * sqrtf(u * u + v * v), h1);
                    };
                    C.x = (h.x < k.desing_eps) ? slow(h.x, hu.x, hv.x) : fast1(h.x, hu.x, hv.x);
                    C.y = (h.y < k.desing_eps) ? slow(h.y, hu.y, hv.y) : fast1(h.y, hu.y, hv.y);
                }
            }
            float2 ne, nhu, nhv;
            if (!stage1) {
                ne = psub(R0.e, pscale(fd0, dt));
                const float2 den = padd(pb(1.0f), C);
                if (RCP) {
                    const float2 rden = make_float2(rcp_approx(den.x), rcp_approx(den.y));
                    nhu = pmul(padd(hu, pscale(L2, dt)), rden);
                    nhv = pmul(padd(hv, pscale(L3, dt)), rden);
                } else {
                    const float2 bu = padd(hu, pscale(L2, dt)), bv = padd(hv, pscale(L3, dt));
                    nhu = make_float2(bu.x / den.x, bu.y / den.y);
                    nhv = make_float2(bv.x / den.x, bv.y / den.y);
                }
            } else {
                ne = pscale(padd(qn_e, psub(R0.e, pscale(fd0, dt))), 0.5f);
                const float2 den = padd(pb(1.0f), pscale(C, 0.5f));
                const float2 bu = pscale(padd(qn_hu, padd(hu, pscale(L2, dt))), 0.5f);
                const float2 bv = pscale(padd(qn_hv, padd(hv, pscale(L3, dt))), 0.5f);
                if (RCP) {
                    const float2 rden = make_float2(rcp_approx(den.x), rcp_approx(den.y));
                    nhu = pmul(bu, rden);
                    nhv = pmul(bv, rden);
                } else {
                    nhu = make_float2(bu.x / den.x, bu.y / den.y);
                    nhv = make_float2(bv.x / den.x, bv.y / den.y);
                }
            }
            const float2 lim = psub(pb(k.cutoff), Hm);   // -Hm + cutoff
            const float2 hn = padd(ne, Hm);
            const bool dryx = hn.x <= k.cutoff, dryy = hn.y <= k.cutoff;
            if (dryx || dryy) {
                ne = psel(dryx, dryy, lim, ne);
                nhu = psel(dryx, dryy, pb(0.0f), nhu);
                nhv = psel(dryx, dryy, pb(0.0f), nhv);
            }
            ne = make_float2(fmaxf(lim.x, ne.x), fmaxf(lim.y, ne.y));
            const float2 chk = padd(padd(ne, nhu), nhv);
            if (a.status && ((wr_x && !isfinite(chk.x)) || (wr_y && !isfinite(chk.y)))) atomicOr(a.status, 1u);

            const size_t o = (size_t)j * a.pout + cl;
            if (!EDGE && TMA) {
                if (wr_y) {
                    st2(a.eta_out, o, ne, xout, a.status);
                    st2(a.hu_out, o, nhu, xout, a.status);
                    st2(a.hv_out, o, nhv, xout, a.status);
                } else {   // the last written column of the grid is this pair's first
                    st1(a.eta_out, o, ne.x, xout, a.status);
                    st1(a.hu_out, o, nhu.x, xout, a.status);
                    st1(a.hv_out, o, nhv.x, xout, a.status);
                }
            } else {
                auto put = [&](int col, float e1, float u1, float v1) {
                    const size_t oo = (size_t)j * a.pout + col;
                    st1(a.eta_out, oo, e1, xout, a.status);
                    st1(a.hu_out, oo, u1, xout, a.status);
                    st1(a.hv_out, oo, v1, xout, a.status);
                    if (EDGE) {
                        // periodic ghost images (the reference's BC kernels after the stage)
                        int rows_img[2] = {-1, -1}, cols_img[2] = {-1, -1};
                        if (k.bcN == kPeriodic) {
                            if (j < 4) rows_img[0] = j + k.ny;
                            if (j >= k.ny) rows_img[1] = j - k.ny;
                        }
                        if (k.bcE == kPeriodic) {
                            if (col < 4) cols_img[0] = col + k.nx;
                            if (col >= k.nx) cols_img[1] = col - k.nx;
                        }
                        if (rows_img[0] >= 0 || rows_img[1] >= 0 || cols_img[0] >= 0 || cols_img[1] >= 0) {
                            const int rr[3] = {j, rows_img[0], rows_img[1]};
                            const int cc[3] = {col, cols_img[0], cols_img[1]};
                            for (int ri2 = 0; ri2 < 3; ++ri2) {
                                for (int ci = 0; ci < 3; ++ci) {
                                    if ((ri2 == 0 && ci == 0) || rr[ri2] < 0 || cc[ci] < 0) continue;
                                    const size_t o2 = (size_t)rr[ri2] * a.pout + cc[ci];
                                    st1(a.eta_out, o2, e1, xout, a.status);
                                    st1(a.hu_out, o2, u1, xout, a.status);
                                    st1(a.hv_out, o2, v1, xout, a.status);
                                }
                            }
                        }
                    }
                };
                if (wr_x) put(cl, ne.x, nhu.x, nhv.x);
                if (wr_y) put(cl + 1, ne.y, nhu.y, nhv.y);
            }
        }
        // ---- carry the y state to row j+1; the new corner row -------------------
        Y.uy = uy1; Y.vy = vy1; Y.Ly = Ly1;
        Y.G0 = G0; Y.G1 = G1; Y.G2 = G2;
        R0.Ha = N.Ha; R0.Hb = N.Hb;   // R0's slot becomes row j+3 next: its south corners are row j+3
        return true;
    };

    // rows: the window slots rotate A -> B -> C; R0's corners are replaced by
    // those of corner row j+3 at the end of each body, which is the south
    // corner row of the row the slot holds next (j+3)
    int j = r0;
    int c = 0;
    if (UNR == 3) {
        for (; j + 2 < r1; j += 3, ++c) {
            if (!body(j, A, B, C, 0, c)) return;
            if (!body(j + 1, B, C, A, 1, c)) return;
            if (!body(j + 2, C, A, B, 2, c)) return;
        }
        if (j < r1) {
            if (!body(j, A, B, C, 0, c)) return;
            if (j + 1 < r1) {
                if (!body(j + 1, B, C, A, 1, c)) return;
            }
        }
    } else if (UNR == 2) {
        // two rows per iteration, the window rotated once per iteration
        int ri = 0;
#pragma unroll 1
        for (; j + 1 < r1; j += 2) {
            if (!body(j, A, B, C, ri, c)) return;
            if (++ri == kPairRingRows) { ri = 0; ++c; }
            if (!body(j + 1, B, C, A, ri, c)) return;
            if (++ri == kPairRingRows) { ri = 0; ++c; }
            const PRow t0 = A;
            A = C;
            C = B;
            B = t0;
        }
        if (j < r1) {
            if (!body(j, A, B, C, ri, c)) return;
        }
    } else {
        // one row per iteration: a third of the code, the window moved in registers
        int ri = 0;
#pragma unroll 1
        for (; j < r1; ++j) {
            if (!body(j, A, B, C, ri, c)) return;
            const PRow t0 = A;
            A = B;
            B = C;
            C = t0;
            if (++ri == kPairRingRows) { ri = 0; ++c; }
        }
    }
    if (use_ring) chunk_base += (unsigned)nchunks;
}

}  // namespace go

namespace go {

// Zeroes the exchange rows (the halves of slots 0 and T that belong to no
// column stay zero) and initialises the ring's mbarriers.
template <int T, int NS>
__device__ __forceinline__ void pair_init(PairSmem<T>& sm) {
    float* p = reinterpret_cast<float*>(&sm.x);
    for (int i = threadIdx.x; i < (int)(sizeof(PairX<T>) / sizeof(float)); i += T) p[i] = 0.0f;
    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; ++s) mbar_init(&sm.bar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
}

// Dynamic shared memory of the ring: NS chunks (stage 0 needs no Q^n).
template <int T>
constexpr size_t pair_ring_bytes(int ns, int rk_step) {
    return (size_t)ns * (rk_step ? PairChunk<T>::kFloats1 : PairChunk<T>::kFloats0) * sizeof(float);
}

// Block grid of one stage launch.  The region, column blocks [bx0, bx1)
// over rows [4, ny), runs the TMA path in strips of `rows` rows (the last
// one shorter); it reaches the ghost columns of periodic and open sides,
// not those of walls.  The frame runs the boundary path in strips of rf
// rows: the column blocks left of bx0 and right of bx1 (wall sides) over
// every row, and the two rows next to the north and south ghost rows of the
// region's column blocks.
struct PairGrid {
    int nbx, bx0, bx1;
    int rows, nby;             // nby: strips of rows [4, ny)
    int rf;                    // rows per strip of the frame blocks (>= 2)
    int ny;
};

__host__ __device__ inline int pair_frame_strips(const PairGrid& g, int& nfull, int& full, int& nband) {
    full = (g.ny + g.rf - 1) / g.rf;
    nfull = g.bx0 + (g.nbx - g.bx1);
    nband = g.bx1 - g.bx0;
    return nfull * full + nband * 2;
}

// Frame block idx: its column block and row range.
__host__ __device__ inline void pair_frame_block(const PairGrid& g, int idx, int& bx, int& r0, int& r1) {
    int nfull, full, nband;
    pair_frame_strips(g, nfull, full, nband);
    if (idx < nfull * full) {
        const int c = idx / full, s = idx % full;
        bx = c < g.bx0 ? c : g.bx1 + (c - g.bx0);
        r0 = 2 + s * g.rf;
        r1 = min(r0 + g.rf, g.ny + 2);
        return;
    }
    idx -= nfull * full;
    bx = g.bx0 + (idx >> 1);
    if ((idx & 1) == 0) { r0 = 2; r1 = 4; }
    else { r0 = g.ny; r1 = g.ny + 2; }
}

// The stage over one part of the block grid.  PART 0: the region of TMA
// strips, column block bx0 + blockIdx.x, strip blockIdx.y; PART 1: the
// boundary frame (blockIdx.x numbers its strips), per-lane loads with wall
// mirroring and periodic images.  The parts are separate
// kernels so that the boundary-free one is compiled, and given registers,
// without the boundary logic; they write disjoint cells and run
// concurrently.
template <int T, int MINB, int NS, int UNR, int FRIC, int WIND, bool GEN_NORTH, bool RCP, bool LAND, int PART>
__global__ void __launch_bounds__(T, MINB)
    cdklm_pair_kernel(const StageArgs a, const __grid_constant__ PairMapParams mp, const PairGrid g) {
    __shared__ PairSmem<T> sm;
    extern __shared__ __align__(128) float pair_ring[];
    pair_init<T, NS>(sm);
    const PairMaps maps{{&mp.q[0], &mp.q[1], &mp.q[2]}, {&mp.qn[0], &mp.qn[1], &mp.qn[2]}, &mp.h};
    unsigned chunk_base = 0;
    if (PART == 0) {
        const int r0 = 4 + (int)blockIdx.y * g.rows;
        const int r1 = min(r0 + g.rows, a.k.ny);
        pair_strip<T, NS, UNR, FRIC, WIND, GEN_NORTH, RCP, LAND, false, true>(a, maps, a.dt, g.bx0 + blockIdx.x, r0,
                                                                              r1, sm, pair_ring, chunk_base);
    } else {
        int bx, r0, r1;
        pair_frame_block(g, blockIdx.x, bx, r0, r1);
        pair_strip<T, NS, UNR, FRIC, WIND, GEN_NORTH, RCP, LAND, true, false>(a, maps, a.dt, bx, r0, r1, sm,
                                                                              pair_ring, chunk_base);
    }
}

// Makes a tensor map that the host copied to global memory visible to the
// TMA unit before its first use (the maps of a batch live in device memory).
__device__ __forceinline__ void tensormap_acquire(const CUtensorMap* m) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(m) : "memory");
}

// Batched column-pair stage: a packed list of (member, column block, first
// row, end row) tiles over every member, walked by a persistent grid.  args
// and maps hold two entries per member (stage 0: h0 -> h1, stage 1: h1 ->
// h0); dts holds the member's time step, read at launch so a captured graph
// picks up new values.  PART 0 tiles take the TMA path with the member's
// maps, PART 1 tiles the boundary path.
template <int T, int MINB, int NS, int UNR, int FRIC, int WIND, bool GEN_NORTH, bool RCP, bool LAND, int PART>
__global__ void __launch_bounds__(T, MINB)
    cdklm_pair_batch_kernel(const StageArgs* __restrict__ args, const float* __restrict__ dts,
                            const int4* __restrict__ tiles, const int ntiles, const int rk_step,
                            const PairMapParams* __restrict__ maps) {
    __shared__ PairSmem<T> sm;
    extern __shared__ __align__(128) float pair_ring[];
    pair_init<T, NS>(sm);
    unsigned chunk_base = 0;
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const int4 tile = tiles[ti];
        const int e = 2 * tile.x + rk_step;
        const StageArgs& a = args[e];
        if (PART == 0) {
            const PairMapParams& p = maps[e];
            const PairMaps m{{&p.q[0], &p.q[1], &p.q[2]}, {&p.qn[0], &p.qn[1], &p.qn[2]}, &p.h};
            if (threadIdx.x == 0) {
                for (int f = 0; f < 3; ++f) tensormap_acquire(m.q[f]);
                if (rk_step == 1)
                    for (int f = 0; f < 3; ++f) tensormap_acquire(m.qn[f]);
                tensormap_acquire(m.h);
            }
            pair_strip<T, NS, UNR, FRIC, WIND, GEN_NORTH, RCP, LAND, false, true>(
                a, m, __ldg(dts + tile.x), tile.y, tile.z, tile.w, sm, pair_ring, chunk_base);
        } else {
            const PairMaps m{};
            pair_strip<T, NS, UNR, FRIC, WIND, GEN_NORTH, RCP, LAND, true, false>(a, m, __ldg(dts + tile.x), tile.y,
                                                                                  tile.z, tile.w, sm, pair_ring,
                                                                                  chunk_base);
        }
        __syncthreads();
        if (sm.x.abort_flag) break;
    }
}

}  // namespace go
