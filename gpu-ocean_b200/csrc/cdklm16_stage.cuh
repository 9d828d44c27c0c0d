// One Runge-Kutta sub-step of CDKLM16 as a column-marching stencil.
//
// Restates cdklm_swe_2D (gpu_ocean/SWESimulators/gpu_kernels/CDKLM16_kernel.cu:429-1006)
// followed by the periodic ghost refresh the host issues after it
// (Common.py:1219-1239 -> boundary_kernels.cu:35-110).
//
// Work layout.  A block of BW threads covers BW consecutive ghost-inclusive
// columns cl = c0-2 .. c0+BW-3 and writes the BW-4 interior columns
// c0 .. c0+BW-5.  Each thread owns one column and marches down the block's
// strip of rows [r0, r1).  The y direction (slopes u_y, v_y, L_y, G fluxes)
// lives in registers as a sliding window of rows; the x direction (slopes
// u_x, v_x, K_x, F fluxes) is exchanged between neighbouring threads through
// three shared-memory row buffers of float4.  Each face flux is evaluated
// once (the reference evaluates every face twice, once per adjacent cell).
//
// Paired arithmetic.  At row j the x-direction work of row j and the
// y-direction work of row j+1 have the same shape (slopes, slope
// adjustment, central-upwind flux), so they run side by side as the two
// lanes of float2 values, evaluated as two scalar operations per pair.
// (Built with GO_PACKED_PAIRS, sums and differences issue as packed
// add/sub.rn.ftz.f32x2 instead, per lane the same IEEE round-to-nearest,
// flush-to-zero result as the scalar operation.  Measured at 4096^2 on a
// B200 that build executes as many instructions per cell, 601 against 600:
// the 52 additions per cell it saves come back as register moves that
// assemble the operand pairs, and it runs 4% slower, so it is off by
// default.)  In the
// flux, lane x carries (u normal, v tangential) and lane y (v normal, u
// tangential), which is how the reference swaps u and v for the G flux
// (CDKLM16_kernel.cu:361-369).  Signs: a - b*c is written a + (-b)*c, which
// IEEE arithmetic rounds identically.
//
// Ghost cells: walls are mirrored on load (as handleWallBC,
// CDKLM16_kernel.cu:373-424, does in shared memory); periodic sides read the
// ghost cells of the input, which the previous stage refreshed.  Blocks that
// touch no boundary (EDGE = false) compile without any of that logic.
//
// RCP selects how a quotient a/b is evaluated: false keeps the '/' of the
// reference source (div.full.f32 under --prec-div=false); true evaluates
// a * rcp.approx.ftz(b) with reciprocals of shared denominators hoisted.
#pragma once

#include "cdklm16_device.cuh"
#include "checked.cuh"

namespace go {

struct StageArgs {
    Scheme k;
    float dt;
    int rk_step;                 // 0: Q* = Q + dt L(Q);  1: Heun average
    const float* eta_in; const float* hu_in; const float* hv_in;
    int pin;                     // pitch of the inputs, floats
    float* eta_out; float* hu_out; float* hv_out;
    int pout;                    // pitch of the outputs, floats
    // Q^n read by stage 1 at each cell: the output buffer itself (the
    // reference's in-place update) unless a separate state is given
    const float* qn_eta; const float* qn_hu; const float* qn_hv;
    int pqn;
    const float* Hi; int phi;    // corners (ny+5) x (nx+5)
    const float* f_rows;         // Coriolis per ghost-inclusive row
    float wind_t, wxc, wxn, wyc, wyn;
    const float* wx_cur; const float* wx_next;
    const float* wy_cur; const float* wy_next; int pw;  // interior-indexed
    int rows_per_block;
    unsigned int* status;
    float neg_zero;              // -0.0f: the addend of the packed products (column-pair kernel)
    int fric;                    // friction law kFric* (column-pair kernel; the marching kernel has it as a template)
    unsigned debug;              // GO_DEBUG_* test hooks (go_domain_set_debug), 0 in normal runs
};

// Friction law selector.
enum { kFricNone = 0, kFricQuad = 1, kFricLinear = 2 };

__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <bool RCP>
__device__ __forceinline__ float quot(float a, float b) {
    if (RCP) return a * rcp_approx(b);
    return a / b;
}

// ---- paired float2 helpers -----------------------------------------------
// Default: each lane is a scalar add.rn.ftz / mul.rn.ftz, as the reference's
// --ftz=true --fmad=false build computes it.  GO_PACKED_PAIRS: sums and
// differences run as packed add/sub.rn.ftz.f32x2 (per lane the same IEEE
// round-to-nearest result with subnormals flushed).  Products stay two
// scalar multiplies in both builds: ptxas may contract a packed multiply
// feeding a packed add into a fused FFMA2 (observed on sm_100a even with
// explicit .rn and -fmad=false), which would round differently from the
// reference, while a scalar product cannot be fused into a packed add.
__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
#ifndef GO_PACKED_PAIRS
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return f2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return f2(a.x - b.x, a.y - b.y); }
#else
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.ftz.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.ftz.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
#endif
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return f2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ float2 neg2(float2 a) { return f2(-a.x, -a.y); }
__device__ __forceinline__ float2 sel2(bool cx, bool cy, float2 a, float2 b) {
    return f2(cx ? a.x : b.x, cy ? a.y : b.y);
}

template <bool RCP>
__device__ __forceinline__ float2 quot2(float2 a, float2 b) {
    if (RCP) return mul2(a, f2(rcp_approx(b.x), rcp_approx(b.y)));
    return f2(a.x / b.x, a.y / b.y);
}

// minmod of three differences per lane (common.cu:544-551; see minmod_raw).
__device__ __forceinline__ float2 minmod2(float2 b, float2 c, float2 f) {
    return f2(minmod_raw(b.x, c.x, f.x), minmod_raw(b.y, c.y, f.y));
}

// minmodSlope per lane (common.cu:532-542)
__device__ __forceinline__ float2 minmod_slope2(float2 l, float2 c, float2 r, float2 theta) {
    const float2 backward = mul2(sub2(c, l), theta);
    const float2 central = mul2(sub2(r, l), f2(0.5f, 0.5f));
    const float2 forward = mul2(sub2(r, c), theta);
    return minmod2(backward, central, forward);
}

// CDKLM16_flux (CDKLM16_kernel.cu:101-140) on two faces at once.  Per lane
// the face states are (h, un, ut) with un the velocity normal to the face;
// returns (mass, normal momentum, tangential momentum) fluxes per lane.
template <bool RCP>
__device__ __forceinline__ void central_upwind2(float2 hm, float2 um, float2 vm, float2 hp, float2 up,
                                                float2 vp, const Scheme& k, float2& F0, float2& F1,
                                                float2& F2) {
    const bool wpx = hp.x > k.cutoff, wpy = hp.y > k.cutoff;
    const bool wmx = hm.x > k.cutoff, wmy = hm.y > k.cutoff;
    const float2 hg = f2(k.half_g, k.half_g);
    const float2 g2 = f2(k.g, k.g);
    const float2 z = f2(0.0f, 0.0f);
    // F = (h u, h u u + 0.5 g h h, h u v), CDKLM16_kernel.cu:80-88
    const float2 hpu = mul2(hp, up);
    const float2 hmu = mul2(hm, um);
    float2 Fp0 = hpu, Fp1 = add2(mul2(hpu, up), mul2(mul2(hg, hp), hp)), Fp2 = mul2(hpu, vp), upw = up;
    float2 Fm0 = hmu, Fm1 = add2(mul2(hmu, um), mul2(mul2(hg, hm), hm)), Fm2 = mul2(hmu, vm), umw = um;
    const float2 gp = mul2(g2, hp), gm = mul2(g2, hm);
    float2 cp, cm;
    if (wpx && wpy && wmx && wmy) {   // all four face states wet: no selection needed
        cp = f2(sqrtf(gp.x), sqrtf(gp.y));
        cm = f2(sqrtf(gm.x), sqrtf(gm.y));
    } else {                          // a dry side contributes nothing (:108-123)
        Fp0 = sel2(wpx, wpy, Fp0, z); Fp1 = sel2(wpx, wpy, Fp1, z); Fp2 = sel2(wpx, wpy, Fp2, z);
        upw = sel2(wpx, wpy, upw, z);
        Fm0 = sel2(wmx, wmy, Fm0, z); Fm1 = sel2(wmx, wmy, Fm1, z); Fm2 = sel2(wmx, wmy, Fm2, z);
        umw = sel2(wmx, wmy, umw, z);
        cp = f2(wpx ? sqrtf(gp.x) : 0.0f, wpy ? sqrtf(gp.y) : 0.0f);
        cm = f2(wmx ? sqrtf(gm.x) : 0.0f, wmy ? sqrtf(gm.y) : 0.0f);
    }
    const float2 a1 = sub2(umw, cm), a2 = sub2(upw, cp);
    const float2 b1 = add2(umw, cm), b2 = add2(upw, cp);
    const float2 am = f2(fminf(fminf(a1.x, a2.x), 0.0f), fminf(fminf(a1.y, a2.y), 0.0f));
    const float2 ap = f2(fmaxf(fmaxf(b1.x, b2.x), 0.0f), fmaxf(fmaxf(b1.y, b2.y), 0.0f));
    const float2 d = sub2(ap, am);
    const float2 apam = mul2(ap, am);
    const float2 n0 = add2(sub2(mul2(ap, Fm0), mul2(am, Fp0)), mul2(apam, sub2(hp, hm)));
    const float2 n1 = add2(sub2(mul2(ap, Fm1), mul2(am, Fp1)), mul2(apam, sub2(Fp0, Fm0)));
    F0 = quot2<RCP>(n0, d);
    F1 = quot2<RCP>(n1, d);
    const float2 s = add2(um, up);
    F2 = f2(s.x > 0.0f ? Fm2.x : Fp2.x, s.y > 0.0f ? Fm2.y : Fp2.y);   // upwinded tangential flux
    const bool zx = fabsf(d.x) < k.flux_slope_eps, zy = fabsf(d.y) < k.flux_slope_eps;
    if (zx || zy) {   // symmetric Riemann fan: zero flux (:128-131)
        F0 = sel2(zx, zy, z, F0); F1 = sel2(zx, zy, z, F1); F2 = sel2(zx, zy, z, F2);
    }
}

struct Cell { float e, u, v; };     // reconstruction state (eta, u, v)

// Read-ahead ring (launch shape 5).  Each thread copies the inputs of its
// own column for row j + kReadAhead (cp.async, 4 bytes per value) into a
// private ring of kReadAhead + 1 shared-memory slots while it computes row
// j, so the global-load latency of a row is hidden behind kReadAhead rows of
// arithmetic without holding the values in registers; the thread reads only
// its own slots, so no barrier is involved.  The slot refilled at row j is
// the one read at row j - 1, whose values were consumed by then.  Measured
// on a B200 (us per RK2 step, 128 x 5 blocks): 4096^2 720 -> 686, 2048^2
// 207 -> 200, but 1024^2 66 -> 70 and 512^2 29 -> 32: once the grid fits in
// one wave of blocks the plain one-row register prefetch is faster.
constexpr int kReadAhead = 2;

__device__ __forceinline__ void cp_async4(void* smem, const float* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Per thread: Q of row j+2, Q^n of row j (stage 1), corners (cl, cl+1) of
// corner row j+3, for SLOTS rows.
template <int BW, int SLOTS>
struct ReadRing {
    float4 q[SLOTS][BW];
    float4 qn[SLOTS][BW];
    float2 h[SLOTS][BW];
};
template <int BW>
struct ReadRing<BW, 0> {};

// Shared-memory row buffers of one block (DEPTH: rows read ahead, 0 = none).
template <int BW, int DEPTH>
struct RowBufs {
    float4 r[BW];   // (eta, u, v, f*v along north)
    float4 s[BW];   // (u_x, v_x, K_x, -)
    float4 f[BW];   // F flux on the face west of the column
    ReadRing<BW, (DEPTH > 0 ? DEPTH + 1 : 0)> ring;
};

// Divisor by a domain constant c: a/c, or a * (1/c) with 1/c hoisted.
template <bool RCP>
struct ConstDiv {
    float c, inv;
    __device__ __forceinline__ explicit ConstDiv(float c_) : c(c_), inv(RCP ? rcp_approx(c_) : 0.0f) {}
    __device__ __forceinline__ float operator()(float a) const { return RCP ? a * inv : a / c; }
    __device__ __forceinline__ float2 operator()(float2 a) const {
        if (RCP) return mul2(a, f2(inv, inv));
        return f2(a.x / c, a.y / c);
    }
};

// True when the strip [r0, r1) of columns starting at c0 touches no ghost
// cell, wall flip, or periodic image: such blocks run the EDGE = false path.
template <int BW>
__device__ __forceinline__ bool interior_block(const Scheme& k, int c0, int r0, int r1) {
    return c0 >= 6 && c0 + BW - 3 <= k.nx - 1 && r0 >= 4 && r1 <= k.ny;
}

// One block strip: columns of block bx, rows of block by.
template <int BW, int FRIC, bool GEN_NORTH, bool WIND_FIELD, bool RCP, bool LAND, bool EDGE, int D>
__device__ __forceinline__ void stage_strip(const StageArgs& a, const float dt, const int bx, const int by,
                                            RowBufs<BW, D>& sb) {
    const Scheme& k = a.k;
    const int t = threadIdx.x;
    const int c0 = 2 + bx * (BW - 4);
    const int cl = c0 - 2 + t;
    const int r0 = 2 + by * a.rows_per_block;
    const int r1 = min(r0 + a.rows_per_block, k.ny + 2);

    const ConstDiv<RCP> by2g(k.two_g);
    const float inv_dx = RCP ? rcp_approx(k.dx) : 0.0f;
    const float inv_dy = RCP ? rcp_approx(k.dy) : 0.0f;
    auto bydxdy = [&](float2 v) -> float2 {
        if (RCP) return mul2(v, f2(inv_dx, inv_dy));
        return f2(v.x / k.dx, v.y / k.dy);
    };

    // ---- column addressing ------------------------------------------------
    int qc = cl;
    float hu_sgn = 1.0f;
    if (EDGE) {
        // wall ghosts mirror the interior with hu odd; columns past the array
        // (threads of the last block) clamp and are never written
        qc = min(cl, k.nx + 3);
        if (k.bcW == kWall && cl < 2) { qc = 3 - cl; hu_sgn = -1.0f; }
        if (k.bcE == kWall && cl > k.nx + 1 && cl <= k.nx + 3) { qc = 2 * k.nx + 3 - cl; hu_sgn = -1.0f; }
    }
    const int hca = EDGE ? min(cl, k.nx + 4) : cl;          // corner column west of the cell
    const int hcb = EDGE ? min(cl + 1, k.nx + 4) : cl + 1;  // east

    // Wall sign flips that the reference applies by global index.
    const bool flipKx = EDGE && ((k.bcW == kWall && cl < 2) || (k.bcE == kWall && cl > k.nx + 1));   // :633-641
    const bool flipAdjX = EDGE && ((k.bcW == kWall && cl < 2) || (k.bcE == kWall && cl > k.nx + 2)); // :172-174
    const bool flipFm = EDGE && (k.bcW == kWall && cl == 2);            // :286 (face west of cl)
    const bool flipFp = EDGE && (k.bcE == kWall && cl == k.nx + 2);     // :288
    auto flipLy = [&](int r) { return EDGE && ((k.bcS == kWall && r < 2) || (k.bcN == kWall && r > k.ny + 1)); };
    auto flipAdjY = [&](int r) { return EDGE && ((k.bcS == kWall && r < 2) || (k.bcN == kWall && r > k.ny + 2)); };

    const float eX = k.nY, eY = -k.nX;      // east = (north.y, -north.x), :681

    const float* __restrict__ eta_in = a.eta_in;
    const float* __restrict__ hu_in = a.hu_in;
    const float* __restrict__ hv_in = a.hv_in;
    const float* __restrict__ Hi = a.Hi;
    const float* __restrict__ frow = a.f_rows;
    // array extents of the checked-index build (unused otherwise)
    const long long xin = ext_in(a), xout = ext_out(a), xqn = ext_qn(a), xhi = ext_hi(a), xf = ext_f(a),
                    xw = ext_w(a);

    // wall ghost rows mirror the interior with hv odd
    auto mirror_row = [&](int r, float& hv_sgn) {
        hv_sgn = 1.0f;
        int rr = r;
        if (EDGE) {
            if (k.bcS == kWall && r < 2) { hv_sgn = -1.0f; rr = 3 - r; }
            else if (k.bcN == kWall && r > k.ny + 1) { hv_sgn = -1.0f; rr = 2 * k.ny + 3 - r; }
        }
        return rr;
    };
    auto load_q = [&](int r, float& e, float& hu, float& hv) {
        float hv_sgn;
        const int rr = mirror_row(r, hv_sgn);
        const size_t o = (size_t)rr * a.pin + qc;
        e = ldg1(eta_in, o, xin, a.status);
        hu = ldg1(hu_in, o, xin, a.status);
        hv = ldg1(hv_in, o, xin, a.status);
        if (EDGE) { hu *= hu_sgn; hv *= hv_sgn; }
    };
    auto load_h = [&](int r, float& ha, float& hb) {
        const size_t o = (size_t)r * a.phi;
        ha = ldg1(Hi, o + hca, xhi, a.status);
        hb = ldg1(Hi, o + hcb, xhi, a.status);
        if (LAND) { ha = corner(ha, k); hb = corner(hb, k); }
    };
    auto to_cell = [&](float e, float hu, float hv, float ha0, float hb0, float ha1, float hb1) {
        const float s = ((ha0 + ha1) + hb0) + hb1;
        const float Bm = LAND ? cell_bm(ha0, ha1, hb0, hb1, s, k) : s * 0.25f;
        Cell p;
        const float h = e + Bm;
        if (LAND && fabsf(Bm - k.land) <= kDryEps) {
            p.e = kDryFlag; p.u = 0.0f; p.v = 0.0f;
        } else if (h < k.desing_eps) {
            if (h <= k.cutoff) {
                p.e = -Bm + k.cutoff; p.u = 0.0f; p.v = 0.0f;
            } else {
                p.e = e;
                p.u = desingularize(h, hu, k.desing_eps);
                p.v = desingularize(h, hv, k.desing_eps);
            }
        } else {
            p.e = e;
            const float2 uv = quot2<RCP>(f2(hu, hv), f2(h, h));
            p.u = uv.x; p.v = uv.y;
        }
        return p;
    };
    // Coriolis part of L_y of a cell of row r, (east . (u', v)) f with u'
    // flipped in wall ghost rows (:738-758)
    auto fu_of = [&](const Cell& p, int r, float f) {
        const float uu = flipLy(r) ? -p.u : p.u;
        if (GEN_NORTH) return (eX * uu + eY * p.v) * f;
        return uu * f;
    };
    // y slope (u_y, v_y, L_y) at row r, scalar; used for the first rows only
    auto y_slope = [&](const Cell& lo, const Cell& c, const Cell& up, int r, float fulo, float fuc,
                       float fuup, float fc, float Hs, float Hn, float& du, float& dv) {
        du = minmod_slope(lo.u, c.u, up.u, k.theta);
        dv = minmod_slope(lo.v, c.v, up.v, k.theta);
        const float backward = k.theta_g * ((c.e - lo.e) + k.U * (fuc + fulo));
        const float central = k.half_g * ((up.e - lo.e) + k.U * ((fuup + 2.0f * fuc) + fulo));
        const float forward = k.theta_g * ((up.e - c.e) + k.U * (fuc + fuup));
        float L = minmod_raw(backward, central, forward);
        const float uu = flipAdjY(r) ? -c.u : c.u;   // adjustSlopes_y, :198-241
        const float dyfu = (k.dy * fc) * uu;
        const float q = by2g(L - dyfu);
        const float h_s = (c.e + Hs) - q;
        const float h_n = (c.e + Hn) + q;
        L = (h_s > 0.0f) ? L : dyfu + k.two_g * (c.e + Hs);
        L = (h_n > 0.0f) ? L : dyfu - k.two_g * (c.e + Hn);
        return L;
    };

    // ---- prime the window for rows r0-2 .. r0+1 ---------------------------
    float Ha0, Hb0, Ha1, Hb1, Ha2, Hb2;   // corner rows j, j+1, j+2 at cl (a), cl+1 (b)
    float ham2, hbm2, ham1, hbm1;
    load_h(r0 - 2, ham2, hbm2);
    load_h(r0 - 1, ham1, hbm1);
    load_h(r0, Ha0, Hb0);
    load_h(r0 + 1, Ha1, Hb1);
    load_h(r0 + 2, Ha2, Hb2);
    Cell Pm2, Pm1, P0, P1;
    {
        float e, hu, hv;
        load_q(r0 - 2, e, hu, hv); Pm2 = to_cell(e, hu, hv, ham2, hbm2, ham1, hbm1);
        load_q(r0 - 1, e, hu, hv); Pm1 = to_cell(e, hu, hv, ham1, hbm1, Ha0, Hb0);
        load_q(r0, e, hu, hv);     P0 = to_cell(e, hu, hv, Ha0, Hb0, Ha1, Hb1);
        load_q(r0 + 1, e, hu, hv); P1 = to_cell(e, hu, hv, Ha1, Hb1, Ha2, Hb2);
    }
    const float f_m2 = ldg1(frow, r0 - 2, xf, a.status), f_m1 = ldg1(frow, r0 - 1, xf, a.status);
    float f0 = ldg1(frow, r0, xf, a.status), f1 = ldg1(frow, r0 + 1, xf, a.status);
    const float fu_m2 = fu_of(Pm2, r0 - 2, f_m2);
    const float fu_m1 = fu_of(Pm1, r0 - 1, f_m1);
    float fu0 = fu_of(P0, r0, f0);
    float fu1 = fu_of(P1, r0 + 1, f1);
    const float Hy_m1 = 0.5f * (ham1 + hbm1);
    float Hy0 = 0.5f * (Ha0 + Hb0);
    float Hy1 = 0.5f * (Ha1 + Hb1);
    // slopes at r0-1 and r0, G flux on the face (r0-1 | r0)
    float uy_m1, vy_m1, uy0, vy0;
    const float Ly_m1 = y_slope(Pm2, Pm1, P0, r0 - 1, fu_m2, fu_m1, fu0, f_m1, Hy_m1, Hy0, uy_m1, vy_m1);
    float Ly0 = y_slope(Pm1, P0, P1, r0, fu_m1, fu0, fu1, f0, Hy0, Hy1, uy0, vy0);
    float Gs0, Gs1, Gs2;   // G on the face south of row j: (mass, hu, hv) fluxes
    {
        const bool dry = (P0.e == kDryFlag || Pm1.e == kDryFlag);
        const float um = (EDGE && k.bcS == kWall && r0 == 2) ? -Pm1.u : Pm1.u;
        const float upp = (EDGE && k.bcN == kWall && r0 == k.ny + 2) ? -P0.u : P0.u;
        float up_east = upp, um_east = um;
        if (GEN_NORTH) { up_east = upp * eX + P0.v * eY; um_east = um * eX + Pm1.v * eY; }
        const float hp = fmaxf(0.0f, (P0.e + Hy0) - by2g(Ly0 - (k.dy * f0) * up_east));
        const float hm = fmaxf(0.0f, (Pm1.e + Hy0) + by2g(Ly_m1 - (k.dy * f_m1) * um_east));
        float2 F0, F1, F2;
        central_upwind2<RCP>(f2(hm, hm), f2(Pm1.v + 0.5f * vy_m1, 0.0f), f2(Pm1.u + 0.5f * uy_m1, 0.0f),
                             f2(hp, hp), f2(P0.v - 0.5f * vy0, 0.0f), f2(P0.u - 0.5f * uy0, 0.0f), k, F0, F1, F2);
        Gs0 = dry ? 0.0f : F0.x;
        Gs1 = dry ? 0.0f : F2.x;
        Gs2 = dry ? 0.0f : F1.x;
    }

    const int tl = max(t - 1, 0), tr = min(t + 1, BW - 1);
    const bool writer = (t >= 2) && (t < BW - 2) && (!EDGE || cl <= k.nx + 1);
    const bool stage1 = (a.rk_step == 1);

    // Inputs of output row jj: Q of row jj+2, corner row jj+3, Q^n of row jj.
    // D > 0: copied into ring slot `slot`, one commit group per row (an
    // empty group past the strip keeps the group count per row fixed).
    auto stage_row = [&](int jj, int slot) {
        if constexpr (D > 0) {
            if (jj < r1) {
                float hv_sgn;
                // checked build: a copy whose source lies outside its array is skipped
                auto cpa = [&](float* dst, const float* src, size_t i, long long extent) {
                    if (idx_ok((long long)i, 1, extent, a.status)) cp_async4(dst, src + i);
                };
                const size_t o = (size_t)mirror_row(jj + 2, hv_sgn) * a.pin + qc;
                cpa(&sb.ring.q[slot][t].x, eta_in, o, xin);
                cpa(&sb.ring.q[slot][t].y, hu_in, o, xin);
                cpa(&sb.ring.q[slot][t].z, hv_in, o, xin);
                const size_t oh = (size_t)(jj + 3) * a.phi;
                cpa(&sb.ring.h[slot][t].x, Hi, oh + hca, xhi);
                cpa(&sb.ring.h[slot][t].y, Hi, oh + hcb, xhi);
                if (stage1 && writer) {
                    const size_t on = (size_t)jj * a.pqn + cl;
                    cpa(&sb.ring.qn[slot][t].x, a.qn_eta, on, xqn);
                    cpa(&sb.ring.qn[slot][t].y, a.qn_hu, on, xqn);
                    cpa(&sb.ring.qn[slot][t].z, a.qn_hv, on, xqn);
                }
            }
            cp_async_commit();
        }
    };

    // prefetch row r0+2 (Q), corner row r0+3, f(r0+2) and, for stage 1, Q^n(r0)
    float nq_e = 0.0f, nq_hu = 0.0f, nq_hv = 0.0f, nha = 0.0f, nhb = 0.0f, nf;
    float nqn_e = 0.0f, nqn_hu = 0.0f, nqn_hv = 0.0f;
    nf = ldg1(frow, r0 + 2, xf, a.status);
    int slot = 0;
    if constexpr (D > 0) {
#pragma unroll
        for (int d = 0; d < D; ++d) stage_row(r0 + d, d);
    } else {
        load_q(r0 + 2, nq_e, nq_hu, nq_hv);
        load_h(r0 + 3, nha, nhb);
        if (stage1 && writer) {
            const size_t o = (size_t)r0 * a.pqn + cl;
            nqn_e = ld1(a.qn_eta, o, xqn, a.status);
            nqn_hu = ld1(a.qn_hu, o, xqn, a.status);
            nqn_hv = ld1(a.qn_hv, o, xqn, a.status);
        }
    }
    const bool col_img = EDGE && (k.bcE == kPeriodic) && (cl < 4 || cl >= k.nx);
    const float2 theta2 = f2(k.theta, k.theta);
    const float2 thg2 = f2(k.theta_g, k.theta_g);
    const float2 hg2 = f2(k.half_g, k.half_g);
    const float2 VU2 = f2(-k.V, k.U);          // K_x subtracts V*(.), L_y adds U*(.)
    const float2 two_g2 = f2(k.two_g, k.two_g);

    // not unrolled: unrolled by 2, 3 or 4 the row loop spills under the
    // 96-register cap of 128 x 5 blocks and runs 2-16% slower at 4096^2
#pragma unroll 1
    for (int j = r0; j < r1; ++j) {
        // ---- row j+2 arrives; prefetch what a later row reads --------------
        float Ha3, Hb3, q_e, q_hu, q_hv, qn_e, qn_hu, qn_hv;
        const float f2r = nf;
        if constexpr (D > 0) {
            // refill the slot read at row j-1 with the inputs of row j+D,
            // then wait for this row's group (D groups may stay in flight)
            stage_row(j + D, (slot == 0) ? D : slot - 1);
            cp_async_wait<D>();
            const float4 q = sb.ring.q[slot][t];
            const float2 h = sb.ring.h[slot][t];
            q_e = q.x; q_hu = q.y; q_hv = q.z;
            if (EDGE) {
                float hv_sgn;
                mirror_row(j + 2, hv_sgn);
                q_hu *= hu_sgn; q_hv *= hv_sgn;
            }
            Ha3 = h.x; Hb3 = h.y;
            if (LAND) { Ha3 = corner(Ha3, k); Hb3 = corner(Hb3, k); }
            qn_e = qn_hu = qn_hv = 0.0f;
            if (stage1 && writer) {
                const float4 qn = sb.ring.qn[slot][t];
                qn_e = qn.x; qn_hu = qn.y; qn_hv = qn.z;
            }
            slot = (slot == D) ? 0 : slot + 1;
            nf = ldg1(frow, min(j + 3, k.ny + 3), xf, a.status);
        } else {
            Ha3 = nha; Hb3 = nhb;
            q_e = nq_e; q_hu = nq_hu; q_hv = nq_hv;
            qn_e = nqn_e; qn_hu = nqn_hu; qn_hv = nqn_hv;
            load_q(min(j + 3, r1 + 1), nq_e, nq_hu, nq_hv);
            load_h(min(j + 4, r1 + 2), nha, nhb);
            nf = ldg1(frow, min(j + 3, k.ny + 3), xf, a.status);
            if (stage1 && writer && j + 1 < r1) {
                const size_t o = (size_t)(j + 1) * a.pqn + cl;
                nqn_e = ld1(a.qn_eta, o, xqn, a.status);
                nqn_hu = ld1(a.qn_hu, o, xqn, a.status);
                nqn_hv = ld1(a.qn_hv, o, xqn, a.status);
            }
        }
        const Cell P2 = to_cell(q_e, q_hu, q_hv, Ha2, Hb2, Ha3, Hb3);
        const float fu2 = fu_of(P2, j + 2, f2r);
        const float Hy2 = 0.5f * (Ha2 + Hb2);

        // ---- publish row j --------------------------------------------------
        const float vK = flipKx ? -P0.v : P0.v;
        const float fv = GEN_NORTH ? (k.nX * P0.u + k.nY * vK) * f0 : vK * f0;
        sb.r[t] = make_float4(P0.e, P0.u, P0.v, fv);
        __syncthreads();
        const float4 RL = sb.r[tl], RR = sb.r[tr];

        // ---- slopes: lane x = x direction at row j, lane y = y at row j+1 ---
        //   x: l = (j, cl-1), c = (j, cl), r = (j, cl+1)
        //   y: l = (j, cl),   c = (j+1, cl), r = (j+2, cl)
        const float2 lu = f2(RL.y, P0.u), cu = f2(P0.u, P1.u), ru = f2(RR.y, P2.u);
        const float2 lv = f2(RL.z, P0.v), cv = f2(P0.v, P1.v), rv = f2(RR.z, P2.v);
        const float2 le = f2(RL.x, P0.e), ce = f2(P0.e, P1.e), re = f2(RR.x, P2.e);
        const float2 lf = f2(RL.w, fu0), cf = f2(fv, fu1), rf = f2(RR.w, fu2);
        const float2 du = minmod_slope2(lu, cu, ru, theta2);   // (u_x(j), u_y(j+1))
        const float2 dv = minmod_slope2(lv, cv, rv, theta2);   // (v_x(j), v_y(j+1))
        float2 K;                                              // (K_x(j), L_y(j+1))
        {
            const float2 backward = mul2(thg2, add2(sub2(ce, le), mul2(VU2, add2(cf, lf))));
            const float2 central = mul2(hg2, add2(sub2(re, le),
                                                  mul2(VU2, add2(add2(rf, mul2(f2(2.0f, 2.0f), cf)), lf))));
            const float2 forward = mul2(thg2, add2(sub2(re, ce), mul2(VU2, add2(cf, rf))));
            K = minmod2(backward, central, forward);
        }
        const float Hw = 0.5f * (Ha0 + Ha1);   // x-face depth west of the cell (row j)
        const float He = 0.5f * (Hb0 + Hb1);   // east
        const float dxf = k.dx * f0;
        {   // adjustSlopes_x (:148-191) and adjustSlopes_y (:198-241) in one:
            // nw = (-dx f v, dy f u); K_x + dx f v = K_x - nw.x, L_y - dy f u = L_y - nw.y;
            // fallbacks -dx f v + 2g(..) (x) and dy f u + 2g(..) (y) are nw + 2g(..)
            const float vv = flipAdjX ? -P0.v : P0.v;
            const float uu = flipAdjY(j + 1) ? -P1.u : P1.u;
            const float2 nw = f2((-dxf) * vv, (k.dy * f1) * uu);
            const float2 q = by2g(sub2(K, nw));
            const float2 Hlo = f2(Hw, Hy1), Hhi = f2(He, Hy2);
            const float2 hlo = sub2(add2(ce, Hlo), q);
            const float2 hhi = add2(add2(ce, Hhi), q);
            if (!(hlo.x > 0.0f && hlo.y > 0.0f && hhi.x > 0.0f && hhi.y > 0.0f)) {
                const float2 Klo = add2(nw, mul2(two_g2, add2(ce, Hlo)));
                const float2 Khi = sub2(nw, mul2(two_g2, add2(ce, Hhi)));
                K = sel2(hlo.x > 0.0f, hlo.y > 0.0f, K, Klo);
                K = sel2(hhi.x > 0.0f, hhi.y > 0.0f, K, Khi);
            }
        }
        sb.s[t] = make_float4(du.x, dv.x, K.x, 0.0f);
        __syncthreads();
        const float4 SL = sb.s[tl];

        // ---- fluxes: lane x = F on face (cl-1 | cl), lane y = G on (j | j+1)
        float2 F0, F1, F2;
        {
            // minus / plus sides; lane x: m = (j, cl-1), p = (j, cl)
            //                      lane y: m = (j, cl),   p = (j+1, cl)
            const float2 em = f2(RL.x, P0.e), ep = f2(P0.e, P1.e);
            // normal velocity and its slope per lane: x -> u, y -> v
            const float2 unm = f2(RL.y, P0.v), unp = f2(P0.u, P1.v);
            const float2 utm = f2(RL.z, P0.u), utp = f2(P0.v, P1.u);
            const float2 dnm = f2(SL.x, vy0), dnp = f2(du.x, dv.y);
            const float2 dtm = f2(SL.y, uy0), dtp = f2(dv.x, du.y);
            const float2 Km = f2(SL.z, Ly0), Kp = K;
            const float2 half = f2(0.5f, 0.5f);
            const float2 Rpn = sub2(unp, mul2(half, dnp)), Rpt = sub2(utp, mul2(half, dtp));
            const float2 Rmn = add2(unm, mul2(half, dnm)), Rmt = add2(utm, mul2(half, dtm));
            // velocity used in the Coriolis part of the face depth:
            //   x: v along north (flipped at walls), coefficient +dx f
            //   y: u along east (flipped at walls), coefficient -dy f
            float vmx = flipFm ? -RL.z : RL.z;
            float vpx = flipFp ? -P0.v : P0.v;
            float umy = (EDGE && k.bcS == kWall && j + 1 == 2) ? -P0.u : P0.u;
            float upy = (EDGE && k.bcN == kWall && j + 1 == k.ny + 2) ? -P1.u : P1.u;
            if (GEN_NORTH) {
                vmx = RL.y * k.nX + vmx * k.nY; vpx = P0.u * k.nX + vpx * k.nY;
                umy = umy * eX + P0.v * eY; upy = upy * eX + P1.v * eY;
            }
            const float2 cm = f2(dxf, -(k.dy * f0)), cp = f2(dxf, -(k.dy * f1));
            const float2 Hf = f2(Hw, Hy1);
            const float2 hp = sub2(add2(ep, Hf), by2g(add2(Kp, mul2(cp, f2(vpx, upy)))));
            const float2 hm = add2(add2(em, Hf), by2g(add2(Km, mul2(cm, f2(vmx, umy)))));
            const float2 hp0 = f2(fmaxf(0.0f, hp.x), fmaxf(0.0f, hp.y));
            const float2 hm0 = f2(fmaxf(0.0f, hm.x), fmaxf(0.0f, hm.y));
            central_upwind2<RCP>(hm0, Rmn, Rmt, hp0, Rpn, Rpt, k, F0, F1, F2);
            const bool dryx = (P0.e == kDryFlag || RL.x == kDryFlag);
            const bool dryy = (P1.e == kDryFlag || P0.e == kDryFlag);
            if (dryx || dryy) {   // a land cell on either side: zero flux (:271-273)
                const float2 z = f2(0.0f, 0.0f);
                F0 = sel2(dryx, dryy, z, F0);
                F1 = sel2(dryx, dryy, z, F1);
                F2 = sel2(dryx, dryy, z, F2);
            }
        }
        // F on the west face of cl: (mass, hu, hv) = (F0.x, F1.x, F2.x)
        // G on the north face of row j: (mass, hu, hv) = (F0.y, F2.y, F1.y)
        sb.f[t] = make_float4(F0.x, F1.x, F2.x, 0.0f);
        __syncthreads();
        const float4 FE = sb.f[tr];

        // ---- update the cell (j, cl), :807-1004 -----------------------------
        if (writer) {
            const float Hm = 0.25f * (((Ha0 + Ha1) + Hb0) + Hb1);
            // flux differences: (F_e - F_w)/dx + (G_n - G_s)/dy per component
            const float2 d0 = bydxdy(f2(FE.x - F0.x, F0.y - Gs0));
            const float2 d1 = bydxdy(f2(FE.y - F1.x, F2.y - Gs1));
            const float2 d2 = bydxdy(f2(FE.z - F2.x, F1.y - Gs2));
            const float fd0 = d0.x + d0.y, fd1 = d1.x + d1.y, fd2 = d2.x + d2.y;
            // face values of eta for the bathymetry source (:706-707, :803-804):
            //   (K_x + dx f v)/2g and (L_y - dy f u)/2g of the own cell
            const float2 tt = by2g(add2(f2(K.x, Ly0), mul2(f2(dxf, -(k.dy * f0)), f2(P0.v, P0.u))));
            const float2 eta_lo = sub2(f2(P0.e, P0.e), tt);   // (west, south)
            const float2 eta_hi = add2(f2(P0.e, P0.e), tt);   // (east, north)

            const float h = P0.e + Hm;
            float2 huv = f2(0.0f, 0.0f);
            if (h > k.cutoff) huv = mul2(f2(P0.u, P0.v), f2(h, h));

            float2 st = f2(0.0f, 0.0f);
            if (h >= k.cutoff && P0.e != kDryFlag) {
                float X, Y;
                if (WIND_FIELD) {
                    // one load when the current and next fields are one array
                    const size_t o = (size_t)(j - 2) * a.pw + (cl - 2);
                    const float xn = ldg1(a.wx_next, o, xw, a.status), yn = ldg1(a.wy_next, o, xw, a.status);
                    const float xc = (a.wx_cur == a.wx_next) ? xn : ldg1(a.wx_cur, o, xw, a.status);
                    const float yc = (a.wy_cur == a.wy_next) ? yn : ldg1(a.wy_cur, o, xw, a.status);
                    X = a.wind_t * xn + (1.0f - a.wind_t) * xc;
                    Y = a.wind_t * yn + (1.0f - a.wind_t) * yc;
                } else {
                    X = a.wind_t * a.wxn + (1.0f - a.wind_t) * a.wxc;
                    Y = a.wind_t * a.wyn + (1.0f - a.wind_t) * a.wyc;
                }
                const float2 Hxy = f2(He - Hw, Hy1 - Hy0);
                const float2 eta_mid = mul2(f2(0.5f, 0.5f), add2(eta_lo, eta_hi));   // (we, sn)
                const float2 bb = mul2(mul2(f2(k.g, k.g), add2(eta_mid, f2(Hm, Hm))), Hxy);
                float2 cor;
                if (GEN_NORTH) {
                    const float hu_east = huv.x * eX + huv.y * eY;
                    const float hv_north = huv.x * k.nX + huv.y * k.nY;
                    const float hu_east_cor = f0 * hv_north;
                    const float hv_north_cor = -f0 * hu_east;
                    const float upx = -k.nX, upy = k.nY;
                    const float rx = upy, ry = -upx;
                    cor = f2(rx * hu_east_cor + ry * hv_north_cor, upx * hu_east_cor + upy * hv_north_cor);
                } else {
                    cor = mul2(f2(f0, -f0), f2(huv.y, huv.x));
                }
                st = add2(add2(f2(X, Y), cor), bydxdy(bb));
            }
            const float L1 = -fd0;
            const float2 L23 = sub2(st, f2(fd1, fd2));   // -fd + st

            float C = 0.0f;
            if (FRIC == kFricLinear) {
                C = quot<RCP>(k.two_r * dt, P0.e + Hm);
            } else if (FRIC == kFricQuad) {
                if (h < k.desing_eps) {
                    const float u = desingularize(h, huv.x, k.desing_eps);
                    const float v = desingularize(h, huv.y, k.desing_eps);
                    C = dt * k.r * desingularize(h, sqrtf(u * u + v * v), k.desing_eps);
                } else {
                    const float2 uv = quot2<RCP>(huv, f2(h, h));
                    const float2 uv2 = mul2(uv, uv);
                    C = quot<RCP>(dt * k.r * sqrtf(uv2.x + uv2.y), h);
                }
            }
            const float2 dt2 = f2(dt, dt);
            float ne;
            float2 nuv;
            if (!stage1) {
                ne = P0.e + dt * L1;
                const float den = 1.0f + C;
                nuv = quot2<RCP>(add2(huv, mul2(dt2, L23)), f2(den, den));
            } else {
                ne = 0.5f * (qn_e + (P0.e + dt * L1));
                const float den = 1.0f + 0.5f * C;
                const float2 b = mul2(f2(0.5f, 0.5f), add2(f2(qn_hu, qn_hv), add2(huv, mul2(dt2, L23))));
                nuv = quot2<RCP>(b, f2(den, den));
            }
            float nhu = nuv.x, nhv = nuv.y;
            if (ne + Hm <= k.cutoff) {
                ne = -Hm + k.cutoff; nhu = 0.0f; nhv = 0.0f;
            }
            ne = fmaxf(-Hm + k.cutoff, ne);
            if (!isfinite(ne + nhu + nhv) && a.status) atomicOr(a.status, 1u);

            const size_t o = (size_t)j * a.pout + cl;
            st1(a.eta_out, o, ne, xout, a.status);
            st1(a.hu_out, o, nhu, xout, a.status);
            st1(a.hv_out, o, nhv, xout, a.status);
            if (EDGE) {
                // periodic ghost images (the reference's BC kernels after the stage)
                const bool row_img = (k.bcN == kPeriodic) && (j < 4 || j >= k.ny);
                if (row_img || col_img) {
                    int rows_img[2] = {-1, -1}, cols_img[2] = {-1, -1};
                    if (k.bcN == kPeriodic) {
                        if (j < 4) rows_img[0] = j + k.ny;
                        if (j >= k.ny) rows_img[1] = j - k.ny;
                    }
                    if (k.bcE == kPeriodic) {
                        if (cl < 4) cols_img[0] = cl + k.nx;
                        if (cl >= k.nx) cols_img[1] = cl - k.nx;
                    }
                    const int rr[3] = {j, rows_img[0], rows_img[1]};
                    const int cc[3] = {cl, cols_img[0], cols_img[1]};
                    for (int ri = 0; ri < 3; ++ri) {
                        for (int ci = 0; ci < 3; ++ci) {
                            if ((ri == 0 && ci == 0) || rr[ri] < 0 || cc[ci] < 0) continue;
                            const size_t oo = (size_t)rr[ri] * a.pout + cc[ci];
                            st1(a.eta_out, oo, ne, xout, a.status);
                            st1(a.hu_out, oo, nhu, xout, a.status);
                            st1(a.hv_out, oo, nhv, xout, a.status);
                        }
                    }
                }
            }
        }

        // ---- slide the window -----------------------------------------------
        Pm1 = P0; P0 = P1; P1 = P2;
        fu0 = fu1; fu1 = fu2;
        uy0 = du.y; vy0 = dv.y; Ly0 = K.y;
        Gs0 = F0.y; Gs1 = F2.y; Gs2 = F1.y;
        Ha0 = Ha1; Hb0 = Hb1; Ha1 = Ha2; Hb1 = Hb2; Ha2 = Ha3; Hb2 = Hb3;
        Hy0 = Hy1; Hy1 = Hy2;
        f0 = f1; f1 = f2r;
    }
}

template <int BW, int FRIC, bool GEN_NORTH, bool WIND_FIELD, bool RCP, bool LAND, int D>
__device__ __forceinline__ void stage_block(const StageArgs& a, const float dt, const int bx, const int by,
                                            RowBufs<BW, D>& sb) {
    const int c0 = 2 + bx * (BW - 4);
    const int r0 = 2 + by * a.rows_per_block;
    const int r1 = min(r0 + a.rows_per_block, a.k.ny + 2);
    if (interior_block<BW>(a.k, c0, r0, r1))
        stage_strip<BW, FRIC, GEN_NORTH, WIND_FIELD, RCP, LAND, false, D>(a, dt, bx, by, sb);
    else
        stage_strip<BW, FRIC, GEN_NORTH, WIND_FIELD, RCP, LAND, true, D>(a, dt, bx, by, sb);
}

template <int BW, int MINB, int FRIC, bool GEN_NORTH, bool WIND_FIELD, bool RCP, bool LAND, int D>
__global__ void __launch_bounds__(BW, MINB) cdklm_stage_kernel(const StageArgs a) {
    __shared__ RowBufs<BW, D> sb;
    stage_block<BW, FRIC, GEN_NORTH, WIND_FIELD, RCP, LAND, D>(a, a.dt, blockIdx.x, blockIdx.y, sb);
}

// Batched stage: a packed list of (member, column block, row block) tiles
// over every member of an ensemble or set of domains, walked by a
// persistent grid.  args holds two entries per member (stage 0: h0 -> h1,
// stage 1: h1 -> h0); dts holds the member's time step, read at launch so a
// captured graph picks up new values.
template <int BW, int MINB, int FRIC, bool GEN_NORTH, bool WIND_FIELD, bool RCP, bool LAND, int D>
__global__ void __launch_bounds__(BW, MINB)
    cdklm_batch_kernel(const StageArgs* __restrict__ args, const float* __restrict__ dts,
                       const int4* __restrict__ tiles, const int ntiles, const int rk_step) {
    __shared__ RowBufs<BW, D> sb;
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const int4 tile = tiles[ti];
        const StageArgs& a = args[2 * tile.x + rk_step];
        stage_block<BW, FRIC, GEN_NORTH, WIND_FIELD, RCP, LAND, D>(a, __ldg(dts + tile.x), tile.y, tile.z, sb);
        __syncthreads();
    }
}

}  // namespace go
