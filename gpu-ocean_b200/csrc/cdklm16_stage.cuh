// One Runge-Kutta sub-step of CDKLM16 as a column-marching stencil.
//
// Restates cdklm_swe_2D (gpu_ocean/SWESimulators/gpu_kernels/CDKLM16_kernel.cu:429-1006)
// followed by the periodic ghost refresh the host issues after it
// (Common.py:1219-1239 -> boundary_kernels.cu:35-110).
//
// Layout of the work: a block of BW threads covers BW consecutive
// ghost-inclusive columns cl = c0-2 .. c0+BW-3 and writes the BW-4 interior
// columns c0 .. c0+BW-5.  Each thread owns one column and marches down the
// block's strip of rows [r0, r1).  Everything along y (the slopes u_y, v_y,
// L_y and the G fluxes) lives in registers as a sliding window of rows; the
// x direction (slopes u_x, v_x, K_x and the F fluxes) is exchanged between
// neighbouring threads through three shared-memory row buffers.  Each face
// flux is evaluated once (the reference evaluates every face twice, once
// per adjacent cell).  Ghost cells: wall sides are mirrored on load (as
// handleWallBC, CDKLM16_kernel.cu:373-424, does in shared memory);
// periodic sides read the ghost cells of the input, which the previous
// stage refreshed.
#pragma once

#include "cdklm16_device.cuh"

namespace go {

struct StageArgs {
    Scheme k;
    float dt;
    int rk_step;                 // 0: Q* = Q + dt L(Q);  1: Heun average
    const float* eta_in; const float* hu_in; const float* hv_in;
    int pin;                     // pitch of the inputs, floats
    float* eta_out; float* hu_out; float* hv_out;
    int pout;                    // pitch of the outputs, floats
    const float* Hi; int phi;    // corners (ny+5) x (nx+5)
    const float* f_rows;         // Coriolis per ghost-inclusive row
    float wind_t, wxc, wxn, wyc, wyn;
    const float* wx_cur; const float* wx_next;
    const float* wy_cur; const float* wy_next; int pw;  // interior-indexed
    int rows_per_block;
    unsigned int* status;
};

// Friction law selector.
enum { kFricNone = 0, kFricQuad = 1, kFricLinear = 2 };

template <int BW, int FRIC, bool GEN_NORTH, bool WIND_FIELD>
__global__ void __launch_bounds__(BW) cdklm_stage_kernel(const StageArgs a) {
    const Scheme& k = a.k;
    const int t = threadIdx.x;
    const int c0 = 2 + blockIdx.x * (BW - 4);
    const int cl = c0 - 2 + t;
    const int r0 = 2 + blockIdx.y * a.rows_per_block;
    const int r1 = min(r0 + a.rows_per_block, k.ny + 2);

    __shared__ float sE[BW], sU[BW], sV[BW], sFv[BW];
    __shared__ float sUx[BW], sVx[BW], sKx[BW];
    __shared__ float sF0[BW], sF1[BW], sF2[BW];

    // ---- column addressing ------------------------------------------------
    // Q columns: wall ghosts mirror the interior with hu odd; columns past
    // the array (threads of the last block) clamp and are never written.
    int qc = min(cl, k.nx + 3);
    float hu_sgn = 1.0f;
    if (k.bcW == kWall && cl < 2) { qc = 3 - cl; hu_sgn = -1.0f; }
    if (k.bcE == kWall && cl > k.nx + 1 && cl <= k.nx + 3) { qc = 2 * k.nx + 3 - cl; hu_sgn = -1.0f; }
    const int hca = min(cl, k.nx + 4);      // corner column of the cell's west side
    const int hcb = min(cl + 1, k.nx + 4);  // east side

    // Wall sign flips that the reference applies by global index.
    const bool flipKx = (k.bcW == kWall && cl < 2) || (k.bcE == kWall && cl > k.nx + 1);    // :633-641
    const bool flipAdjX = (k.bcW == kWall && cl < 2) || (k.bcE == kWall && cl > k.nx + 2);  // :172-174
    const bool flipFm = (k.bcW == kWall && cl == 2);            // :286 (face west of cl)
    const bool flipFp = (k.bcE == kWall && cl == k.nx + 2);     // :288

    const float eX = k.nY, eY = -k.nX;      // east = (north.y, -north.x), :681

    const float* __restrict__ eta_in = a.eta_in;
    const float* __restrict__ hu_in = a.hu_in;
    const float* __restrict__ hv_in = a.hv_in;
    const float* __restrict__ Hi = a.Hi;
    const float* __restrict__ frow = a.f_rows;

    auto qrow = [&](int r, float& hv_sgn) -> int {
        hv_sgn = 1.0f;
        if (k.bcS == kWall && r < 2) { hv_sgn = -1.0f; return 3 - r; }
        if (k.bcN == kWall && r > k.ny + 1) { hv_sgn = -1.0f; return 2 * k.ny + 3 - r; }
        return r;
    };
    auto load_q = [&](int r, float& e, float& hu, float& hv) {
        float s;
        const int rr = qrow(r, s);
        const size_t o = (size_t)rr * a.pin + qc;
        e = __ldg(eta_in + o);
        hu = hu_sgn * __ldg(hu_in + o);
        hv = s * __ldg(hv_in + o);
    };
    auto load_h = [&](int r, float& ha, float& hb) {
        const size_t o = (size_t)r * a.phi;
        ha = corner(__ldg(Hi + o + hca), k);
        hb = corner(__ldg(Hi + o + hcb), k);
    };
    auto bm_of = [&](float ha0, float hb0, float ha1, float hb1) {
        const float s = ((ha0 + ha1) + hb0) + hb1;
        return cell_bm(ha0, ha1, hb0, hb1, s, k);
    };
    // v used in the Coriolis part of K_x, and u in that of L_y
    auto fv_of = [&](const Prim& p, float f) {
        const float vv = flipKx ? -p.v : p.v;
        if (GEN_NORTH) return (k.nX * p.u + k.nY * vv) * f;
        return vv * f;
    };
    auto fu_of = [&](const Prim& p, int r, float f) {
        const bool fl = (k.bcS == kWall && r < 2) || (k.bcN == kWall && r > k.ny + 1);  // :738-746
        const float uu = fl ? -p.u : p.u;
        if (GEN_NORTH) return (eX * uu + eY * p.v) * f;
        return uu * f;
    };
    // y slope at row r from rows r-1 (lo), r (c), r+1 (up); Hs/Hn are the
    // y-face depths south and north of the cell.  :715-777
    auto y_slope = [&](const Prim& lo, const Prim& c, const Prim& up, int r,
                       float flo, float fc, float fup, float Hs, float Hn) {
        Slp s;
        s.du = minmod_slope(lo.u, c.u, up.u, k.theta);
        s.dv = minmod_slope(lo.v, c.v, up.v, k.theta);
        const float fulo = fu_of(lo, r - 1, flo);
        const float fuc = fu_of(c, r, fc);
        const float fuup = fu_of(up, r + 1, fup);
        const float backward = k.theta_g * ((c.e - lo.e) + k.U * (fuc + fulo));
        const float central = k.half_g * ((up.e - lo.e) + k.U * ((fuup + 2.0f * fuc) + fulo));
        const float forward = k.theta_g * ((up.e - c.e) + k.U * (fuc + fuup));
        float L = minmod_raw(backward, central, forward);
        // adjustSlopes_y, :198-241
        const bool fl = (k.bcS == kWall && r < 2) || (k.bcN == kWall && r > k.ny + 2);
        const float uu = fl ? -c.u : c.u;
        const float dyfu = (k.dy * fc) * uu;
        const float h_s = (c.e + Hs) - (L - dyfu) / k.two_g;
        const float h_n = (c.e + Hn) + (L - dyfu) / k.two_g;
        L = (h_s > 0.0f) ? L : dyfu + k.two_g * (c.e + Hs);
        L = (h_n > 0.0f) ? L : dyfu - k.two_g * (c.e + Hn);
        s.K = L;
        return s;
    };
    // G flux on the face between rows r (m) and r+1 (p).  :309-370
    auto g_face = [&](const Prim& m, const Slp& sm, const Prim& p, const Slp& sp, int r,
                      float fm, float fp, float Hface) {
        if (p.e == kDryFlag || m.e == kDryFlag) return F3{0.0f, 0.0f, 0.0f};
        const float Rpu = p.u - 0.5f * sp.du, Rpv = p.v - 0.5f * sp.dv;
        const float Rmu = m.u + 0.5f * sm.du, Rmv = m.v + 0.5f * sm.dv;
        const float um = (k.bcS == kWall && r + 1 == 2) ? -m.u : m.u;
        const float upp = (k.bcN == kWall && r + 1 == k.ny + 2) ? -p.u : p.u;
        float up_east, um_east;
        if (GEN_NORTH) { up_east = upp * eX + p.v * eY; um_east = um * eX + m.v * eY; }
        else { up_east = upp; um_east = um; }
        const float hp = fmaxf(0.0f, (p.e + Hface) - (sp.K - (k.dy * fp) * up_east) / k.two_g);
        const float hm = fmaxf(0.0f, (m.e + Hface) + (sm.K - (k.dy * fm) * um_east) / k.two_g);
        const F3 F = central_upwind(hm, Rmv, Rmu, hp, Rpv, Rpu, k);
        return F3{F.a, F.c, F.b};
    };

    // ---- prime the window for rows r0-2 .. r0+1 ---------------------------
    float Ha[4], Hb[4];  // corner rows j..j+3 at columns cl (a) and cl+1 (b)
    float ha_m2, hb_m2, ha_m1, hb_m1;
    load_h(r0 - 2, ha_m2, hb_m2);
    load_h(r0 - 1, ha_m1, hb_m1);
    load_h(r0, Ha[0], Hb[0]);
    load_h(r0 + 1, Ha[1], Hb[1]);
    load_h(r0 + 2, Ha[2], Hb[2]);

    Prim Pm2, Pm1, P0, P1;
    {
        float e, hu, hv;
        load_q(r0 - 2, e, hu, hv); Pm2 = to_prim(e, hu, hv, bm_of(ha_m2, hb_m2, ha_m1, hb_m1), k);
        load_q(r0 - 1, e, hu, hv); Pm1 = to_prim(e, hu, hv, bm_of(ha_m1, hb_m1, Ha[0], Hb[0]), k);
        load_q(r0, e, hu, hv);     P0 = to_prim(e, hu, hv, bm_of(Ha[0], Hb[0], Ha[1], Hb[1]), k);
        load_q(r0 + 1, e, hu, hv); P1 = to_prim(e, hu, hv, bm_of(Ha[1], Hb[1], Ha[2], Hb[2]), k);
    }
    float f_m2 = __ldg(frow + r0 - 2), f_m1 = __ldg(frow + r0 - 1);
    float f0 = __ldg(frow + r0), f1 = __ldg(frow + r0 + 1);

    const float Hy_m1 = 0.5f * (ha_m1 + hb_m1);
    const float Hy_0 = 0.5f * (Ha[0] + Hb[0]);
    const float Hy_1 = 0.5f * (Ha[1] + Hb[1]);
    const Slp Sm1 = y_slope(Pm2, Pm1, P0, r0 - 1, f_m2, f_m1, f0, Hy_m1, Hy_0);
    Slp S0 = y_slope(Pm1, P0, P1, r0, f_m1, f0, f1, Hy_0, Hy_1);
    F3 Gs = g_face(Pm1, Sm1, P0, S0, r0 - 1, f_m1, f0, Hy_0);

    // prefetch row r0+2 (Q) and corner row r0+3
    float nq_e, nq_hu, nq_hv, nha, nhb, nf;
    load_q(r0 + 2, nq_e, nq_hu, nq_hv);
    load_h(r0 + 3, nha, nhb);
    nf = __ldg(frow + r0 + 2);

    const int tl = max(t - 1, 0), tr = min(t + 1, BW - 1);
    const bool writer = (t >= 2) && (t < BW - 2) && (cl <= k.nx + 1);

    for (int j = r0; j < r1; ++j) {
        // ---- row j+2 arrives; prefetch j+3 --------------------------------
        Ha[3] = nha; Hb[3] = nhb;
        const float f2 = nf;
        float q_e = nq_e, q_hu = nq_hu, q_hv = nq_hv;
        {
            const int rn = min(j + 3, r1 + 1);
            load_q(rn, nq_e, nq_hu, nq_hv);
            const int hn = min(j + 4, r1 + 2);
            load_h(hn, nha, nhb);
            nf = __ldg(frow + min(j + 3, k.ny + 3));
        }
        float qn_e = 0.0f, qn_hu = 0.0f, qn_hv = 0.0f;
        if (a.rk_step == 1 && writer) {
            const size_t o = (size_t)j * a.pout + cl;
            qn_e = a.eta_out[o]; qn_hu = a.hu_out[o]; qn_hv = a.hv_out[o];
        }
        const Prim P2 = to_prim(q_e, q_hu, q_hv, bm_of(Ha[2], Hb[2], Ha[3], Hb[3]), k);

        // ---- y direction: slope at j+1, G on face (j | j+1) ----------------
        const float Hy1 = 0.5f * (Ha[1] + Hb[1]);
        const float Hy2 = 0.5f * (Ha[2] + Hb[2]);
        const Slp S1 = y_slope(P0, P1, P2, j + 1, f0, f1, f2, Hy1, Hy2);
        const F3 Gn = g_face(P0, S0, P1, S1, j, f0, f1, Hy1);

        // ---- x direction on row j ------------------------------------------
        const float fv = fv_of(P0, f0);
        sE[t] = P0.e; sU[t] = P0.u; sV[t] = P0.v; sFv[t] = fv;
        __syncthreads();
        const float eL = sE[tl], uL = sU[tl], vL = sV[tl], fvL = sFv[tl];
        const float eR = sE[tr], uR = sU[tr], fvR = sFv[tr];
        const float vR = sV[tr];
        const float ux = minmod_slope(uL, P0.u, uR, k.theta);
        const float vx = minmod_slope(vL, P0.v, vR, k.theta);
        float Kx;
        {
            const float backward = k.theta_g * ((P0.e - eL) - k.V * (fv + fvL));
            const float central = k.half_g * ((eR - eL) - k.V * ((fvR + 2.0f * fv) + fvL));
            const float forward = k.theta_g * ((eR - P0.e) - k.V * (fv + fvR));
            Kx = minmod_raw(backward, central, forward);
        }
        const float Hw = 0.5f * (Ha[0] + Ha[1]);  // x-face depth west of the cell
        const float He = 0.5f * (Hb[0] + Hb[1]);  // east
        {   // adjustSlopes_x, :148-191
            const float vv = flipAdjX ? -P0.v : P0.v;
            const float dxfv = (k.dx * f0) * vv;
            const float h_w = (P0.e + Hw) - (Kx + dxfv) / k.two_g;
            const float h_e = (P0.e + He) + (Kx + dxfv) / k.two_g;
            Kx = (h_w > 0.0f) ? Kx : -dxfv + k.two_g * (P0.e + Hw);
            Kx = (h_e > 0.0f) ? Kx : -dxfv - k.two_g * (P0.e + He);
        }
        sUx[t] = ux; sVx[t] = vx; sKx[t] = Kx;
        __syncthreads();
        F3 Fw;   // F on the face (cl-1 | cl), :246-304
        {
            const float uxm = sUx[tl], vxm = sVx[tl], Kxm = sKx[tl];
            if (P0.e == kDryFlag || eL == kDryFlag) {
                Fw = F3{0.0f, 0.0f, 0.0f};
            } else {
                const float Rpu = P0.u - 0.5f * ux, Rpv = P0.v - 0.5f * vx;
                const float Rmu = uL + 0.5f * uxm, Rmv = vL + 0.5f * vxm;
                const float vm = flipFm ? -vL : vL;
                const float vp = flipFp ? -P0.v : P0.v;
                float vp_n, vm_n;
                if (GEN_NORTH) { vp_n = P0.u * k.nX + vp * k.nY; vm_n = uL * k.nX + vm * k.nY; }
                else { vp_n = vp; vm_n = vm; }
                const float dxf = k.dx * f0;
                const float hp = fmaxf(0.0f, (P0.e + Hw) - (Kx + dxf * vp_n) / k.two_g);
                const float hm = fmaxf(0.0f, (eL + Hw) + (Kxm + dxf * vm_n) / k.two_g);
                Fw = central_upwind(hm, Rmu, Rmv, hp, Rpu, Rpv, k);
            }
        }
        sF0[t] = Fw.a; sF1[t] = Fw.b; sF2[t] = Fw.c;
        __syncthreads();
        const float Fe0 = sF0[tr], Fe1 = sF1[tr], Fe2 = sF2[tr];

        // ---- update the cell (j, cl), :807-1004 -----------------------------
        if (writer) {
            const float Hm = 0.25f * (((Ha[0] + Ha[1]) + Hb[0]) + Hb[1]);
            const float fd0 = (Fe0 - Fw.a) / k.dx + (Gn.a - Gs.a) / k.dy;
            const float fd1 = (Fe1 - Fw.b) / k.dx + (Gn.b - Gs.b) / k.dy;
            const float fd2 = (Fe2 - Fw.c) / k.dx + (Gn.c - Gs.c) / k.dy;
            const float tw = (Kx + (k.dx * f0) * P0.v) / k.two_g;
            const float eta_west = P0.e - tw;
            const float eta_east = P0.e + tw;
            const float ts = (S0.K - (k.dy * f0) * P0.u) / k.two_g;
            const float eta_south = P0.e - ts;
            const float eta_north = P0.e + ts;

            const float h = P0.e + Hm;
            float hu = 0.0f, hv = 0.0f;
            if (h > k.cutoff) { hu = P0.u * h; hv = P0.v * h; }

            float st1 = 0.0f, st2 = 0.0f;
            if (h >= k.cutoff && P0.e != kDryFlag) {
                float X, Y;
                if (WIND_FIELD) {
                    const size_t o = (size_t)(j - 2) * a.pw + (cl - 2);
                    X = a.wind_t * __ldg(a.wx_next + o) + (1.0f - a.wind_t) * __ldg(a.wx_cur + o);
                    Y = a.wind_t * __ldg(a.wy_next + o) + (1.0f - a.wind_t) * __ldg(a.wy_cur + o);
                } else {
                    X = a.wind_t * a.wxn + (1.0f - a.wind_t) * a.wxc;
                    Y = a.wind_t * a.wyn + (1.0f - a.wind_t) * a.wyc;
                }
                const float H_x = He - Hw;
                const float H_y = Hy1 - 0.5f * (Ha[0] + Hb[0]);
                const float eta_sn = 0.5f * (eta_north + eta_south);
                const float eta_we = 0.5f * (eta_west + eta_east);
                const float b1 = (k.g * (eta_we + Hm)) * H_x;
                const float b2 = (k.g * (eta_sn + Hm)) * H_y;
                float hu_cor, hv_cor;
                if (GEN_NORTH) {
                    const float hu_east = hu * eX + hv * eY;
                    const float hv_north = hu * k.nX + hv * k.nY;
                    const float hu_east_cor = f0 * hv_north;
                    const float hv_north_cor = -f0 * hu_east;
                    const float upx = -k.nX, upy = k.nY;
                    const float rx = upy, ry = -upx;
                    hu_cor = rx * hu_east_cor + ry * hv_north_cor;
                    hv_cor = upx * hu_east_cor + upy * hv_north_cor;
                } else {
                    hu_cor = f0 * hv;
                    hv_cor = -f0 * hu;
                }
                st1 = (X + hu_cor) + b1 / k.dx;
                st2 = (Y + hv_cor) + b2 / k.dy;
            }
            const float L1 = -fd0;
            const float L2 = -fd1 + st1;
            const float L3 = -fd2 + st2;

            float C = 0.0f;
            if (FRIC == kFricLinear) {
                C = k.two_r * a.dt / (P0.e + Hm);
            } else if (FRIC == kFricQuad) {
                if (h < k.desing_eps) {
                    const float u = desingularize(h, hu, k.desing_eps);
                    const float v = desingularize(h, hv, k.desing_eps);
                    C = a.dt * k.r * desingularize(h, sqrtf(u * u + v * v), k.desing_eps);
                } else {
                    const float u = hu / h;
                    const float v = hv / h;
                    C = a.dt * k.r * sqrtf(u * u + v * v) / h;
                }
            }
            float ne, nhu, nhv;
            if (a.rk_step == 0) {
                ne = P0.e + a.dt * L1;
                nhu = (hu + a.dt * L2) / (1.0f + C);
                nhv = (hv + a.dt * L3) / (1.0f + C);
            } else {
                ne = 0.5f * (qn_e + (P0.e + a.dt * L1));
                nhu = (0.5f * (qn_hu + (hu + a.dt * L2))) / (1.0f + 0.5f * C);
                nhv = (0.5f * (qn_hv + (hv + a.dt * L3))) / (1.0f + 0.5f * C);
            }
            if (ne + Hm <= k.cutoff) {
                ne = -Hm + k.cutoff; nhu = 0.0f; nhv = 0.0f;
            }
            ne = fmaxf(-Hm + k.cutoff, ne);
            if (!(isfinite(ne) && isfinite(nhu) && isfinite(nhv)) && a.status) atomicOr(a.status, 1u);

            // own cell plus its periodic ghost images (NS rows, EW columns)
            int rows_img[3] = {j, -1, -1};
            int cols_img[3] = {cl, -1, -1};
            if (k.bcN == kPeriodic) {
                if (j < 4) rows_img[1] = j + k.ny;
                if (j >= k.ny) rows_img[2] = j - k.ny;
            }
            if (k.bcE == kPeriodic) {
                if (cl < 4) cols_img[1] = cl + k.nx;
                if (cl >= k.nx) cols_img[2] = cl - k.nx;
            }
#pragma unroll
            for (int ri = 0; ri < 3; ++ri) {
#pragma unroll
                for (int ci = 0; ci < 3; ++ci) {
                    const int rr = rows_img[ri], cc = cols_img[ci];
                    if (rr < 0 || cc < 0) continue;
                    const size_t o = (size_t)rr * a.pout + cc;
                    a.eta_out[o] = ne; a.hu_out[o] = nhu; a.hv_out[o] = nhv;
                }
            }
        }

        // ---- slide the window -----------------------------------------------
        P0 = P1; P1 = P2;
        S0 = S1;
        Gs = Gn;
        Ha[0] = Ha[1]; Ha[1] = Ha[2]; Ha[2] = Ha[3];
        Hb[0] = Hb[1]; Hb[1] = Hb[2]; Hb[2] = Hb[3];
        f0 = f1; f1 = f2;
    }
}

}  // namespace go
