// Reverse mode (adjoint) of one CDKLM16 Runge-Kutta stage.
//
// Forward stage (cdklm_swe_2D, CDKLM16_kernel.cu:429-1006): per cell the
// primitive state (eta, u, v); minmod slopes of u, v and of the Coriolis
// potentials K (x) and L (y) with the positivity adjustment (adjustSlopes,
// CDKLM16_kernel.cu:148-245); central-upwind face fluxes
// (CDKLM16_kernel.cu:80-140, 246-370); bathymetry, Coriolis and wind sources
// and bottom friction (CDKLM16_kernel.cu:817-904); the RK update
// (CDKLM16_kernel.cu:905-1004).  Given lambda, the adjoint of the stage
// output, this kernel returns the adjoint with respect to the stage input,
// to Q^n (stage 1) and to the wind-stress field.  Non-smooth operations
// (minmod, the max/min wave speeds, the zero-flux cut, max(h, 0), the upwind
// choice of the transverse flux, the dry clamp) are differentiated as the
// subgradient of the branch the forward recomputation takes.
//
// Scope: north-up grids (angle 0), with land and shallow cells.  The cell
// state map has four branches (CDKLM16_kernel.cu:551-602): land (all four
// corners land: the dry flag, a constant), dry (h <= cutoff: a constant
// state), desingularised (cutoff < h < desing_eps: u = hu / D(h) with
// D(h) = h^2 / (2 eps) + eps / 2, common.cu:822-824) and wet (u = hu / h);
// the constant branches pass no adjoint to their input.  A face with a land
// cell on either side carries no flux (CDKLM16_kernel.cu:271-273) and passes
// none either; corners on land read as the dry flag, as the forward's do.
//
// Arithmetic: this unit is compiled with FMA contraction (the adjoint is
// compared with FP64 derivatives, not bit for bit), but every value a branch
// decision reads (minmod arguments, the positivity tests, face depths and
// velocities, wave speeds) keeps the forward kernel's rounding: products that
// feed a sum are written with __fmul_rn so that they are never contracted.
//
// Two launch forms compute the same adjoint.  Tile form: one CTA per output
// tile of TX x TY cells of the ghost-inclusive grid.  The forward state of the tile plus a 3-cell halo is recomputed in
// shared memory; the adjoint then flows output -> fluxes -> slopes -> cell
// state as in the forward, each face handled once (two passes, even and odd
// faces, so that no two threads update one cell at the same time) and each
// slope gathered by its three cells.  The adjoint of ghost cells is written
// to the ghost positions and moved to the interior cells they mirror or wrap
// (k_adj_fold) afterwards.
#include <vector>

#include "internal.h"
#include "trace.h"

using namespace go;

namespace {

constexpr int HALO = 3;
constexpr int NT = 256;

// Programmatic dependent launch of the stage-adjoint and fold kernels
// (launch_pdl): the blocks of such a grid may be scheduled while the kernel
// before it on the stream is still running.  pdl_enter is the first statement
// of each of these kernels: griddepcontrol.wait holds the block until the
// previous grid has completed and its writes are visible (it returns at once
// for a launch without the attribute); launch_dependents then lets the next
// launch on the stream be scheduled once every block of this grid has started.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

struct AdjArgs {
    Scheme k;
    float dt;
    const float *qe, *qu, *qv; int pq;     // stage input (ghost-inclusive)
    const float *oe, *ou, *ov; int po;     // stage output
    const float *le, *lu, *lv; int pl;     // adjoint of the output (interior cells read)
    float *ie, *iu, *iv; int pi;           // adjoint of the input (all cells written)
    float *ne, *nu, *nv; int pn;           // stage 1: adjoint of Q^n (written);
                                           // stage 0: added to the input adjoint (may be null)
    float *wx, *wy; int pw;                // wind adjoint, accumulated (interior-indexed, may be null)
    const float* Hi; int phi;
    const float* f_rows;
    unsigned int* status;
    int rows;                              // rows per strip (marching form)
    int land;                              // the bathymetry may hold land (the domain's land flag)
};

// Branch codes
enum { kBrZero = 0, kBrBack = 1, kBrCent = 2, kBrFwd = 3 };
enum { kAdjNone = 0, kAdjA = 1, kAdjB = 2 };

// Which argument minmod_raw (common.cu:544-551) returns: the one of least
// magnitude when the three signs agree, else none.  When that magnitude is
// exactly zero (a state at rest, or the mirrored difference at a wall) the
// slope is taken as locally constant: the zero subgradient.
__device__ __forceinline__ int mm_branch(float b, float c, float f) {
    const uint32_t sb = __float_as_uint(b), sc = __float_as_uint(c), sf = __float_as_uint(f);
    if ((((sb ^ sc) | (sc ^ sf)) & 0x80000000u) != 0u) return kBrZero;
    const float ab = fabsf(b), ac = fabsf(c), af = fabsf(f);
    if (ab <= ac && ab <= af) return ab > 0.0f ? kBrBack : kBrZero;
    if (ac <= af) return ac > 0.0f ? kBrCent : kBrZero;
    return af > 0.0f ? kBrFwd : kBrZero;
}

// d slope / d value at position pos (-1 left, 0 centre, +1 right) for the
// minmod of theta*(c-l), (r-l)/2, theta*(r-c).
__device__ __forceinline__ float slope_coef(int br, int pos, float theta) {
    if (br == kBrBack) return pos < 0 ? -theta : (pos == 0 ? theta : 0.0f);
    if (br == kBrCent) return pos < 0 ? -0.5f : (pos == 0 ? 0.0f : 0.5f);
    if (br == kBrFwd) return pos < 0 ? 0.0f : (pos == 0 ? -theta : theta);
    return 0.0f;
}

// d (sum of the Coriolis terms inside K or L) / d f*v at position pos:
// backward (fc + fl), central ((fr + 2 fc) + fl)/2... scaled by theta*g or g/2.
__device__ __forceinline__ float pot_coef(int br, int pos, float theta_g, float half_g) {
    if (br == kBrBack) return pos > 0 ? 0.0f : theta_g;
    if (br == kBrCent) return pos == 0 ? 2.0f * half_g : half_g;
    if (br == kBrFwd) return pos < 0 ? 0.0f : theta_g;
    return 0.0f;
}

__device__ __forceinline__ float flip(bool f) { return f ? -1.0f : 1.0f; }

struct Trip3 { float a, b, c; };

// Cell classes of the state map (2 bits).
enum { kCellWet = 0, kCellDesing = 1, kCellDry = 2, kCellLand = 3 };

// Denominator of desingularize (common.cu:822-824) and its derivative in h:
// D = max(min(a, eps), |h|) with a = h^2/(2 eps) + eps/2, which is a for
// |h| <= eps (then a <= eps and a >= |h|), and |h| beyond.
__device__ __forceinline__ float desing_den(float h, float eps) {
    const float a = (float)((double)(h * h / (2.0f * eps)) + 0.5 * (double)eps);
    return fmaxf(fminf(a, eps), fabsf(h));
}
__device__ __forceinline__ float desing_den_dh(float h, float eps) {
    return (fabsf(h) <= eps) ? h / eps : (h < 0.0f ? -1.0f : 1.0f);
}

// Cell state (e, u, v) and class of one cell from its input (e, hu, hv) and
// its (dry-flagged) corners, as the forward's to_prim with land: Bm is the
// mean over the wet corners (initBm).
template <bool LAND>
__device__ __forceinline__ int adj_prim(float qe, float qu, float qv, float sw, float nw, float se, float ne,
                                        const Scheme& k, float& e, float& u, float& v) {
    const float s4 = ((sw + nw) + se) + ne;
    const float Bm = LAND ? cell_bm(sw, nw, se, ne, s4, k) : __fmul_rn(s4, 0.25f);
    if (LAND && fabsf(Bm - k.land) <= kDryEps) { e = kDryFlag; u = 0.0f; v = 0.0f; return kCellLand; }
    const float h = qe + Bm;
    if (h < k.desing_eps) {
        if (h <= k.cutoff) { e = -Bm + k.cutoff; u = 0.0f; v = 0.0f; return kCellDry; }
        e = qe;
        u = desingularize(h, qu, k.desing_eps);
        v = desingularize(h, qv, k.desing_eps);
        return kCellDesing;
    }
    e = qe; u = qu / h; v = qv / h;
    return kCellWet;
}

// Adjoint of the state map: (lE, lU, lV) of the input (e, hu, hv) from the
// adjoint (l0, l1, l2) of the state (e, u, v); zero for the constant classes.
template <bool LAND>
__device__ __forceinline__ Trip3 adj_prim_vjp(int cls, float qe, float u, float v, float sw, float nw, float se,
                                              float ne, const Scheme& k, float l0, float l1, float l2) {
    if (cls >= kCellDry) return Trip3{0.0f, 0.0f, 0.0f};
    const float s4 = ((sw + nw) + se) + ne;
    const float Bm = LAND ? cell_bm(sw, nw, se, ne, s4, k) : __fmul_rn(s4, 0.25f);
    const float h = qe + Bm;
    float D = h, gD = 1.0f / h;                 // u = hu / D(h): du/dh = -u D'(h) / D
    if (cls == kCellDesing) {
        D = desing_den(h, k.desing_eps);
        gD = desing_den_dh(h, k.desing_eps) / D;
    }
    return Trip3{l0 - (l1 * u + l2 * v) * gD, l1 / D, l2 / D};
}

struct CuGrad { float hm, um, vm, hp, up, vp; };

// Vector-Jacobian product of the central-upwind flux (CDKLM16_kernel.cu:80-140)
// for the face states (hm, um, vm | hp, up, vp) and flux adjoint (l0, l1, l2).
__device__ __forceinline__ CuGrad cu_vjp(float hm, float um, float vm, float hp, float up, float vp,
                                         float l0, float l1, float l2, const Scheme& k) {
    CuGrad g{0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    const bool wp = hp > k.cutoff, wm = hm > k.cutoff;
    float Fp0 = 0.0f, Fp1 = 0.0f, upw = 0.0f, cp = 0.0f;
    if (wp) {
        Fp0 = hp * up;
        Fp1 = hp * up * up + k.half_g * hp * hp;
        upw = up;
        cp = sqrtf(k.g * hp);
    }
    float Fm0 = 0.0f, Fm1 = 0.0f, umw = 0.0f, cm = 0.0f;
    if (wm) {
        Fm0 = hm * um;
        Fm1 = hm * um * um + k.half_g * hm * hm;
        umw = um;
        cm = sqrtf(k.g * hm);
    }
    const float a1 = umw - cm, a2 = upw - cp;
    const float b1 = umw + cm, b2 = upw + cp;
    const float am = fminf(fminf(a1, a2), 0.0f);
    const float ap = fmaxf(fmaxf(b1, b2), 0.0f);
    if (fabsf(ap - am) < k.flux_slope_eps) return g;
    const float id = 1.0f / (ap - am);
    const float dh = hp - hm, dF0 = Fp0 - Fm0;
    const float F0 = ((ap * Fm0 - am * Fp0) + ap * am * dh) * id;
    const float F1 = ((ap * Fm1 - am * Fp1) + ap * am * dF0) * id;
    const float lap = l0 * ((Fm0 + am * dh) - F0) * id + l1 * ((Fm1 + am * dF0) - F1) * id;
    const float lam = l0 * ((ap * dh - Fp0) + F0) * id + l1 * ((ap * dF0 - Fp1) + F1) * id;
    const float apam = ap * am * id;
    const float lFm0 = l0 * ap * id - l1 * apam, lFp0 = l1 * apam - l0 * am * id;
    const float lFm1 = l1 * ap * id, lFp1 = -l1 * am * id;
    const bool up_side = (um + up > 0.0f);
    const float lFm2 = up_side ? l2 : 0.0f, lFp2 = up_side ? 0.0f : l2;
    g.hp = l0 * apam;
    g.hm = -l0 * apam;
    float lumw = 0.0f, lcm = 0.0f, lupw = 0.0f, lcp = 0.0f;
    if (fmaxf(b1, b2) > 0.0f) {
        if (b1 >= b2) { lumw += lap; lcm += lap; } else { lupw += lap; lcp += lap; }
    }
    if (fminf(a1, a2) < 0.0f) {
        if (a1 <= a2) { lumw += lam; lcm -= lam; } else { lupw += lam; lcp -= lam; }
    }
    if (wp) {
        g.hp += lFp0 * up + lFp1 * (up * up + k.g * hp) + lFp2 * up * vp + lcp * (0.5f * k.g / cp);
        g.up += lupw + lFp0 * hp + lFp1 * 2.0f * hp * up + lFp2 * hp * vp;
        g.vp += lFp2 * hp * up;
    }
    if (wm) {
        g.hm += lFm0 * um + lFm1 * (um * um + k.g * hm) + lFm2 * um * vm + lcm * (0.5f * k.g / cm);
        g.um += lumw + lFm0 * hm + lFm1 * 2.0f * hm * um + lFm2 * hm * vm;
        g.vm += lFm2 * hm * um;
    }
    return g;
}

// Tile form.  Shared arrays are kept in the shape each phase needs: the
// state and lambda_L on the whole region (rows padded to an odd stride, so
// that threads walking down rows hit distinct banks), x-slope data on the
// tile rows only, y-slope data on the tile columns only (74.7 KB per CTA,
// three CTAs per SM).
// Tile of TX x TY output cells and its region (the tile with a HALO-cell
// rim): the region's row stride RXS, and the sizes of the region arrays
// (NR), the tile-row arrays (NXR) and the tile-column arrays (NYC).
template <int TX_, int TY_>
struct TileDims {
    static constexpr int TX = TX_, TY = TY_;
    static constexpr int RX = TX + 2 * HALO, RY = TY + 2 * HALO;
    static constexpr int RXS = RX + 1;       // padded row stride of region arrays
    static constexpr int NR = RXS * RY;      // region
    static constexpr int NXR = TY * RXS;     // tile rows x region columns
    static constexpr int NYC = RY * TX;      // region rows x tile columns
};

template <int TX_, int TY_>
struct AdjSmem {
    using D = TileDims<TX_, TY_>;
    static constexpr int RX = D::RX, RY = D::RY, NR = D::NR, NXR = D::NXR, NYC = D::NYC;
    float R0[NR], R1[NR], R2[NR];           // primitive state (eta, u, v)
    float LL0[NR], LL1[NR], LL2[NR];        // adjoint of the cell tendencies L
    float Ux[NXR], Vx[NXR], Kx[NXR];        // x slopes (K after adjustment)
    float Ax0[NXR], Ax1[NXR], Ax2[NXR];     // adjoint of (eta, u, v): own terms + x faces
    float AKx[NXR], AUx[NXR], AVx[NXR];     // adjoint of the x slopes
    float Uy[NYC], Vy[NYC], Ly[NYC];        // y slopes
    float Ay0[NYC], Ay1[NYC], Ay2[NYC];     // adjoint of (eta, u, v): y faces
    float ALy[NYC], AUy[NYC], AVy[NYC];     // adjoint of the y slopes
    uint16_t bx[NXR], by[NYC];              // branch codes
    float Hi[(RY + 1) * (RX + 1)];
    float f[RY];
};

// branch-code fields (x codes in bx, y codes in by)
__device__ __forceinline__ int br_u(uint32_t b) { return b & 3; }
__device__ __forceinline__ int br_v(uint32_t b) { return (b >> 2) & 3; }
__device__ __forceinline__ int br_k(uint32_t b) { return (b >> 4) & 3; }
__device__ __forceinline__ int br_a(uint32_t b) { return (b >> 6) & 3; }
__device__ __forceinline__ bool br_has(uint32_t b) { return (b >> 8) & 1; }

template <int FRIC, bool STAGE1, int TX, int TY, int MINB, bool LAND>
__global__ void __launch_bounds__(NT, MINB) cdklm_adjoint_stage_kernel(const AdjArgs a) {
    pdl_enter();
    using D = TileDims<TX, TY>;
    constexpr int RX = D::RX, RY = D::RY, RXS = D::RXS, NXR = D::NXR, NYC = D::NYC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    AdjSmem<TX, TY>& S = *reinterpret_cast<AdjSmem<TX, TY>*>(smem_raw);
    const Scheme& k = a.k;
    const int nx = k.nx, ny = k.ny;
    const int ox = blockIdx.x * TX - HALO, oy = blockIdx.y * TY - HALO;
    const int tid = threadIdx.x;
    const bool wallN = k.bcN == kWall, wallS = k.bcS == kWall, wallE = k.bcE == kWall, wallW = k.bcW == kWall;
    const float inv2g = 1.0f / k.two_g;
    auto RI = [](int ry, int rx) { return ry * RXS + rx; };                 // region
    auto XI = [](int ry, int rx) { return (ry - HALO) * RXS + rx; };        // tile rows
    auto YI = [](int ry, int rx) { return ry * TX + (rx - HALO); };         // tile columns

    // ---- corners and Coriolis rows; zero the accumulators ----------------
    for (int c = tid; c < (RY + 1) * (RX + 1); c += NT) {
        const int ry = c / (RX + 1), rx = c % (RX + 1);
        const int j = min(max(oy + ry, 0), ny + 4), i = min(max(ox + rx, 0), nx + 4);
        const float H = a.Hi[(size_t)j * a.phi + i];
        S.Hi[c] = LAND ? corner(H, k) : H;
    }
    for (int r = tid; r < RY; r += NT) S.f[r] = a.f_rows[min(max(oy + r, 0), ny + 3)];
    for (int c = tid; c < NXR; c += NT) {
        S.Ax0[c] = 0.0f; S.Ax1[c] = 0.0f; S.Ax2[c] = 0.0f;
        S.AKx[c] = 0.0f; S.AUx[c] = 0.0f; S.AVx[c] = 0.0f;
        S.bx[c] = 0;
    }
    for (int c = tid; c < NYC; c += NT) {
        S.Ay0[c] = 0.0f; S.Ay1[c] = 0.0f; S.Ay2[c] = 0.0f;
        S.ALy[c] = 0.0f; S.AUy[c] = 0.0f; S.AVy[c] = 0.0f;
        S.by[c] = 0;
    }
    __syncthreads();
    auto HI = [&](int ry, int rx) { return S.Hi[ry * (RX + 1) + rx]; };

    // ---- P1: primitive state of every region cell (loads first) ---------
    {
        constexpr int IT = (RX * RY + NT - 1) / NT;
        float qe[IT], qu[IT], qv[IT];
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int c = tid + it * NT;
            qe[it] = 0.0f; qu[it] = 0.0f; qv[it] = 0.0f;
            if (c < RX * RY) {
                const int ry = c / RX, rx = c % RX;
                const int j = oy + ry, i = ox + rx;
                if (j >= 0 && j < ny + 4 && i >= 0 && i < nx + 4) {
                    int sj = j, si = i;
                    float shu = 1.0f, shv = 1.0f;
                    if (wallS && j < 2) { sj = 3 - j; shv = -1.0f; }
                    if (wallN && j > ny + 1) { sj = 2 * ny + 3 - j; shv = -1.0f; }
                    if (wallW && i < 2) { si = 3 - i; shu = -1.0f; }
                    if (wallE && i > nx + 1) { si = 2 * nx + 3 - i; shu = -1.0f; }
                    const size_t q = (size_t)sj * a.pq + si;
                    qe[it] = a.qe[q]; qu[it] = a.qu[q] * shu; qv[it] = a.qv[q] * shv;
                }
            }
        }
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int c = tid + it * NT;
            if (c >= RX * RY) continue;
            const int ry = c / RX, rx = c % RX;
            const int j = oy + ry, i = ox + rx;
            float e = 0.0f, u = 0.0f, v = 0.0f;
            if (j >= 0 && j < ny + 4 && i >= 0 && i < nx + 4) {
                const int cls = adj_prim<LAND>(qe[it], qu[it], qv[it], HI(ry, rx), HI(ry + 1, rx), HI(ry, rx + 1),
                                         HI(ry + 1, rx + 1), k, e, u, v);
                if (ry >= HALO && ry < HALO + TY) S.bx[XI(ry, rx)] = (uint16_t)(cls << 9);
            }
            const int r = RI(ry, rx);
            S.R0[r] = e; S.R1[r] = u; S.R2[r] = v;
            S.LL0[r] = 0.0f; S.LL1[r] = 0.0f; S.LL2[r] = 0.0f;
        }
    }
    __syncthreads();

    // ---- P2: x slopes on the tile rows, y slopes on the tile columns -------
    for (int c = tid; c < TY * RX; c += NT) {
        const int ry = HALO + c / RX, rx = c % RX;
        const int j = oy + ry, i = ox + rx;
        if (rx < 1 || rx > RX - 2 || !(j >= 2 && j < ny + 2 && i >= 1 && i <= nx + 2)) continue;
        const int q = RI(ry, rx);
        const float fJ = S.f[ry];
        const float ul = S.R1[q - 1], uc = S.R1[q], ur = S.R1[q + 1];
        const float vl = S.R2[q - 1], vc = S.R2[q], vr = S.R2[q + 1];
        const float el = S.R0[q - 1], ec = S.R0[q], er = S.R0[q + 1];
        const int xi = XI(ry, rx);
        S.Ux[xi] = minmod_slope(ul, uc, ur, k.theta);
        S.Vx[xi] = minmod_slope(vl, vc, vr, k.theta);
        const int bu = mm_branch((uc - ul) * k.theta, (ur - ul) * 0.5f, (ur - uc) * k.theta);
        const int bv = mm_branch((vc - vl) * k.theta, (vr - vl) * 0.5f, (vr - vc) * k.theta);
        const float fvl = (vl * flip((wallW && i - 1 < 2) || (wallE && i - 1 > nx + 1))) * fJ;
        const float fvc = (vc * flip((wallW && i < 2) || (wallE && i > nx + 1))) * fJ;
        const float fvr = (vr * flip((wallW && i + 1 < 2) || (wallE && i + 1 > nx + 1))) * fJ;
        const float bw = k.theta_g * ((ec - el) - __fmul_rn(k.V, fvc + fvl));
        const float ce = k.half_g * ((er - el) - __fmul_rn(k.V, (fvr + __fmul_rn(2.0f, fvc)) + fvl));
        const float fw = k.theta_g * ((er - ec) - __fmul_rn(k.V, fvc + fvr));
        const float Kraw = minmod_raw(bw, ce, fw);
        const int bk = mm_branch(bw, ce, fw);
        const float dxfv = __fmul_rn(k.dx * fJ, vc * flip((wallW && i < 2) || (wallE && i > nx + 2)));
        const float Hw = 0.5f * (HI(ry, rx) + HI(ry + 1, rx));
        const float He = 0.5f * (HI(ry, rx + 1) + HI(ry + 1, rx + 1));
        const float hw = (ec + Hw) - (Kraw + dxfv) / k.two_g;
        const float he = (ec + He) + (Kraw + dxfv) / k.two_g;
        float K = Kraw;
        int ba = kAdjNone;
        if (!(hw > 0.0f)) { K = -dxfv + __fmul_rn(k.two_g, ec + Hw); ba = kAdjA; }
        if (!(he > 0.0f)) { K = -dxfv - __fmul_rn(k.two_g, ec + He); ba = kAdjB; }
        S.Kx[xi] = K;
        S.bx[xi] = (uint16_t)((S.bx[xi] & (3 << 9)) | bu | (bv << 2) | (bk << 4) | (ba << 6) | (1 << 8));
    }
    for (int c = tid; c < RY * TX; c += NT) {
        const int ry = c / TX, rx = HALO + c % TX;
        const int j = oy + ry, i = ox + rx;
        if (ry < 1 || ry > RY - 2 || !(i >= 2 && i < nx + 2 && j >= 1 && j <= ny + 2)) continue;
        const int q = RI(ry, rx);
        const float ul = S.R1[q - RXS], uc = S.R1[q], ur = S.R1[q + RXS];
        const float vl = S.R2[q - RXS], vc = S.R2[q], vr = S.R2[q + RXS];
        const float el = S.R0[q - RXS], ec = S.R0[q], er = S.R0[q + RXS];
        const int yi = YI(ry, rx);
        S.Uy[yi] = minmod_slope(ul, uc, ur, k.theta);
        S.Vy[yi] = minmod_slope(vl, vc, vr, k.theta);
        const int bu = mm_branch((uc - ul) * k.theta, (ur - ul) * 0.5f, (ur - uc) * k.theta);
        const int bv = mm_branch((vc - vl) * k.theta, (vr - vl) * 0.5f, (vr - vc) * k.theta);
        const float ful = (ul * flip((wallS && j - 1 < 2) || (wallN && j - 1 > ny + 1))) * S.f[ry - 1];
        const float fuc = (uc * flip((wallS && j < 2) || (wallN && j > ny + 1))) * S.f[ry];
        const float fur = (ur * flip((wallS && j + 1 < 2) || (wallN && j + 1 > ny + 1))) * S.f[ry + 1];
        const float bw = k.theta_g * ((ec - el) + __fmul_rn(k.U, fuc + ful));
        const float ce = k.half_g * ((er - el) + __fmul_rn(k.U, (fur + __fmul_rn(2.0f, fuc)) + ful));
        const float fw = k.theta_g * ((er - ec) + __fmul_rn(k.U, fuc + fur));
        const float Lraw = minmod_raw(bw, ce, fw);
        const int bl = mm_branch(bw, ce, fw);
        const float dyfu = __fmul_rn(k.dy * S.f[ry], uc * flip((wallS && j < 2) || (wallN && j > ny + 2)));
        const float Hs = 0.5f * (HI(ry, rx) + HI(ry, rx + 1));
        const float Hn = 0.5f * (HI(ry + 1, rx) + HI(ry + 1, rx + 1));
        const float hs = (ec + Hs) - (Lraw - dyfu) / k.two_g;
        const float hn = (ec + Hn) + (Lraw - dyfu) / k.two_g;
        float L = Lraw;
        int ba = kAdjNone;
        if (!(hs > 0.0f)) { L = dyfu + __fmul_rn(k.two_g, ec + Hs); ba = kAdjA; }
        if (!(hn > 0.0f)) { L = dyfu - __fmul_rn(k.two_g, ec + Hn); ba = kAdjB; }
        S.Ly[yi] = L;
        S.by[yi] = (uint16_t)(bu | (bv << 2) | (bl << 4) | (ba << 6) | (1 << 8));
    }

    // ---- P3: adjoint of the RK update, friction and sources on the cross --
    // (tile rows x region columns 1..RX-2, plus tile columns x rows 1, 2 and
    // the two rows above the tile), loads first
    {
        constexpr int NCROSS = TY * (RX - 2) + 4 * TX;
        constexpr int IT = (NCROSS + NT - 1) / NT;
        float lE[IT], lU[IT], lV[IT], oE[IT], oU[IT], oV[IT], wX[IT], wY[IT];
        int cry[IT], crx[IT];
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int c = tid + it * NT;
            int ry = -1, rx = -1;
            if (c < TY * (RX - 2)) {
                ry = HALO + c / (RX - 2);
                rx = 1 + c % (RX - 2);
            } else if (c < NCROSS) {
                const int t = c - TY * (RX - 2), kk = t / TX;
                rx = HALO + t % TX;
                ry = (kk < 2) ? 1 + kk : HALO + TY + (kk - 2);
            }
            cry[it] = ry; crx[it] = rx;
            lE[it] = lU[it] = lV[it] = oE[it] = oU[it] = oV[it] = wX[it] = wY[it] = 0.0f;
            if (ry < 0) continue;
            const int j = oy + ry, i = ox + rx;
            if (j < 2 || j >= ny + 2 || i < 2 || i >= nx + 2) continue;
            const size_t lo = (size_t)j * a.pl + i, oo = (size_t)j * a.po + i;
            lE[it] = a.le[lo]; lU[it] = a.lu[lo]; lV[it] = a.lv[lo];
            oE[it] = a.oe[oo]; oU[it] = a.ou[oo]; oV[it] = a.ov[oo];
            const bool tile = ry >= HALO && ry < HALO + TY && rx >= HALO && rx < HALO + TX;
            if (tile && a.wx) {
                const size_t wo = (size_t)(j - 2) * a.pw + (i - 2);
                wX[it] = a.wx[wo];
                wY[it] = a.wy[wo];
            }
        }
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int ry = cry[it], rx = crx[it];
            if (ry < 0) continue;
            const int j = oy + ry, i = ox + rx;
            if (j < 2 || j >= ny + 2 || i < 2 || i >= nx + 2) continue;
            const bool tile = ry >= HALO && ry < HALO + TY && rx >= HALO && rx < HALO + TX;
            const int r = RI(ry, rx);
            float le = lE[it], lu = lU[it], lv = lV[it];
            const float s4 = ((HI(ry, rx) + HI(ry + 1, rx)) + HI(ry, rx + 1)) + HI(ry + 1, rx + 1);
            const float Hm = __fmul_rn(0.25f, s4);
            if (oE[it] + Hm <= k.cutoff) { le = 0.0f; lu = 0.0f; lv = 0.0f; }   // dry clamp: constant output
            const float e = S.R0[r], u = S.R1[r], v = S.R2[r];
            const float h = e + Hm;
            const bool wet = h > k.cutoff;
            const float hu = wet ? u * h : 0.0f, hv = wet ? v * h : 0.0f;
            float Cf = 0.0f, sq = 0.0f, uw = 0.0f, vw = 0.0f, Dn = h;
            if (FRIC == kFricQuad) {
                // below desing_eps the speed and C are desingularised (CDKLM16_kernel.cu:884-900)
                if (h < k.desing_eps) Dn = desing_den(h, k.desing_eps);
                uw = hu / Dn; vw = hv / Dn;
                sq = sqrtf(uw * uw + vw * vw);
                Cf = (a.dt * k.r * sq) / Dn;
            } else if (FRIC == kFricLinear) {
                Cf = (k.two_r * a.dt) / h;
            }
            const float w = STAGE1 ? 0.5f : 1.0f;
            const float iD = 1.0f / (1.0f + w * Cf);
            const float lL1 = w * a.dt * le, lL2 = w * a.dt * lu * iD, lL3 = w * a.dt * lv * iD;
            S.LL0[r] = lL1; S.LL1[r] = lL2; S.LL2[r] = lL3;
            if (!tile) continue;        // the own-cell terms are needed for the tile's cells only
            float lhu = w * lu * iD, lhv = w * lv * iD, leta = w * le, lh = 0.0f;
            const float lCf = -w * (lu * oU[it] + lv * oV[it]) * iD;
            if (FRIC == kFricQuad) {
                const float ls = lCf * a.dt * k.r / Dn;
                float lD = -lCf * Cf / Dn;
                if (sq > 0.0f) {
                    const float luw = ls * uw / sq, lvw = ls * vw / sq;
                    lhu += luw / Dn; lhv += lvw / Dn;
                    lD -= (luw * uw + lvw * vw) / Dn;
                }
                lh += (h < k.desing_eps) ? lD * desing_den_dh(h, k.desing_eps) : lD;
            } else if (FRIC == kFricLinear) {
                lh -= lCf * Cf / h;
            }
            const float fc = S.f[ry];
            if (h >= k.cutoff && e != kDryFlag) {
                const float Hx = 0.5f * (HI(ry, rx + 1) + HI(ry + 1, rx + 1)) - 0.5f * (HI(ry, rx) + HI(ry + 1, rx));
                const float Hy = 0.5f * (HI(ry + 1, rx) + HI(ry + 1, rx + 1)) - 0.5f * (HI(ry, rx) + HI(ry, rx + 1));
                lhv += fc * lL2;
                lhu -= fc * lL3;
                leta += lL2 * k.g * Hx / k.dx + lL3 * k.g * Hy / k.dy;
                if (a.wx) {
                    const size_t wo = (size_t)(j - 2) * a.pw + (i - 2);
                    a.wx[wo] = wX[it] + lL2;
                    a.wy[wo] = wY[it] + lL3;
                }
            }
            float lR1 = 0.0f, lR2 = 0.0f;
            if (wet) {
                lh += lhu * u + lhv * v;
                lR1 = lhu * h;
                lR2 = lhv * h;
            }
            const int xi = XI(ry, rx);
            S.Ax0[xi] = lh + leta; S.Ax1[xi] = lR1; S.Ax2[xi] = lR2;
            if (STAGE1) {
                const size_t no = (size_t)j * a.pn + i;
                a.ne[no] = w * le;
                a.nu[no] = w * lu * iD;
                a.nv[no] = w * lv * iD;
            }
        }
    }
    __syncthreads();

    // ---- P4: faces, even then odd (x faces: consecutive threads on
    // consecutive rows; y faces: on consecutive columns) -------------------
    constexpr int NXH = (RX - 2) / 2;        // face pairs per tile row: m at 1 + parity + 2p
    constexpr int NYH = (RY - 2) / 2;        // face pairs per tile column
    for (int parity = 0; parity < 2; ++parity) {
        const int nxi = TY * NXH, nyi = TX * NYH;
        for (int it = tid; it < nxi + nyi; it += NT) {
            if (it < nxi) {
                const int ry = HALO + it % TY;
                const int rx = 1 + parity + 2 * (it / TY);
                if (rx > RX - 3) continue;
                const int j = oy + ry, im = ox + rx, ip = im + 1;
                if (j < 2 || j >= ny + 2 || im < 1 || im > nx + 1) continue;
                const int m = RI(ry, rx), p = m + 1;
                if (S.R0[m] == kDryFlag || S.R0[p] == kDryFlag) continue;   // land beside the face: no flux
                const int xm = XI(ry, rx), xp = xm + 1;
                const float fJ = S.f[ry];
                const float Rmu = S.R1[m] + __fmul_rn(0.5f, S.Ux[xm]), Rmv = S.R2[m] + __fmul_rn(0.5f, S.Vx[xm]);
                const float Rpu = S.R1[p] - __fmul_rn(0.5f, S.Ux[xp]), Rpv = S.R2[p] - __fmul_rn(0.5f, S.Vx[xp]);
                const float fm = flip(wallW && ip == 2), fp = flip(wallE && ip == nx + 2);
                const float Hf = 0.5f * (HI(ry, rx + 1) + HI(ry + 1, rx + 1));
                const float Ep = (S.R0[p] + Hf) - (S.Kx[xp] + __fmul_rn(k.dx * fJ, S.R2[p] * fp)) / k.two_g;
                const float Em = (S.R0[m] + Hf) + (S.Kx[xm] + __fmul_rn(k.dx * fJ, S.R2[m] * fm)) / k.two_g;
                const float hp = fmaxf(Ep, 0.0f), hm = fmaxf(Em, 0.0f);
                const float l0 = (S.LL0[p] - S.LL0[m]) / k.dx;
                const float l1 = (S.LL1[p] - S.LL1[m]) / k.dx;
                const float l2 = (S.LL2[p] - S.LL2[m]) / k.dx;
                const CuGrad g = cu_vjp(hm, Rmu, Rmv, hp, Rpu, Rpv, l0, l1, l2, k);
                if (Ep > 0.0f) {
                    S.Ax0[xp] += g.hp;
                    S.AKx[xp] -= g.hp * inv2g;
                    S.Ax2[xp] -= g.hp * (k.dx * fJ) * fp * inv2g;
                }
                if (Em > 0.0f) {
                    S.Ax0[xm] += g.hm;
                    S.AKx[xm] += g.hm * inv2g;
                    S.Ax2[xm] += g.hm * (k.dx * fJ) * fm * inv2g;
                }
                S.Ax1[xp] += g.up; S.AUx[xp] -= 0.5f * g.up;
                S.Ax2[xp] += g.vp; S.AVx[xp] -= 0.5f * g.vp;
                S.Ax1[xm] += g.um; S.AUx[xm] += 0.5f * g.um;
                S.Ax2[xm] += g.vm; S.AVx[xm] += 0.5f * g.vm;
            } else {
                const int t = it - nxi;
                const int rx = HALO + t % TX;
                const int ry = 1 + parity + 2 * (t / TX);
                if (ry > RY - 3) continue;
                const int i = ox + rx, jm = oy + ry, jp = jm + 1;
                if (i < 2 || i >= nx + 2 || jm < 1 || jm > ny + 1) continue;
                const int m = RI(ry, rx), p = m + RXS;
                if (S.R0[m] == kDryFlag || S.R0[p] == kDryFlag) continue;
                const int ym = YI(ry, rx), yp = ym + TX;
                const float Rmu = S.R1[m] + __fmul_rn(0.5f, S.Uy[ym]), Rmv = S.R2[m] + __fmul_rn(0.5f, S.Vy[ym]);
                const float Rpu = S.R1[p] - __fmul_rn(0.5f, S.Uy[yp]), Rpv = S.R2[p] - __fmul_rn(0.5f, S.Vy[yp]);
                const float fm = flip(wallS && jp == 2), fp = flip(wallN && jp == ny + 2);
                const float fpr = S.f[ry + 1], fmr = S.f[ry];
                const float Hf = 0.5f * (HI(ry + 1, rx) + HI(ry + 1, rx + 1));
                const float Ep = (S.R0[p] + Hf) - (S.Ly[yp] - __fmul_rn(k.dy * fpr, S.R1[p] * fp)) / k.two_g;
                const float Em = (S.R0[m] + Hf) + (S.Ly[ym] - __fmul_rn(k.dy * fmr, S.R1[m] * fm)) / k.two_g;
                const float hp = fmaxf(Ep, 0.0f), hm = fmaxf(Em, 0.0f);
                // G = CU(hm, v, u | hp, v, u) with outputs (G0, G2, G1)
                const float l0 = (S.LL0[p] - S.LL0[m]) / k.dy;
                const float l1 = (S.LL1[p] - S.LL1[m]) / k.dy;
                const float l2 = (S.LL2[p] - S.LL2[m]) / k.dy;
                const CuGrad g = cu_vjp(hm, Rmv, Rmu, hp, Rpv, Rpu, l0, l2, l1, k);
                if (Ep > 0.0f) {
                    S.Ay0[yp] += g.hp;
                    S.ALy[yp] -= g.hp * inv2g;
                    S.Ay1[yp] += g.hp * (k.dy * fpr) * fp * inv2g;
                }
                if (Em > 0.0f) {
                    S.Ay0[ym] += g.hm;
                    S.ALy[ym] += g.hm * inv2g;
                    S.Ay1[ym] -= g.hm * (k.dy * fmr) * fm * inv2g;
                }
                S.Ay2[yp] += g.up; S.AVy[yp] -= 0.5f * g.up;
                S.Ay1[yp] += g.vp; S.AUy[yp] -= 0.5f * g.vp;
                S.Ay2[ym] += g.um; S.AVy[ym] += 0.5f * g.um;
                S.Ay1[ym] += g.vm; S.AUy[ym] += 0.5f * g.vm;
            }
        }
        __syncthreads();
    }

    // ---- P5: positivity adjustment of K (tile rows) and L (tile columns) --
    for (int c = tid; c < TY * (TX + 2); c += NT) {
        const int ry = HALO + c / (TX + 2), rx = HALO - 1 + c % (TX + 2);
        const int xi = XI(ry, rx);
        const uint32_t b = S.bx[xi];
        if (!br_has(b) || br_a(b) == kAdjNone) continue;
        const float lK = S.AKx[xi];
        const int i = ox + rx;
        const float fv = flip((wallW && i < 2) || (wallE && i > nx + 2));
        S.Ax0[xi] += (br_a(b) == kAdjA ? k.two_g : -k.two_g) * lK;
        S.Ax2[xi] -= lK * (k.dx * S.f[ry]) * fv;
        S.AKx[xi] = 0.0f;
    }
    for (int c = tid; c < (TY + 2) * TX; c += NT) {
        const int ry = HALO - 1 + c / TX, rx = HALO + c % TX;
        const int yi = YI(ry, rx);
        const uint32_t b = S.by[yi];
        if (!br_has(b) || br_a(b) == kAdjNone) continue;
        const float lL = S.ALy[yi];
        const int j = oy + ry;
        const float fu = flip((wallS && j < 2) || (wallN && j > ny + 2));
        S.Ay0[yi] += (br_a(b) == kAdjA ? k.two_g : -k.two_g) * lL;
        S.Ay1[yi] += lL * (k.dy * S.f[ry]) * fu;
        S.ALy[yi] = 0.0f;
    }
    __syncthreads();

    // ---- P6: gather the slopes, cell state -> conserved variables --------
    for (int c = tid; c < TX * TY; c += NT) {
        const int ry = HALO + c / TX, rx = HALO + c % TX;
        const int j = oy + ry, i = ox + rx;
        if (j >= ny + 4 || i >= nx + 4) continue;
        const int q = RI(ry, rx), xq = XI(ry, rx), yq = YI(ry, rx);
        float l0 = S.Ax0[xq] + S.Ay0[yq];
        float l1 = S.Ax1[xq] + S.Ay1[yq];
        float l2 = S.Ax2[xq] + S.Ay2[yq];
        float lfv = 0.0f, lfu = 0.0f;
#pragma unroll
        for (int o = -1; o <= 1; ++o) {
            const int pos = -o;       // position of this cell in the stencil of slope cell q+o
            const uint32_t bxo = S.bx[xq + o];
            if (br_has(bxo)) {
                l1 += S.AUx[xq + o] * slope_coef(br_u(bxo), pos, k.theta);
                l2 += S.AVx[xq + o] * slope_coef(br_v(bxo), pos, k.theta);
                const float lk = S.AKx[xq + o];
                const int bk = br_k(bxo);
                l0 += lk * k.g * slope_coef(bk, pos, k.theta);
                lfv -= lk * k.V * pot_coef(bk, pos, k.theta_g, k.half_g);
            }
            const uint32_t byo = S.by[yq + o * TX];
            if (br_has(byo)) {
                l1 += S.AUy[yq + o * TX] * slope_coef(br_u(byo), pos, k.theta);
                l2 += S.AVy[yq + o * TX] * slope_coef(br_v(byo), pos, k.theta);
                const float ll = S.ALy[yq + o * TX];
                const int bl = br_k(byo);
                l0 += ll * k.g * slope_coef(bl, pos, k.theta);
                lfu += ll * k.U * pot_coef(bl, pos, k.theta_g, k.half_g);
            }
        }
        l2 += lfv * S.f[ry] * flip((wallW && i < 2) || (wallE && i > nx + 1));
        l1 += lfu * S.f[ry] * flip((wallS && j < 2) || (wallN && j > ny + 1));
        const Trip3 lq = adj_prim_vjp<LAND>((S.bx[xq] >> 9) & 3, S.R0[q], S.R1[q], S.R2[q], HI(ry, rx), HI(ry + 1, rx),
                                      HI(ry, rx + 1), HI(ry + 1, rx + 1), k, l0, l1, l2);
        float lE = lq.a, lU = lq.b, lV = lq.c;
        if (!STAGE1 && a.ne && j >= 2 && j < ny + 2 && i >= 2 && i < nx + 2) {
            const size_t no = (size_t)j * a.pn + i;
            lE += a.ne[no]; lU += a.nu[no]; lV += a.nv[no];
        }
        const size_t io = (size_t)j * a.pi + i;
        a.ie[io] = lE; a.iu[io] = lU; a.iv[io] = lV;
    }
}

// ---------------------------------------------------------------------------
// Column-marching form of the same adjoint stage.
//
// One thread per column, BW columns per block of which the middle BW - 6 are
// written (the x direction of the adjoint reaches 3 columns); a block walks a
// strip of rows upward with the y direction in registers.  At output row j
// the block loads row j+3, takes the y slopes of row j+2 and the own-cell
// adjoint (lambda_L) of row j+2, the y face (j+1, j+2), which completes the
// y-slope adjoint of row j+1, then the whole x direction of row j (x slopes,
// x faces, x-slope adjoints: four shared-memory exchanges), and writes the
// adjoint of row j.  Only 3 priming rows per strip are recomputed.
// ---------------------------------------------------------------------------

struct Cor { float a, b; };                 // corners Hi(r, i), Hi(r, i+1)
struct PrimC { float e, u, v; int cls; };
struct SlopeC { float u, v, K; uint32_t code; };
struct Trip { float a, b, c; };

__device__ __forceinline__ Trip trip0() { return Trip{0.0f, 0.0f, 0.0f}; }

template <int BW>
struct MarchBufs {
    float e[BW], u[BW], v[BW];              // state of the row
    float su[BW], sv[BW], sK[BW];           // x slopes of the row
    uint32_t code[BW];                      // their branch codes
    float l0[BW], l1[BW], l2[BW];           // lambda_L of the row
    float pe[BW], pu[BW], pv[BW], pK[BW], pux[BW], pvx[BW];   // face (t, t+1) -> cell t+1
    float gu[BW], gv[BW], gK[BW];           // x-slope adjoints after the adjustment
};

template <int BW, int FRIC, bool STAGE1, bool EDGE, bool LAND>
__device__ __forceinline__ void adjoint_march_strip(const AdjArgs& a, const int bx, const int by,
                                                    MarchBufs<BW>& sb) {
    const Scheme& k = a.k;
    const int nx = k.nx, ny = k.ny;
    const int t = threadIdx.x;
    const int i = bx * (BW - 6) - 3 + t;
    const int r0 = by * a.rows;
    const int r1 = min(r0 + a.rows, ny + 4);
    const bool wallN = k.bcN == kWall, wallS = k.bcS == kWall, wallE = k.bcE == kWall, wallW = k.bcW == kWall;
    // EDGE = false: the block's columns and rows (with their halos) are all
    // interior, so no wall, ghost or range test is needed
    const bool col_ok = !EDGE || (i >= 0 && i < nx + 4);
    const bool col_int = !EDGE || (i >= 2 && i < nx + 2);
    const bool writer = t >= 3 && t < BW - 3 && col_ok;
    const float inv2g = 1.0f / k.two_g;
    // column mirror of the load and sign of hu
    int si = i;
    float shu = 1.0f;
    if (EDGE && wallW && i < 2) { si = 3 - i; shu = -1.0f; }
    if (EDGE && wallE && i > nx + 1) { si = 2 * nx + 3 - i; shu = -1.0f; }
    const float vflip_kx = flip(EDGE && ((wallW && i < 2) || (wallE && i > nx + 1)));
    const float vflip_adj = flip(EDGE && ((wallW && i < 2) || (wallE && i > nx + 2)));

    auto corners = [&](int r) -> Cor {
        if (EDGE && (r < 0 || r > ny + 4 || i < 0 || i > nx + 3)) return Cor{0.0f, 0.0f};
        const float* row = a.Hi + (size_t)r * a.phi;
        if (!LAND) return Cor{row[i], row[i + 1]};
        return Cor{corner(row[i], k), corner(row[i + 1], k)};
    };
    auto frow = [&](int r) -> float { return a.f_rows[min(max(r, 0), ny + 3)]; };
    // raw (mirrored) state of row r, and its primitive form
    auto load_q = [&](int r) -> Trip {
        if (EDGE && (r < 0 || r >= ny + 4 || !col_ok)) return trip0();
        int sj = r;
        float shv = 1.0f;
        if (EDGE && wallS && r < 2) { sj = 3 - r; shv = -1.0f; }
        if (EDGE && wallN && r > ny + 1) { sj = 2 * ny + 3 - r; shv = -1.0f; }
        const size_t q = (size_t)sj * a.pq + si;
        return Trip{a.qe[q], a.qu[q] * shu, a.qv[q] * shv};
    };
    auto prim = [&](int r, const Trip& q, const Cor& lo, const Cor& hi) -> PrimC {
        if (EDGE && (r < 0 || r >= ny + 4 || !col_ok)) return PrimC{0.0f, 0.0f, 0.0f, kCellWet};
        PrimC p;
        p.cls = adj_prim<LAND>(q.a, q.b, q.c, lo.a, hi.a, lo.b, hi.b, k, p.e, p.u, p.v);
        return p;
    };
    // inputs of the own-cell adjoint of row r (output adjoint, stored stage
    // output, and for output cells the wind adjoint accumulated so far)
    struct OwnIn { float le, lu, lv, oe, ou, ov, wx, wy; };
    auto load_own = [&](int r) -> OwnIn {
        OwnIn o{0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (EDGE && !(col_int && r >= 2 && r < ny + 2)) return o;
        const size_t lo = (size_t)r * a.pl + i, oo = (size_t)r * a.po + i;
        o.le = a.le[lo]; o.lu = a.lu[lo]; o.lv = a.lv[lo];
        o.oe = a.oe[oo]; o.ou = a.ou[oo]; o.ov = a.ov[oo];
        if (a.wx && writer && r >= r0 && r < r1) {
            const size_t wo = (size_t)(r - 2) * a.pw + (i - 2);
            o.wx = a.wx[wo];
            o.wy = a.wy[wo];
        }
        return o;
    };
    // stage 0: the adjoint of Q^n to add at row r
    auto load_qn = [&](int r) -> Trip {
        if (STAGE1 || !a.ne || !(writer && r >= r0 && r < r1)) return trip0();
        if (EDGE && !(col_int && r >= 2 && r < ny + 2)) return trip0();
        const size_t no = (size_t)r * a.pn + i;
        return Trip{a.ne[no], a.nu[no], a.nv[no]};
    };
    auto uflip_ly = [&](int r) -> float { return flip(EDGE && ((wallS && r < 2) || (wallN && r > ny + 1))); };

    // y slopes of row r (cells r-1, r, r+1 of this column); lo/hi corners of row r
    auto yslope = [&](int r, const PrimC& pl, const PrimC& pc, const PrimC& pr, float fl, float fc, float fr,
                      const Cor& clo, const Cor& chi) -> SlopeC {
        SlopeC s{0.0f, 0.0f, 0.0f, 0u};
        if (EDGE && !(col_int && r >= 1 && r <= ny + 2)) return s;
        s.u = minmod_slope(pl.u, pc.u, pr.u, k.theta);
        s.v = minmod_slope(pl.v, pc.v, pr.v, k.theta);
        const int bu = mm_branch((pc.u - pl.u) * k.theta, (pr.u - pl.u) * 0.5f, (pr.u - pc.u) * k.theta);
        const int bv = mm_branch((pc.v - pl.v) * k.theta, (pr.v - pl.v) * 0.5f, (pr.v - pc.v) * k.theta);
        const float ful = (pl.u * uflip_ly(r - 1)) * fl;
        const float fuc = (pc.u * uflip_ly(r)) * fc;
        const float fur = (pr.u * uflip_ly(r + 1)) * fr;
        const float bw = k.theta_g * ((pc.e - pl.e) + __fmul_rn(k.U, fuc + ful));
        const float ce = k.half_g * ((pr.e - pl.e) + __fmul_rn(k.U, (fur + __fmul_rn(2.0f, fuc)) + ful));
        const float fw = k.theta_g * ((pr.e - pc.e) + __fmul_rn(k.U, fuc + fur));
        const float Lraw = minmod_raw(bw, ce, fw);
        const int bl = mm_branch(bw, ce, fw);
        const float dyfu = __fmul_rn(k.dy * fc, pc.u * flip(EDGE && ((wallS && r < 2) || (wallN && r > ny + 2))));
        const float Hs = 0.5f * (clo.a + clo.b);
        const float Hn = 0.5f * (chi.a + chi.b);
        const float hs = (pc.e + Hs) - (Lraw - dyfu) / k.two_g;
        const float hn = (pc.e + Hn) + (Lraw - dyfu) / k.two_g;
        float L = Lraw;
        int ba = kAdjNone;
        if (!(hs > 0.0f)) { L = dyfu + __fmul_rn(k.two_g, pc.e + Hs); ba = kAdjA; }
        if (!(hn > 0.0f)) { L = dyfu - __fmul_rn(k.two_g, pc.e + Hn); ba = kAdjB; }
        s.K = L;
        s.code = (uint32_t)bu | ((uint32_t)bv << 2) | ((uint32_t)bl << 4) | ((uint32_t)ba << 6) | (1u << 16);
        return s;
    };

    // own-cell adjoint of row r: lambda_L and the cell's own (e, u, v) terms
    auto own = [&](int r, const PrimC& p, const Cor& clo, const Cor& chi, float fc, const OwnIn& in,
                   Trip& own_out) -> Trip {
        own_out = trip0();
        if (EDGE && !(col_int && r >= 2 && r < ny + 2)) return trip0();
        float lE = in.le, lU = in.lu, lV = in.lv;
        const float s4 = ((clo.a + chi.a) + clo.b) + chi.b;
        const float Hm = __fmul_rn(0.25f, s4);
        if (in.oe + Hm <= k.cutoff) { lE = 0.0f; lU = 0.0f; lV = 0.0f; }
        const float h = p.e + Hm;
        const bool wet = h > k.cutoff;
        const float hu = wet ? p.u * h : 0.0f, hv = wet ? p.v * h : 0.0f;
        float Cf = 0.0f, sq = 0.0f, uw = 0.0f, vw = 0.0f, Dn = h;
        if (FRIC == kFricQuad) {
            // below desing_eps the speed and C are desingularised (CDKLM16_kernel.cu:884-900)
            if (h < k.desing_eps) Dn = desing_den(h, k.desing_eps);
            uw = hu / Dn; vw = hv / Dn;
            sq = sqrtf(uw * uw + vw * vw);
            Cf = (a.dt * k.r * sq) / Dn;
        } else if (FRIC == kFricLinear) {
            Cf = (k.two_r * a.dt) / h;
        }
        const float w = STAGE1 ? 0.5f : 1.0f;
        const float iD = 1.0f / (1.0f + w * Cf);
        const Trip LL{w * a.dt * lE, w * a.dt * lU * iD, w * a.dt * lV * iD};
        float lhu = w * lU * iD, lhv = w * lV * iD, leta = w * lE, lh = 0.0f;
        const float lCf = -w * (lU * in.ou + lV * in.ov) * iD;
        if (FRIC == kFricQuad) {
            const float ls = lCf * a.dt * k.r / Dn;
            float lD = -lCf * Cf / Dn;
            if (sq > 0.0f) {
                const float luw = ls * uw / sq, lvw = ls * vw / sq;
                lhu += luw / Dn; lhv += lvw / Dn;
                lD -= (luw * uw + lvw * vw) / Dn;
            }
            lh += (h < k.desing_eps) ? lD * desing_den_dh(h, k.desing_eps) : lD;
        } else if (FRIC == kFricLinear) {
            lh -= lCf * Cf / h;
        }
        const bool out_cell = writer && r >= r0 && r < r1;
        if (h >= k.cutoff && p.e != kDryFlag) {
            const float Hx = 0.5f * (clo.b + chi.b) - 0.5f * (clo.a + chi.a);
            const float Hy = 0.5f * (chi.a + chi.b) - 0.5f * (clo.a + clo.b);
            lhv += fc * LL.b;
            lhu -= fc * LL.c;
            leta += LL.b * k.g * Hx / k.dx + LL.c * k.g * Hy / k.dy;
            if (out_cell && a.wx) {
                const size_t wo = (size_t)(r - 2) * a.pw + (i - 2);
                a.wx[wo] = in.wx + LL.b;
                a.wy[wo] = in.wy + LL.c;
            }
        }
        float lR1 = 0.0f, lR2 = 0.0f;
        if (wet) {
            lh += lhu * p.u + lhv * p.v;
            lR1 = lhu * h;
            lR2 = lhv * h;
        }
        own_out = Trip{lh + leta, lR1, lR2};
        if (STAGE1 && out_cell) {
            const size_t no = (size_t)r * a.pn + i;
            a.ne[no] = w * lE;
            a.nu[no] = w * lU * iD;
            a.nv[no] = w * lV * iD;
        }
        return LL;
    };

    // ---- prologue: rows r0-3 .. r0-1 -------------------------------------
    Cor C0 = corners(r0 - 3), C1 = corners(r0 - 2), C2 = corners(r0 - 1), C3 = corners(r0);
    float F0 = frow(r0 - 3), F1 = frow(r0 - 2), F2 = frow(r0 - 1);
    PrimC P0 = prim(r0 - 3, load_q(r0 - 3), C0, C1), P1 = prim(r0 - 2, load_q(r0 - 2), C1, C2);
    PrimC P2 = prim(r0 - 1, load_q(r0 - 1), C2, C3);
    SlopeC S1 = yslope(r0 - 2, P0, P1, P2, F0, F1, F2, C1, C2);
    Trip A0 = trip0(), A1 = trip0(), A2 = trip0();      // lambda of (e, u, v), rows j, j+1, j+2
    Trip B1 = trip0(), B2 = trip0();                    // y-slope adjoints (u, v, L), rows j+1, j+2
    Trip ownx;
    Trip LL0 = trip0();
    Trip LL1 = own(r0 - 2, P1, C1, C2, F1, load_own(r0 - 2), ownx);
    A1 = ownx;
    // loads of the first iteration, then always one iteration ahead
    Trip nq = load_q(r0);
    Cor nC = corners(r0 + 1);
    float nF = frow(r0);
    OwnIn nO = load_own(r0 - 1);
    Trip nQN = load_qn(r0 - 3);

#pragma unroll 1
    for (int j = r0 - 3; j < r1; ++j) {
        // (1) front row j+3 (its loads were issued one iteration ago)
        const Cor C4 = nC;
        const float F3 = nF;
        const Trip q3 = nq;
        const OwnIn o2 = nO;
        const Trip qn0 = nQN;
        nq = load_q(j + 4);
        nC = corners(j + 5);
        nF = frow(j + 4);
        nO = load_own(j + 3);
        nQN = load_qn(j + 1);
        const PrimC P3 = prim(j + 3, q3, C3, C4);
        // (2) y slopes of row j+2
        const SlopeC S2 = yslope(j + 2, P1, P2, P3, F1, F2, F3, C2, C3);
        // (3) own-cell adjoint of row j+2
        const Trip LL2 = own(j + 2, P2, C2, C3, F2, o2, ownx);
        A2.a += ownx.a; A2.b += ownx.b; A2.c += ownx.c;
        // (4) y face (j+1, j+2)
        {
            const int jm = j + 1, jp = j + 2;
            if ((!EDGE || (col_int && jm >= 1 && jm <= ny + 1)) && P1.e != kDryFlag && P2.e != kDryFlag) {
                const float Rmu = P1.u + __fmul_rn(0.5f, S1.u), Rmv = P1.v + __fmul_rn(0.5f, S1.v);
                const float Rpu = P2.u - __fmul_rn(0.5f, S2.u), Rpv = P2.v - __fmul_rn(0.5f, S2.v);
                const float fm = flip(EDGE && wallS && jp == 2), fp = flip(EDGE && wallN && jp == ny + 2);
                const float Hf = 0.5f * (C2.a + C2.b);
                const float Ep = (P2.e + Hf) - (S2.K - __fmul_rn(k.dy * F2, P2.u * fp)) / k.two_g;
                const float Em = (P1.e + Hf) + (S1.K - __fmul_rn(k.dy * F1, P1.u * fm)) / k.two_g;
                const float hp = fmaxf(Ep, 0.0f), hm = fmaxf(Em, 0.0f);
                const float l0 = (LL2.a - LL1.a) / k.dy, l1 = (LL2.b - LL1.b) / k.dy, l2 = (LL2.c - LL1.c) / k.dy;
                const CuGrad g = cu_vjp(hm, Rmv, Rmu, hp, Rpv, Rpu, l0, l2, l1, k);
                if (Ep > 0.0f) {
                    A2.a += g.hp;
                    B2.c -= g.hp * inv2g;
                    A2.b += g.hp * (k.dy * F2) * fp * inv2g;
                }
                if (Em > 0.0f) {
                    A1.a += g.hm;
                    B1.c += g.hm * inv2g;
                    A1.b -= g.hm * (k.dy * F1) * fm * inv2g;
                }
                A2.c += g.up; B2.b -= 0.5f * g.up;
                A2.b += g.vp; B2.a -= 0.5f * g.vp;
                A1.c += g.um; B1.b += 0.5f * g.um;
                A1.b += g.vm; B1.a += 0.5f * g.vm;
            }
        }
        // (5) y-slope adjoint of row j+1 is complete
        if (S1.code & (1u << 16)) {
            const int r = j + 1;
            float lL = B1.c;
            const int ba = (int)((S1.code >> 6) & 3u);
            if (ba != kAdjNone) {
                A1.a += (ba == kAdjA ? k.two_g : -k.two_g) * lL;
                A1.b += lL * (k.dy * F1) * flip(EDGE && ((wallS && r < 2) || (wallN && r > ny + 2)));
                lL = 0.0f;
            }
            const int bu = (int)(S1.code & 3u), bv = (int)((S1.code >> 2) & 3u), bl = (int)((S1.code >> 4) & 3u);
            // cells r-1 (A0, pos -1), r (A1, pos 0), r+1 (A2, pos +1)
            A0.b += B1.a * slope_coef(bu, -1, k.theta) + lL * k.U * pot_coef(bl, -1, k.theta_g, k.half_g) * F0 * uflip_ly(r - 1);
            A1.b += B1.a * slope_coef(bu, 0, k.theta) + lL * k.U * pot_coef(bl, 0, k.theta_g, k.half_g) * F1 * uflip_ly(r);
            A2.b += B1.a * slope_coef(bu, 1, k.theta) + lL * k.U * pot_coef(bl, 1, k.theta_g, k.half_g) * F2 * uflip_ly(r + 1);
            A0.c += B1.b * slope_coef(bv, -1, k.theta);
            A1.c += B1.b * slope_coef(bv, 0, k.theta);
            A2.c += B1.b * slope_coef(bv, 1, k.theta);
            A0.a += lL * k.g * slope_coef(bl, -1, k.theta);
            A1.a += lL * k.g * slope_coef(bl, 0, k.theta);
            A2.a += lL * k.g * slope_coef(bl, 1, k.theta);
        }
        // (6) x direction of row j (uniform over the block)
        const bool out_row = j >= r0 && j < r1;
        if (out_row && (!EDGE || (j >= 2 && j < ny + 2))) {
            sb.e[t] = P0.e; sb.u[t] = P0.u; sb.v[t] = P0.v;
            __syncthreads();
            // x slopes of row j
            SlopeC sx{0.0f, 0.0f, 0.0f, 0u};
            if (t >= 1 && t < BW - 1 && (!EDGE || (i >= 1 && i <= nx + 2))) {
                const float ul = sb.u[t - 1], uc = P0.u, ur = sb.u[t + 1];
                const float vl = sb.v[t - 1], vc = P0.v, vr = sb.v[t + 1];
                const float el = sb.e[t - 1], ec = P0.e, er = sb.e[t + 1];
                sx.u = minmod_slope(ul, uc, ur, k.theta);
                sx.v = minmod_slope(vl, vc, vr, k.theta);
                const int bu = mm_branch((uc - ul) * k.theta, (ur - ul) * 0.5f, (ur - uc) * k.theta);
                const int bv = mm_branch((vc - vl) * k.theta, (vr - vl) * 0.5f, (vr - vc) * k.theta);
                const float fvl = (vl * flip(EDGE && ((wallW && i - 1 < 2) || (wallE && i - 1 > nx + 1)))) * F0;
                const float fvc = (vc * vflip_kx) * F0;
                const float fvr = (vr * flip(EDGE && ((wallW && i + 1 < 2) || (wallE && i + 1 > nx + 1)))) * F0;
                const float bw = k.theta_g * ((ec - el) - __fmul_rn(k.V, fvc + fvl));
                const float ce = k.half_g * ((er - el) - __fmul_rn(k.V, (fvr + __fmul_rn(2.0f, fvc)) + fvl));
                const float fw = k.theta_g * ((er - ec) - __fmul_rn(k.V, fvc + fvr));
                const float Kraw = minmod_raw(bw, ce, fw);
                const int bk = mm_branch(bw, ce, fw);
                const float dxfv = __fmul_rn(k.dx * F0, vc * vflip_adj);
                const float Hw = 0.5f * (C0.a + C1.a);
                const float He = 0.5f * (C0.b + C1.b);
                const float hw = (ec + Hw) - (Kraw + dxfv) / k.two_g;
                const float he = (ec + He) + (Kraw + dxfv) / k.two_g;
                float K = Kraw;
                int ba = kAdjNone;
                if (!(hw > 0.0f)) { K = -dxfv + __fmul_rn(k.two_g, ec + Hw); ba = kAdjA; }
                if (!(he > 0.0f)) { K = -dxfv - __fmul_rn(k.two_g, ec + He); ba = kAdjB; }
                sx.K = K;
                sx.code = (uint32_t)bu | ((uint32_t)bv << 2) | ((uint32_t)bk << 4) | ((uint32_t)ba << 6) | (1u << 16);
            }
            sb.su[t] = sx.u; sb.sv[t] = sx.v; sb.sK[t] = sx.K; sb.code[t] = sx.code;
            sb.l0[t] = LL0.a; sb.l1[t] = LL0.b; sb.l2[t] = LL0.c;
            __syncthreads();
            // x face (i, i+1)
            float aK = 0.0f, aux = 0.0f, avx = 0.0f;
            float pe = 0.0f, pu = 0.0f, pv = 0.0f, pK = 0.0f, pux = 0.0f, pvx = 0.0f;
            if (t >= 1 && t < BW - 2 && (!EDGE || (i >= 1 && i <= nx + 1)) && P0.e != kDryFlag &&
                sb.e[t + 1] != kDryFlag) {
                const int ip = i + 1;
                const float Rmu = P0.u + __fmul_rn(0.5f, sx.u), Rmv = P0.v + __fmul_rn(0.5f, sx.v);
                const float Rpu = sb.u[t + 1] - __fmul_rn(0.5f, sb.su[t + 1]);
                const float Rpv = sb.v[t + 1] - __fmul_rn(0.5f, sb.sv[t + 1]);
                const float fm = flip(EDGE && wallW && ip == 2), fp = flip(EDGE && wallE && ip == nx + 2);
                const float Hf = 0.5f * (C0.b + C1.b);
                const float Ep = (sb.e[t + 1] + Hf) - (sb.sK[t + 1] + __fmul_rn(k.dx * F0, sb.v[t + 1] * fp)) / k.two_g;
                const float Em = (P0.e + Hf) + (sx.K + __fmul_rn(k.dx * F0, P0.v * fm)) / k.two_g;
                const float hp = fmaxf(Ep, 0.0f), hm = fmaxf(Em, 0.0f);
                const float l0 = (sb.l0[t + 1] - LL0.a) / k.dx;
                const float l1 = (sb.l1[t + 1] - LL0.b) / k.dx;
                const float l2 = (sb.l2[t + 1] - LL0.c) / k.dx;
                const CuGrad g = cu_vjp(hm, Rmu, Rmv, hp, Rpu, Rpv, l0, l1, l2, k);
                if (Ep > 0.0f) {
                    pe = g.hp;
                    pK = -g.hp * inv2g;
                    pv = -g.hp * (k.dx * F0) * fp * inv2g;
                }
                if (Em > 0.0f) {
                    A0.a += g.hm;
                    aK += g.hm * inv2g;
                    A0.c += g.hm * (k.dx * F0) * fm * inv2g;
                }
                pu = g.up; pux = -0.5f * g.up;
                pv += g.vp; pvx = -0.5f * g.vp;
                A0.b += g.um; aux += 0.5f * g.um;
                A0.c += g.vm; avx += 0.5f * g.vm;
            }
            sb.pe[t] = pe; sb.pu[t] = pu; sb.pv[t] = pv; sb.pK[t] = pK; sb.pux[t] = pux; sb.pvx[t] = pvx;
            __syncthreads();
            if (t >= 1) {
                A0.a += sb.pe[t - 1]; A0.b += sb.pu[t - 1]; A0.c += sb.pv[t - 1];
                aK += sb.pK[t - 1]; aux += sb.pux[t - 1]; avx += sb.pvx[t - 1];
            }
            // x-slope adjoint of (j, i): adjustment
            float lKraw = aK;
            if (sx.code & (1u << 16)) {
                const int ba = (int)((sx.code >> 6) & 3u);
                if (ba != kAdjNone) {
                    A0.a += (ba == kAdjA ? k.two_g : -k.two_g) * aK;
                    A0.c -= aK * (k.dx * F0) * vflip_adj;
                    lKraw = 0.0f;
                }
            } else {
                lKraw = 0.0f; aux = 0.0f; avx = 0.0f;
            }
            sb.gu[t] = aux; sb.gv[t] = avx; sb.gK[t] = lKraw;
            __syncthreads();
            // gather the x-slope adjoints of cells i-1, i, i+1
            if (t >= 1 && t < BW - 1) {
                float lfv = 0.0f;
                for (int o = -1; o <= 1; ++o) {
                    const int pos = -o;
                    const uint32_t c = sb.code[t + o];
                    if (!(c & (1u << 16))) continue;
                    A0.b += sb.gu[t + o] * slope_coef((int)(c & 3u), pos, k.theta);
                    A0.c += sb.gv[t + o] * slope_coef((int)((c >> 2) & 3u), pos, k.theta);
                    const int bk = (int)((c >> 4) & 3u);
                    A0.a += sb.gK[t + o] * k.g * slope_coef(bk, pos, k.theta);
                    lfv -= sb.gK[t + o] * k.V * pot_coef(bk, pos, k.theta_g, k.half_g);
                }
                A0.c += lfv * F0 * vflip_kx;
            }
        }
        // (7) write the adjoint of row j
        if (out_row && writer) {
            const Trip3 lq = adj_prim_vjp<LAND>(P0.cls, P0.e, P0.u, P0.v, C0.a, C1.a, C0.b, C1.b, k, A0.a, A0.b, A0.c);
            float lE = lq.a, lU = lq.b, lV = lq.c;
            lE += qn0.a; lU += qn0.b; lV += qn0.c;       // stage 0: the adjoint of Q^n (zero otherwise)
            const size_t io = (size_t)j * a.pi + i;
            a.ie[io] = lE; a.iu[io] = lU; a.iv[io] = lV;
        }
        // (8) slide the window
        P0 = P1; P1 = P2; P2 = P3;
        C0 = C1; C1 = C2; C2 = C3; C3 = C4;
        F0 = F1; F1 = F2; F2 = F3;
        S1 = S2;
        LL0 = LL1; LL1 = LL2;
        A0 = A1; A1 = A2; A2 = trip0();
        B1 = B2; B2 = trip0();
    }
}

// A block needs no boundary logic when all its columns and the rows it
// touches (3 below the strip, 4 above) are interior cells.
template <int BW>
__device__ __forceinline__ bool march_interior(const AdjArgs& a, int bx, int by) {
    const int c0 = bx * (BW - 6) - 3, r0 = by * a.rows;
    const int r1 = min(r0 + a.rows, a.k.ny + 4);
    return c0 >= 3 && c0 + BW + 1 <= a.k.nx + 1 && r0 - 3 >= 2 && r1 + 4 <= a.k.ny + 1;
}

template <int BW, int FRIC, bool STAGE1, bool LAND>
__device__ __forceinline__ void adjoint_march_block(const AdjArgs& a, int bx, int by, MarchBufs<BW>& sb) {
    if (march_interior<BW>(a, bx, by))
        adjoint_march_strip<BW, FRIC, STAGE1, false, LAND>(a, bx, by, sb);
    else
        adjoint_march_strip<BW, FRIC, STAGE1, true, LAND>(a, bx, by, sb);
}

template <int BW, int FRIC, bool STAGE1, bool LAND>
__global__ void __launch_bounds__(BW, 512 / BW) cdklm_adjoint_march_kernel(const AdjArgs a) {
    __shared__ MarchBufs<BW> sb;
    pdl_enter();
    adjoint_march_block<BW, FRIC, STAGE1, LAND>(a, blockIdx.x, blockIdx.y, sb);
}

// Batched form: one block per (member, column block, row strip) tile; the
// member's arguments (2 per member: stage 0 and stage 1) in device memory.
template <int BW, int FRIC, bool STAGE1, bool LAND>
__global__ void __launch_bounds__(BW, 512 / BW) cdklm_adjoint_march_batch_kernel(
        const AdjArgs* __restrict__ args, const int4* __restrict__ tiles) {
    __shared__ MarchBufs<BW> sb;
    pdl_enter();
    const int4 tile = tiles[blockIdx.x];
    adjoint_march_block<BW, FRIC, STAGE1, LAND>(args[2 * tile.x + (STAGE1 ? 1 : 0)], tile.y, tile.z, sb);
}

// Moves the adjoint held at ghost cells to the interior cells whose values
// the ghosts carry: mirror (walls; hv flips at north/south walls, hu at
// east/west) or wrap (periodic).  One thread per interior cell within two
// cells of a side; corner ghosts are never read by the stage and carry none.
struct FoldMember {
    float *e, *u, *v;
    int p, nx, ny, bcN, bcE, bcS, bcW;
};

__device__ __forceinline__ void adj_fold_cell(float* e, float* u, float* v, int p, int nx, int ny, int bcN,
                                              int bcE, int bcS, int bcW, int t);

__global__ void k_adj_fold(float* e, float* u, float* v, int p, int nx, int ny, int bcN, int bcE, int bcS,
                           int bcW) {
    pdl_enter();
    adj_fold_cell(e, u, v, p, nx, ny, bcN, bcE, bcS, bcW, blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void k_adj_fold_batch(const FoldMember* __restrict__ members) {
    pdl_enter();
    const FoldMember M = members[blockIdx.y];
    adj_fold_cell(M.e, M.u, M.v, M.p, M.nx, M.ny, M.bcN, M.bcE, M.bcS, M.bcW, blockIdx.x * blockDim.x + threadIdx.x);
}

__device__ __forceinline__ void adj_fold_cell(float* e, float* u, float* v, int p, int nx, int ny, int bcN,
                                              int bcE, int bcS, int bcW, int t) {
    const int nrow = 4 * nx, ncol = 4 * (ny - 4 > 0 ? ny - 4 : 0);
    if (t >= nrow + ncol) return;
    int j, i;
    if (t < nrow) {
        const int r = t / nx;
        j = (r == 0) ? 2 : (r == 1) ? 3 : (r == 2) ? ny : ny + 1;
        i = 2 + t % nx;
    } else {
        const int s = t - nrow;
        const int cidx = s / (ny - 4);
        i = (cidx == 0) ? 2 : (cidx == 1) ? 3 : (cidx == 2) ? nx : nx + 1;
        j = 4 + s % (ny - 4);
    }
    const size_t o = (size_t)j * p + i;
    float ae = 0.0f, au = 0.0f, av = 0.0f;
    // source ghost row for this row, if any
    int gj = -1;
    float sv = 1.0f;
    if (j == 2) { gj = (bcS == kWall) ? 1 : ny + 2; sv = (bcS == kWall) ? -1.0f : 1.0f; }
    else if (j == 3) { gj = (bcS == kWall) ? 0 : ny + 3; sv = (bcS == kWall) ? -1.0f : 1.0f; }
    if (j == ny + 1) { gj = (bcN == kWall) ? ny + 2 : 1; sv = (bcN == kWall) ? -1.0f : 1.0f; }
    else if (j == ny) { gj = (bcN == kWall) ? ny + 3 : 0; sv = (bcN == kWall) ? -1.0f : 1.0f; }
    if (gj >= 0) {
        const size_t g = (size_t)gj * p + i;
        ae += e[g]; au += u[g]; av += sv * v[g];
    }
    int gi = -1;
    float su = 1.0f;
    if (i == 2) { gi = (bcW == kWall) ? 1 : nx + 2; su = (bcW == kWall) ? -1.0f : 1.0f; }
    else if (i == 3) { gi = (bcW == kWall) ? 0 : nx + 3; su = (bcW == kWall) ? -1.0f : 1.0f; }
    if (i == nx + 1) { gi = (bcE == kWall) ? nx + 2 : 1; su = (bcE == kWall) ? -1.0f : 1.0f; }
    else if (i == nx) { gi = (bcE == kWall) ? nx + 3 : 0; su = (bcE == kWall) ? -1.0f : 1.0f; }
    if (gi >= 0) {
        const size_t g = (size_t)j * p + gi;
        ae += e[g]; au += su * u[g]; av += v[g];
    }
    e[o] += ae; u[o] += au; v[o] += av;
}

template <int FRIC, bool STAGE1, int TX, int TY, int MINB, bool LAND>
cudaError_t launch_adj_tile(const AdjArgs& a, cudaStream_t s) {
    // the dynamic shared-memory limit is raised once per device
    static unsigned long long attr_set = 0ull;
    const int bytes = (int)sizeof(AdjSmem<TX, TY>);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 64 || !((attr_set >> dev) & 1ull)) {
        e = cudaFuncSetAttribute(cdklm_adjoint_stage_kernel<FRIC, STAGE1, TX, TY, MINB, LAND>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
        if (dev < 64) attr_set |= 1ull << dev;
    }
    const dim3 grid((a.k.nx + 4 + TX - 1) / TX, (a.k.ny + 4 + TY - 1) / TY);
    return launch_pdl(cdklm_adjoint_stage_kernel<FRIC, STAGE1, TX, TY, MINB, LAND>, grid, dim3(NT), (size_t)bytes, s, a);
}

// Tile form: 32-column tiles of a.rows rows (8, 12 or 16; CTAs per SM by
// shared memory: 5, 3 and 3 of 44.4, 59.6 and 74.7 KB).
template <int FRIC, bool STAGE1, bool LAND>
cudaError_t launch_adj(const AdjArgs& a, cudaStream_t s) {
    if (a.rows <= 8) return launch_adj_tile<FRIC, STAGE1, 32, 8, 4, LAND>(a, s);
    if (a.rows <= 12) return launch_adj_tile<FRIC, STAGE1, 32, 12, 3, LAND>(a, s);
    return launch_adj_tile<FRIC, STAGE1, 32, 16, 3, LAND>(a, s);
}

template <int BW, int FRIC, bool STAGE1, bool LAND>
cudaError_t launch_march(const AdjArgs& a, cudaStream_t s) {
    const dim3 grid((a.k.nx + 4 + BW - 7) / (BW - 6), (a.k.ny + 4 + a.rows - 1) / a.rows);
    return launch_pdl(cdklm_adjoint_march_kernel<BW, FRIC, STAGE1, LAND>, grid, dim3(BW), 0, s, a);
}

// Kernels without the land branches (corners read as they are, the cell
// depth a plain quarter sum) for domains whose bathymetry holds no land;
// dry and desingularised cells are handled either way.
template <int FRIC, bool STAGE1, bool LAND>
cudaError_t launch_form(const AdjArgs& a, int kind, cudaStream_t s) {
    if (kind == GO_ADJ_TILE) return launch_adj<FRIC, STAGE1, LAND>(a, s);
    if (kind == GO_ADJ_MARCH64) return launch_march<64, FRIC, STAGE1, LAND>(a, s);
    return launch_march<128, FRIC, STAGE1, LAND>(a, s);
}

template <int FRIC, bool STAGE1>
cudaError_t launch_any(const AdjArgs& a, int kind, cudaStream_t s) {
    return a.land ? launch_form<FRIC, STAGE1, true>(a, kind, s) : launch_form<FRIC, STAGE1, false>(a, kind, s);
}

// Launch form and strip (or tile) height for a grid.  A marching block walks
// its strip sequentially, so below ~300 k cells (512^2) the grid has too few
// column strips to fill 148 SMs and the tile form is faster (B200: 49.5 vs
// 58 us per stage at 512^2; 116 vs 170 at 1024^2 the other way).  Marching
// uses 64-thread blocks up to 1024 columns and 128 above, strips of the power
// of two in [8, 32] nearest below (column strips x rows) / 600.
void adjoint_launch(const go_domain* d, int* kind, int* rows) {
    int kd = d->adj_kind;
    const int nx = d->k.nx + 4, ny = d->k.ny + 4;
    // B200, us per stage adjoint with dependent launches, tiles of 8 / 16 rows
    // against the 64-column marching form: 512^2 37.5 / 43.4 / 58.0, 640^2
    // 52.5 / 50.0 / 67.0, 768^2 71.1 / 69.3 / 100.8, 1024^2 (16 rows) 115.0
    // against 114.4.  The tile form runs up to about 1000^2 cells, with 8-row
    // tiles (more, smaller CTAs: fewer partial waves) up to about 590^2.
    // Marching blocks of 64 columns up to 1024 interior columns (1024^2:
    // 114.4 us against 124 with 128-column blocks).
    if (kd == GO_ADJ_AUTO) {
        if ((long long)nx * ny < 1000000LL) kd = GO_ADJ_TILE;
        else kd = (d->k.nx <= 1024) ? GO_ADJ_MARCH64 : GO_ADJ_MARCH128;
    }
    int r = d->adj_rows;
    if (r <= 0 && kd == GO_ADJ_TILE) {
        r = ((long long)nx * ny < 350000LL) ? 8 : 16;
    } else if (r <= 0) {
        const int bw = (kd == GO_ADJ_MARCH64) ? 64 : 128;
        const long long target = (long long)((nx + bw - 7) / (bw - 6)) * ny / 600;
        r = 8;
        while (r < 32 && 2 * r <= target) r *= 2;
    }
    *kind = kd;
    *rows = r;
}

cudaError_t launch_fold(const go_domain* d, const go_state* l, cudaStream_t s) {
    const int nx = d->k.nx, ny = d->k.ny;
    const int n = 4 * nx + 4 * (ny - 4 > 0 ? ny - 4 : 0);
    return launch_pdl(k_adj_fold, dim3((n + 255) / 256), dim3(256), 0, s, l->eta, l->hu, l->hv, (int)(l->pitch / 4), nx,
                      ny, d->k.bcN, d->k.bcE, d->k.bcS, d->k.bcW);
}

int check_state(const go_state* s, int min_floats, const char* what) {
    if (!s || !s->eta || !s->hu || !s->hv) return go_fail(GO_ERR_INVALID, "%s: null state", what);
    return go_check_pitch(s->pitch, min_floats, what);
}

int adjoint_stage(go_domain* d, cudaStream_t s, int rk_step, float dt, const go_state* q_in,
                  const go_state* q_out, const go_state* lam_out, const go_state* lam_in,
                  const go_state* lam_qn, float* lam_wx, float* lam_wy, int wind_pitch, const float* Hi,
                  int Hi_pitch) {
    AdjArgs a;
    memset(&a, 0, sizeof(a));
    a.k = d->k;
    a.dt = dt;
    a.qe = q_in->eta; a.qu = q_in->hu; a.qv = q_in->hv; a.pq = q_in->pitch / 4;
    a.oe = q_out->eta; a.ou = q_out->hu; a.ov = q_out->hv; a.po = q_out->pitch / 4;
    a.le = lam_out->eta; a.lu = lam_out->hu; a.lv = lam_out->hv; a.pl = lam_out->pitch / 4;
    a.ie = lam_in->eta; a.iu = lam_in->hu; a.iv = lam_in->hv; a.pi = lam_in->pitch / 4;
    if (lam_qn) { a.ne = lam_qn->eta; a.nu = lam_qn->hu; a.nv = lam_qn->hv; a.pn = lam_qn->pitch / 4; }
    a.wx = lam_wx; a.wy = lam_wy; a.pw = wind_pitch / 4;
    a.Hi = Hi; a.phi = Hi_pitch / 4;
    a.f_rows = d->d_frows;
    a.status = d->d_status;
    a.land = d->has_land;
    int kind = GO_ADJ_AUTO;
    adjoint_launch(d, &kind, &a.rows);
    const int fric = go_friction_mode(d);
    cudaError_t e;
    if (rk_step == 0) {
        e = fric == kFricQuad ? launch_any<kFricQuad, false>(a, kind, s)
          : fric == kFricLinear ? launch_any<kFricLinear, false>(a, kind, s)
                                : launch_any<kFricNone, false>(a, kind, s);
    } else {
        e = fric == kFricQuad ? launch_any<kFricQuad, true>(a, kind, s)
          : fric == kFricLinear ? launch_any<kFricLinear, true>(a, kind, s)
                                : launch_any<kFricNone, true>(a, kind, s);
    }
    if (e == cudaSuccess) e = launch_fold(d, lam_in, s);
    if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "adjoint stage launch failed: %s", cudaGetErrorString(e));
    return GO_OK;
}

int check_adjoint_domain(const go_domain* d) {
    if (go_general_north(d))
        return go_fail(GO_ERR_UNSUPPORTED, "the adjoint is built for north-up grids (angle 0) only");
    return GO_OK;
}

__global__ void k_obs_misfit(const float* e, const float* u, const float* v, int p, int nx, int ny, int n,
                             const int* ij, const float* obs, float w_eta, float w_vel, double* J) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double acc = 0.0;
    const int oi = (t < n) ? ij[2 * t] : -1, oj = (t < n) ? ij[2 * t + 1] : -1;
    if (oi >= 0 && oi < nx && oj >= 0 && oj < ny) {      // cells outside the interior are skipped
        const size_t o = (size_t)(oj + 2) * p + (oi + 2);
        const double de = (double)e[o] - (double)obs[3 * t];
        const double du = (double)u[o] - (double)obs[3 * t + 1];
        const double dv = (double)v[o] - (double)obs[3 * t + 2];
        acc = (double)w_eta * de * de + (double)w_vel * (du * du + dv * dv);
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0 && acc != 0.0) atomicAdd(J, acc);
}

__global__ void k_obs_adjoint(const float* e, const float* u, const float* v, int p, float* le, float* lu,
                              float* lv, int pl, int nx, int ny, int n, const int* ij, const float* obs,
                              float w_eta, float w_vel) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = ij[2 * t] + 2, j = ij[2 * t + 1] + 2;
    if (i < 2 || i >= nx + 2 || j < 2 || j >= ny + 2) return;   // outside the interior
    const size_t o = (size_t)j * p + i, ol = (size_t)j * pl + i;
    atomicAdd(le + ol, 2.0f * w_eta * (e[o] - obs[3 * t]));
    atomicAdd(lu + ol, 2.0f * w_vel * (u[o] - obs[3 * t + 1]));
    atomicAdd(lv + ol, 2.0f * w_vel * (v[o] - obs[3 * t + 2]));
}

}  // namespace

struct go_adjoint_batch {
    int n = 0;
    std::vector<go_domain*> members;
    std::vector<AdjArgs> args;          // 2 per member: stage 0, stage 1
    std::vector<FoldMember> folds;      // n folds of scratch_star, then n of lam
    std::vector<char> member_set;
    AdjArgs* d_args = nullptr;
    FoldMember* d_folds = nullptr;
    int4* d_tiles = nullptr;
    int ntiles = 0;
    int bw = 128, rows = 32;
    int fric = 0;
    int land = 0;                       // some member's bathymetry may hold land
    int max_fold = 0;
    bool dirty = true;
};

namespace {

template <int BW, int FRIC, bool STAGE1>
cudaError_t launch_march_batch(const go_adjoint_batch* b, cudaStream_t s) {
    if (b->land)
        return launch_pdl(cdklm_adjoint_march_batch_kernel<BW, FRIC, STAGE1, true>, dim3(b->ntiles), dim3(BW), 0, s,
                          (const AdjArgs*)b->d_args, (const int4*)b->d_tiles);
    return launch_pdl(cdklm_adjoint_march_batch_kernel<BW, FRIC, STAGE1, false>, dim3(b->ntiles), dim3(BW), 0, s,
                      (const AdjArgs*)b->d_args, (const int4*)b->d_tiles);
}

template <bool STAGE1>
cudaError_t batch_stage(const go_adjoint_batch* b, cudaStream_t s) {
    if (b->bw == 64)
        return b->fric == kFricQuad ? launch_march_batch<64, kFricQuad, STAGE1>(b, s)
             : b->fric == kFricLinear ? launch_march_batch<64, kFricLinear, STAGE1>(b, s)
                                      : launch_march_batch<64, kFricNone, STAGE1>(b, s);
    return b->fric == kFricQuad ? launch_march_batch<128, kFricQuad, STAGE1>(b, s)
         : b->fric == kFricLinear ? launch_march_batch<128, kFricLinear, STAGE1>(b, s)
                                  : launch_march_batch<128, kFricNone, STAGE1>(b, s);
}

int adjoint_batch_commit(go_adjoint_batch* b) {
    if (!b->dirty) return GO_OK;
    for (int m = 0; m < b->n; ++m)
        if (!b->member_set[m]) return go_fail(GO_ERR_INVALID, "adjoint batch member %d has no buffers set", m);
    std::vector<int4> tiles;
    b->max_fold = 0;
    for (int m = 0; m < b->n; ++m) {
        const Scheme& k = b->members[m]->k;
        const int gx = (k.nx + 4 + b->bw - 7) / (b->bw - 6);
        const int gy = (k.ny + 4 + b->rows - 1) / b->rows;
        for (int y = 0; y < gy; ++y)
            for (int x = 0; x < gx; ++x) tiles.push_back(make_int4(m, x, y, 0));
        b->args[2 * m].rows = b->rows;
        b->args[2 * m + 1].rows = b->rows;
        b->max_fold = max(b->max_fold, 4 * k.nx + 4 * max(k.ny - 4, 0));
    }
    if (b->d_tiles && (int)tiles.size() > b->ntiles) {
        cudaFree(b->d_tiles);
        b->d_tiles = nullptr;
    }
    if (!b->d_tiles) GO_CUDA(cudaMalloc(&b->d_tiles, sizeof(int4) * tiles.size()));
    b->ntiles = (int)tiles.size();
    GO_CUDA(cudaMemcpy(b->d_tiles, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice));
    GO_CUDA(cudaMemcpy(b->d_args, b->args.data(), sizeof(AdjArgs) * b->args.size(), cudaMemcpyHostToDevice));
    GO_CUDA(cudaMemcpy(b->d_folds, b->folds.data(), sizeof(FoldMember) * b->folds.size(), cudaMemcpyHostToDevice));
    b->dirty = false;
    return GO_OK;
}

FoldMember fold_of(const go_domain* d, const go_state* st) {
    FoldMember f;
    f.e = st->eta; f.u = st->hu; f.v = st->hv;
    f.p = st->pitch / 4;
    f.nx = d->k.nx; f.ny = d->k.ny;
    f.bcN = d->k.bcN; f.bcE = d->k.bcE; f.bcS = d->k.bcS; f.bcW = d->k.bcW;
    return f;
}

}  // namespace

extern "C" {

int go_adjoint_batch_create(go_domain* const* members, int n, go_adjoint_batch** out) {
    if (!members || !out || n < 1) return go_fail(GO_ERR_INVALID, "bad arguments");
    *out = nullptr;
    go_adjoint_batch* b = new go_adjoint_batch();
    b->n = n;
    b->members.assign(members, members + n);
    for (int m = 0; m < n; ++m) {
        if (!members[m]) { delete b; return go_fail(GO_ERR_INVALID, "member %d is null", m); }
        int rc = check_adjoint_domain(members[m]);
        if (rc) { delete b; return rc; }
        if (go_friction_mode(members[m]) != go_friction_mode(members[0])) {
            delete b;
            return go_fail(GO_ERR_INVALID, "adjoint batch members must share the friction law");
        }
    }
    b->fric = go_friction_mode(members[0]);
    b->args.assign(2 * n, AdjArgs());
    b->folds.assign(2 * n, FoldMember());
    b->member_set.assign(n, 0);
    cudaError_t e = cudaMalloc(&b->d_args, sizeof(AdjArgs) * 2 * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_folds, sizeof(FoldMember) * 2 * n);
    if (e != cudaSuccess) {
        cudaFree(b->d_args);
        cudaFree(b->d_folds);
        delete b;
        return go_fail(GO_ERR_CUDA, "adjoint batch allocation failed: %s", cudaGetErrorString(e));
    }
    *out = b;
    return GO_OK;
}

int go_adjoint_batch_destroy(go_adjoint_batch* b) {
    if (!b) return GO_OK;
    cudaFree(b->d_args);
    cudaFree(b->d_folds);
    cudaFree(b->d_tiles);
    delete b;
    return GO_OK;
}

int go_adjoint_batch_set_launch(go_adjoint_batch* b, int block_columns, int rows_per_strip) {
    if (!b) return go_fail(GO_ERR_INVALID, "null batch");
    if (block_columns != 64 && block_columns != 128)
        return go_fail(GO_ERR_INVALID, "block_columns must be 64 or 128 (got %d)", block_columns);
    if (rows_per_strip < 0) return go_fail(GO_ERR_INVALID, "rows_per_strip must be >= 0");
    b->bw = block_columns;
    b->rows = rows_per_strip ? rows_per_strip : 32;
    b->dirty = true;
    return GO_OK;
}

int go_adjoint_batch_set_member(go_adjoint_batch* b, int m, float dt, const go_state* q_n, const go_state* q_star,
                                const go_state* q_next, const go_state* lam, const go_state* scratch_star,
                                const go_state* scratch_qn, float* lam_wx, float* lam_wy, int wind_pitch,
                                const float* Hi, int Hi_pitch) {
    if (!b || m < 0 || m >= b->n) return go_fail(GO_ERR_INVALID, "bad batch or member index %d", m);
    go_domain* d = b->members[m];
    const int w = d->k.nx + 4;
    int rc = check_state(q_n, w, "q_n");
    if (!rc) rc = check_state(q_star, w, "q_star");
    if (!rc) rc = check_state(q_next, w, "q_next");
    if (!rc) rc = check_state(lam, w, "lam");
    if (!rc) rc = check_state(scratch_star, w, "scratch_star");
    if (!rc) rc = check_state(scratch_qn, w, "scratch_qn");
    if (!rc) rc = go_check_pitch(Hi_pitch, d->k.nx + 5, "Hi");
    if (!rc && !Hi) rc = go_fail(GO_ERR_INVALID, "null Hi");
    if (!rc && (lam_wx || lam_wy)) {
        if (!lam_wx || !lam_wy) return go_fail(GO_ERR_INVALID, "wind adjoint needs both components");
        rc = go_check_pitch(wind_pitch, d->k.nx, "wind");
    }
    if (rc) return rc;
    if (scratch_star->eta == lam->eta || scratch_qn->eta == lam->eta || scratch_qn->eta == scratch_star->eta)
        return go_fail(GO_ERR_INVALID, "scratch buffers must not alias the adjoint state");
    auto fill = [&](AdjArgs& a, const go_state* qi, const go_state* qo, const go_state* lo, const go_state* li) {
        memset(&a, 0, sizeof(a));
        a.k = d->k;
        a.dt = dt;
        a.qe = qi->eta; a.qu = qi->hu; a.qv = qi->hv; a.pq = qi->pitch / 4;
        a.oe = qo->eta; a.ou = qo->hu; a.ov = qo->hv; a.po = qo->pitch / 4;
        a.le = lo->eta; a.lu = lo->hu; a.lv = lo->hv; a.pl = lo->pitch / 4;
        a.ie = li->eta; a.iu = li->hu; a.iv = li->hv; a.pi = li->pitch / 4;
        a.ne = scratch_qn->eta; a.nu = scratch_qn->hu; a.nv = scratch_qn->hv; a.pn = scratch_qn->pitch / 4;
        a.wx = lam_wx; a.wy = lam_wy; a.pw = wind_pitch / 4;
        a.Hi = Hi; a.phi = Hi_pitch / 4;
        a.f_rows = d->d_frows;
        a.status = d->d_status;
        a.rows = b->rows;
        a.land = d->has_land;
    };
    fill(b->args[2 * m], q_n, q_star, scratch_star, lam);           // stage 0: lam^n = S0^T lam* + lam_qn
    fill(b->args[2 * m + 1], q_star, q_next, lam, scratch_star);    // stage 1: lam* and lam_qn from lam^{n+1}
    b->folds[m] = fold_of(d, scratch_star);
    b->folds[b->n + m] = fold_of(d, lam);
    b->member_set[m] = 1;
    b->land = 0;
    for (int i = 0; i < b->n; ++i) b->land = b->land || b->members[i]->has_land;
    b->dirty = true;
    return GO_OK;
}

int go_adjoint_batch_step(go_adjoint_batch* b, void* stream) {
    GO_TRACE("go_adjoint_batch_step");
    if (!b) return go_fail(GO_ERR_INVALID, "null batch");
    int rc = adjoint_batch_commit(b);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 fg((b->max_fold + 255) / 256, b->n);
    cudaError_t e = batch_stage<true>(b, s);
    if (e == cudaSuccess) {
        e = launch_pdl(k_adj_fold_batch, fg, dim3(256), 0, s, (const FoldMember*)b->d_folds);
    }
    if (e == cudaSuccess) e = batch_stage<false>(b, s);
    if (e == cudaSuccess) {
        e = launch_pdl(k_adj_fold_batch, fg, dim3(256), 0, s, (const FoldMember*)(b->d_folds + b->n));
    }
    if (e != cudaSuccess) return go_fail(GO_ERR_CUDA, "adjoint batch launch failed: %s", cudaGetErrorString(e));
    return GO_OK;
}

int go_domain_set_adjoint_launch(go_domain* d, int kind, int rows_per_strip) {
    if (!d) return go_fail(GO_ERR_INVALID, "null domain");
    if (kind < GO_ADJ_AUTO || kind > GO_ADJ_MARCH128) return go_fail(GO_ERR_INVALID, "adjoint launch kind %d", kind);
    if (rows_per_strip < 0) return go_fail(GO_ERR_INVALID, "rows_per_strip must be >= 0");
    d->adj_kind = kind;
    d->adj_rows = rows_per_strip;
    return GO_OK;
}

int go_adjoint_stage(go_domain* d, void* stream, int rk_step, float dt, const go_state* q_in,
                     const go_state* q_out, const go_state* lam_out, const go_state* lam_in,
                     const go_state* lam_qn, float* lam_wx, float* lam_wy, int wind_pitch,
                     const float* Hi, int Hi_pitch) {
    GO_TRACE("go_adjoint_stage");
    if (!d || !Hi) return go_fail(GO_ERR_INVALID, "null argument");
    if (rk_step != 0 && rk_step != 1) return go_fail(GO_ERR_INVALID, "rk_step %d (RK2 has 0 and 1)", rk_step);
    int rc = check_adjoint_domain(d);
    const int w = d->k.nx + 4;
    if (!rc) rc = check_state(q_in, w, "q_in");
    if (!rc) rc = check_state(q_out, w, "q_out");
    if (!rc) rc = check_state(lam_out, w, "lam_out");
    if (!rc) rc = check_state(lam_in, w, "lam_in");
    if (!rc && (lam_qn || rk_step == 1)) rc = check_state(lam_qn, w, "lam_qn");
    if (!rc) rc = go_check_pitch(Hi_pitch, d->k.nx + 5, "Hi");
    if (!rc && (lam_wx || lam_wy)) {
        if (!lam_wx || !lam_wy) return go_fail(GO_ERR_INVALID, "wind adjoint needs both components");
        rc = go_check_pitch(wind_pitch, d->k.nx, "wind");
    }
    if (rc) return rc;
    if (lam_in->eta == lam_out->eta || lam_in->eta == q_in->eta)
        return go_fail(GO_ERR_INVALID, "lam_in must not alias lam_out or q_in");
    return adjoint_stage(d, (cudaStream_t)stream, rk_step, dt, q_in, q_out, lam_out, lam_in, lam_qn, lam_wx,
                         lam_wy, wind_pitch, Hi, Hi_pitch);
}

int go_adjoint_step(go_domain* d, void* stream, float dt, const go_state* q_n, const go_state* q_star,
                    const go_state* q_next, const go_state* lam_next, const go_state* lam_n,
                    const go_state* scratch_star, const go_state* scratch_qn, float* lam_wx, float* lam_wy,
                    int wind_pitch, const float* Hi, int Hi_pitch) {
    GO_TRACE("go_adjoint_step");
    if (!d || !Hi) return go_fail(GO_ERR_INVALID, "null argument");
    int rc = check_adjoint_domain(d);
    const int w = d->k.nx + 4;
    if (!rc) rc = check_state(q_n, w, "q_n");
    if (!rc) rc = check_state(q_star, w, "q_star");
    if (!rc) rc = check_state(q_next, w, "q_next");
    if (!rc) rc = check_state(lam_next, w, "lam_next");
    if (!rc) rc = check_state(lam_n, w, "lam_n");
    if (!rc) rc = check_state(scratch_star, w, "scratch_star");
    if (!rc) rc = check_state(scratch_qn, w, "scratch_qn");
    if (!rc) rc = go_check_pitch(Hi_pitch, d->k.nx + 5, "Hi");
    if (!rc && (lam_wx || lam_wy)) {
        if (!lam_wx || !lam_wy) return go_fail(GO_ERR_INVALID, "wind adjoint needs both components");
        rc = go_check_pitch(wind_pitch, d->k.nx, "wind");
    }
    if (rc) return rc;
    if (scratch_star->eta == lam_next->eta || scratch_star->eta == lam_n->eta ||
        scratch_qn->eta == lam_n->eta || scratch_qn->eta == scratch_star->eta)
        return go_fail(GO_ERR_INVALID, "scratch buffers must not alias the adjoint states");
    cudaStream_t s = (cudaStream_t)stream;
    rc = adjoint_stage(d, s, 1, dt, q_star, q_next, lam_next, scratch_star, scratch_qn, lam_wx, lam_wy,
                       wind_pitch, Hi, Hi_pitch);
    if (rc) return rc;
    return adjoint_stage(d, s, 0, dt, q_n, q_star, scratch_star, lam_n, scratch_qn, lam_wx, lam_wy, wind_pitch,
                         Hi, Hi_pitch);
}

int go_traj_step(go_domain* d, void* stream, float dt, float wind_stress_t, const go_state* q_n,
                 const go_state* q_star, const go_state* q_next, const float* Hi, int Hi_pitch,
                 float land_value) {
    GO_TRACE("go_traj_step");
    if (!d || !Hi) return go_fail(GO_ERR_INVALID, "null argument");
    const int w = d->k.nx + 4;
    int rc = check_state(q_n, w, "q_n");
    if (!rc) rc = check_state(q_star, w, "q_star");
    if (!rc) rc = check_state(q_next, w, "q_next");
    if (!rc) rc = go_check_pitch(Hi_pitch, d->k.nx + 5, "Hi");
    if (rc) return rc;
    if (q_next->eta == q_n->eta || q_star->eta == q_n->eta || q_star->eta == q_next->eta)
        return go_fail(GO_ERR_INVALID, "q_n, q_star and q_next must be distinct buffers");
    cudaStream_t s = (cudaStream_t)stream;
    const StageArgs a0 = go_stage_args(d, dt, 0, q_n->eta, q_n->hu, q_n->hv, q_n->pitch / 4, q_star->eta,
                                       q_star->hu, q_star->hv, q_star->pitch / 4, Hi, Hi_pitch / 4, land_value,
                                       wind_stress_t);
    StageArgs a1 = go_stage_args(d, dt, 1, q_star->eta, q_star->hu, q_star->hv, q_star->pitch / 4,
                                 q_next->eta, q_next->hu, q_next->hv, q_next->pitch / 4, Hi, Hi_pitch / 4,
                                 land_value, wind_stress_t);
    a1.qn_eta = q_n->eta; a1.qn_hu = q_n->hu; a1.qn_hv = q_n->hv; a1.pqn = q_n->pitch / 4;
    rc = go_launch_stage(d, s, a0);
    if (rc) return rc;
    return go_launch_stage(d, s, a1);
}

int go_obs_misfit(void* stream, const go_state* q, int nx, int ny, int n_obs, const int* obs_ij,
                  const float* obs_values, float w_eta, float w_vel, double* J_dev) {
    if (!q || !q->eta || !q->hu || !q->hv || (n_obs > 0 && (!obs_ij || !obs_values)) || !J_dev)
        return go_fail(GO_ERR_INVALID, "null argument");
    if (n_obs < 0) return go_fail(GO_ERR_INVALID, "n_obs < 0");
    int rc = go_check_pitch(q->pitch, nx + 4, "q");
    if (rc) return rc;
    if (n_obs == 0) return GO_OK;
    k_obs_misfit<<<(n_obs + 255) / 256, 256, 0, (cudaStream_t)stream>>>(q->eta, q->hu, q->hv, q->pitch / 4, nx, ny,
                                                                      n_obs, obs_ij, obs_values, w_eta, w_vel,
                                                                      J_dev);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

int go_obs_adjoint(void* stream, const go_state* q, const go_state* lam, int nx, int ny, int n_obs,
                   const int* obs_ij, const float* obs_values, float w_eta, float w_vel) {
    if (!q || !lam || !q->eta || !q->hu || !q->hv || !lam->eta || !lam->hu || !lam->hv ||
        (n_obs > 0 && (!obs_ij || !obs_values)))
        return go_fail(GO_ERR_INVALID, "null argument");
    if (n_obs < 0) return go_fail(GO_ERR_INVALID, "n_obs < 0");
    int rc = go_check_pitch(q->pitch, nx + 4, "q");
    if (!rc) rc = go_check_pitch(lam->pitch, nx + 4, "lam");
    if (rc) return rc;
    if (n_obs == 0) return GO_OK;
    k_obs_adjoint<<<(n_obs + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        q->eta, q->hu, q->hv, q->pitch / 4, lam->eta, lam->hu, lam->hv, lam->pitch / 4, nx, ny, n_obs, obs_ij,
        obs_values, w_eta, w_vel);
    GO_CUDA(cudaGetLastError());
    return GO_OK;
}

}  // extern "C"
