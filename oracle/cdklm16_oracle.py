"""CPU oracle for the CDKLM16 time step (test infrastructure only).

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs
may import it.  The product path (``SWESimulators.CDKLM16`` over the CUDA
C-ABI) never calls into this file and fails loudly when its extension is
missing.

It is a NumPy restatement of gpu-ocean's CDKLM16 kernel, written over the
whole ghost-inclusive grid instead of per thread block.  It runs in float64
by default (the "FP64 transcription" every result's error is stated
against) and can run in float32 (each NumPy op rounded to float32, i.e. an
emulation of the reference's ``--fmad=false`` arithmetic with IEEE division
and no flush-to-zero).

Reference files followed (paths inside metno/gpu-ocean):

* ``gpu_ocean/SWESimulators/gpu_kernels/CDKLM16_kernel.cu:80-140``   flux
* ``.../CDKLM16_kernel.cu:148-241``  adjustSlopes_x / adjustSlopes_y
* ``.../CDKLM16_kernel.cu:246-370``  computeFFaceFlux / computeGFaceFlux
* ``.../CDKLM16_kernel.cu:373-424``  handleWallBC (wall mirroring)
* ``.../CDKLM16_kernel.cu:429-1006`` cdklm_swe_2D (one RK sub-step)
* ``.../common.cu:532-551``          minmodSlope / minmodRaw
* ``.../common.cu:616-650``          windStressX / windStressY
* ``.../common.cu:822-824``          desingularize
* ``.../max_dt.cu:42-141``           per-cell CFL limit (exact minimum
  here; the reference's shared-memory tree skips threads 256..383)
* ``.../initBm_kernel.cu:38-107``    Bm from Bi
* ``.../boundary_kernels.cu:35-110`` periodic ghost copy (NS, then EW)
* ``.../boundary_kernels.cu:121-246`` Bi ghost-corner fix
* ``gpu_ocean/SWESimulators/CDKLM16.py:494-598`` step() loop
* ``gpu_ocean/SWESimulators/CDKLM16.py:146-148, 237-238, 325-345`` setup
* ``gpu_ocean/SWESimulators/Common.py:1219-1239, 1436-1459`` BC helpers

Semantics that differ on purpose from the reference kernel:

* Wall mirroring is applied globally.  The reference mirrors inside each
  thread block, so when NY % block_height == 1 (or NX % block_width == 1)
  the block just before the wall reads an un-mirrored ghost row; the
  result then depends on the block size.  None of the tested sizes hits
  that case.
* The CFL limit is the exact minimum over all interior cells.
"""

import numpy as np

# Reference constants: CDKLM16_kernel.cu:38-39, max_dt.cu:30-35,
# Common.py:1333 (land value), CDKLM16.py:79-83 (defaults).
DRY_FLAG = 1.0e-30
DRY_EPS = 1.0e-3
LAND_VALUE = 1.0e20

WALL = 1
PERIODIC = 2


class Params:
    """Scheme parameters of one domain (the #defines of CDKLM16.py:179-191)."""

    def __init__(self, nx, ny, dx, dy, g, r=0.0, theta=1.3,
                 desing_eps=0.1, flux_slope_eps=0.1, depth_cutoff=1.0e-5,
                 bc=(WALL, WALL, WALL, WALL), north=(0.0, 1.0),
                 land_value=LAND_VALUE, linear_friction=False):
        self.nx, self.ny = int(nx), int(ny)
        self.dx, self.dy, self.g, self.r = float(dx), float(dy), float(g), float(r)
        self.theta = float(theta)
        self.desing_eps = float(desing_eps)
        self.flux_slope_eps = float(flux_slope_eps)
        self.depth_cutoff = float(depth_cutoff)
        # bc = (north, east, south, west), codes as Common.py:824-857
        self.bc = tuple(int(b) for b in bc)
        for b in self.bc:
            if b not in (WALL, PERIODIC):
                raise NotImplementedError("only wall (1) and periodic (2) boundaries")
        # north vector (sin(angle), cos(angle)) for a constant angle,
        # CDKLM16_kernel.cu:68-77
        self.north = (float(north[0]), float(north[1]))
        self.land_value = float(land_value)
        self.linear_friction = bool(linear_friction)


# ---------------------------------------------------------------------------
# Setup: bathymetry
# ---------------------------------------------------------------------------

def fix_bi_ghost_corners(Bi, nx, ny, bc):
    """Bi ghost corners, boundary_kernels.cu:121-246 as ordered by
    Common.py:1436-1459 (north-south first, then east-west)."""
    Bi = np.array(Bi, dtype=np.float32, copy=True)
    north, east, south, west = bc
    h = 2
    if north == PERIODIC and south == PERIODIC:
        # rows < 2 take row + ny; rows > ny+1 take row - ny
        for j in range(0, h):
            Bi[j, :] = Bi[j + ny, :]
        for j in range(ny + h, ny + 2 * h + 1):
            Bi[j, :] = Bi[j - ny, :]
    else:
        for j in range(h):
            Bi[j, :] = Bi[2 * h - j, :]
        for j in range(h):
            Bi[ny + 2 * h - j, :] = Bi[ny + j, :]
    if east == PERIODIC and west == PERIODIC:
        for i in range(0, h):
            Bi[:, i] = Bi[:, i + nx]
        for i in range(nx + h, nx + 2 * h + 1):
            Bi[:, i] = Bi[:, i - nx]
    else:
        for i in range(h):
            Bi[:, i] = Bi[:, 2 * h - i]
        for i in range(h):
            Bi[:, nx + 2 * h - i] = Bi[:, nx + i]
    return Bi


def init_bm(Bi, land_value=LAND_VALUE):
    """Bm = mean of the wet corners, land where all four are land
    (initBm_kernel.cu:38-107).  float32, computed in float32 exactly as the
    kernel orders the sum: ((a + b) + c) + d with a=(j,i), b=(j+1,i),
    c=(j,i+1), d=(j+1,i+1)."""
    B = np.array(Bi, dtype=np.float32, copy=True)
    B[np.abs(B - np.float32(land_value)) <= np.float32(DRY_EPS)] = np.float32(DRY_FLAG)
    a = B[:-1, :-1]
    b = B[1:, :-1]
    c = B[:-1, 1:]
    d = B[1:, 1:]
    flag = np.float32(DRY_FLAG)
    wet = (np.float32(4.0) - (a == flag).astype(np.float32) - (b == flag).astype(np.float32)
           - (c == flag).astype(np.float32) - (d == flag).astype(np.float32))
    s = ((a + b) + c) + d
    with np.errstate(divide="ignore", invalid="ignore"):
        Bm = np.where(wet == 0, np.float32(land_value), s / np.where(wet == 0, 1, wet))
    return Bm.astype(np.float32)


def coriolis_rows(f, beta, ny, dy, north=(0.0, 1.0)):
    """Per-row Coriolis table, float32, as uploaded to the texture.

    ``f`` is the constructor argument; the constructor compensates it by
    ``beta * 2 * dy`` (CDKLM16.py:146-148) and stores float32 (Simulator.py:87);
    the texture rows are ``f32(f) + beta * y`` with y = (j - 1.5) * dy in
    float64, rounded once to float32 (CDKLM16.py:320-345).  For beta == 0 the
    texture is the 1x1 value ``f32(f)``."""
    f_comp = np.float32(f - beta * (2 * dy * north[1]))
    if beta == 0.0:
        return np.full(ny + 4, f_comp, dtype=np.float32)
    y = np.linspace(-1.5 * dy, (ny + 1.5) * dy, ny + 4)
    n = y * north[1]
    return (f_comp + np.float32(beta) * n).astype(np.float32)


# ---------------------------------------------------------------------------
# Kernel helpers
# ---------------------------------------------------------------------------

def _sign1(x):
    return np.copysign(1.0, x).astype(x.dtype)


def minmod_raw(backward, central, forward):
    """common.cu:544-551"""
    sb = _sign1(backward)
    sc = _sign1(central)
    sf = _sign1(forward)
    m = np.minimum(np.minimum(np.abs(backward), np.abs(central)), np.abs(forward))
    return 0.25 * sb * (sb + sc) * (sc + sf) * m


def minmod_slope(left, center, right, theta):
    """common.cu:532-542"""
    backward = (center - left) * theta
    central = (right - left) * 0.5
    forward = (right - center) * theta
    return minmod_raw(backward, central, forward)


def desingularize(h, hu, eps):
    """common.cu:822-824.  ``0.5*eps`` is a double literal in the reference;
    the float32 path emulates that promotion."""
    if h.dtype == np.float32:
        a = (h * h / np.float32(2.0 * eps)).astype(np.float64) + 0.5 * eps
        a = a.astype(np.float32)
        den = np.maximum(np.minimum(a, np.float32(eps)), np.abs(h))
    else:
        den = np.maximum(np.minimum(h * h / (2.0 * eps) + 0.5 * eps, eps), np.abs(h))
    with np.errstate(divide="ignore", invalid="ignore"):
        return hu / den


def central_upwind_flux(hm, um, vm, hp, up_, vp, g, cutoff, slope_eps):
    """CDKLM16_flux (CDKLM16_kernel.cu:101-140) on arrays.  Inputs are the
    face states (h, u, v) from the minus (m) and plus (p) side."""
    dt = hm.dtype
    wetp = hp > cutoff
    wetm = hm > cutoff
    Fp0 = np.where(wetp, hp * up_, 0)
    Fp1 = np.where(wetp, hp * up_ * up_ + (0.5 * g) * hp * hp, 0)
    Fp2 = np.where(wetp, hp * up_ * vp, 0)
    Fm0 = np.where(wetm, hm * um, 0)
    Fm1 = np.where(wetm, hm * um * um + (0.5 * g) * hm * hm, 0)
    Fm2 = np.where(wetm, hm * um * vm, 0)
    with np.errstate(invalid="ignore"):
        cp = np.where(wetp, np.sqrt(np.where(wetp, g * hp, 0)), 0)
        cm = np.where(wetm, np.sqrt(np.where(wetm, g * hm, 0)), 0)
    upw = np.where(wetp, up_, 0)
    umw = np.where(wetm, um, 0)
    am = np.minimum(np.minimum(umw - cm, upw - cp), 0)
    ap = np.maximum(np.maximum(umw + cm, upw + cp), 0)
    zero = np.abs(ap - am) < slope_eps
    den = np.where(zero, 1, ap - am)
    F0 = ((ap * Fm0 - am * Fp0) + ap * am * (hp - hm)) / den
    F1 = ((ap * Fm1 - am * Fp1) + ap * am * (Fp0 - Fm0)) / den
    F2 = np.where(um + up_ > 0, Fm2, Fp2)
    F0 = np.where(zero, 0, F0).astype(dt)
    F1 = np.where(zero, 0, F1).astype(dt)
    F2 = np.where(zero, 0, F2).astype(dt)
    return F0, F1, F2


# ---------------------------------------------------------------------------
# Ghost cells
# ---------------------------------------------------------------------------

def apply_periodic_bc(eta, hu, hv, bc, nx, ny):
    """Periodic ghost copy, north-south first then east-west
    (boundary_kernels.cu:35-110, Common.py:1219-1239).  In place."""
    north, east, south, west = bc
    for a in (eta, hu, hv):
        if north == PERIODIC:
            a[0:2, :] = a[ny:ny + 2, :]
            a[ny + 2:ny + 4, :] = a[2:4, :]
        if east == PERIODIC:
            a[:, 0:2] = a[:, nx:nx + 2]
            a[:, nx + 2:nx + 4] = a[:, 2:4]


def _mirror_walls(eta, hu, hv, bc, nx, ny):
    """handleWallBC (CDKLM16_kernel.cu:373-424), applied to the interior
    rows/columns adjacent to each wall.  In place on working copies."""
    north, east, south, west = bc
    I = slice(2, nx + 2)
    J = slice(2, ny + 2)
    if north == WALL:
        for a, s in ((eta, 1), (hu, 1), (hv, -1)):
            a[ny + 2, I] = s * a[ny + 1, I]
            a[ny + 3, I] = s * a[ny, I]
    if south == WALL:
        for a, s in ((eta, 1), (hu, 1), (hv, -1)):
            a[1, I] = s * a[2, I]
            a[0, I] = s * a[3, I]
    if east == WALL:
        for a, s in ((eta, 1), (hu, -1), (hv, 1)):
            a[J, nx + 2] = s * a[J, nx + 1]
            a[J, nx + 3] = s * a[J, nx]
    if west == WALL:
        for a, s in ((eta, 1), (hu, -1), (hv, 1)):
            a[J, 1] = s * a[J, 2]
            a[J, 0] = s * a[J, 3]


# ---------------------------------------------------------------------------
# One RK sub-step
# ---------------------------------------------------------------------------

def rk_stage(p, Q_in, Q_n, Hi, Bm, f_rows, dt, rk_step, wind=(0.0, 0.0),
             dtype=np.float64, rk_order=2):
    """One call of ``cdklm_swe_2D`` (CDKLM16_kernel.cu:429-1006).

    Q_in  : (eta, hu, hv) input of this stage, each (ny+4, nx+4).  Ghost
            cells of periodic sides must already hold the wrapped values.
    Q_n   : (eta, hu, hv) of the output buffer (read at the own cell by
            stage 1, as the reference reads Q^n from its output buffer).
    Hi    : (ny+5, nx+5) corner bathymetry with fixed ghost corners.
    Bm    : (ny+4, nx+4) cell bathymetry from ``init_bm``.
    f_rows: (ny+4,) Coriolis per ghost-inclusive row.
    wind  : (X, Y) either scalars or (ny+4, nx+4) arrays of the wind at
            each cell's sample point, already interpolated in time.
    Returns (eta, hu, hv) new interior values, each (ny, nx).
    """
    T = dtype
    nx, ny = p.nx, p.ny
    g = T(p.g)
    DX, DY = T(p.dx), T(p.dy)
    theta = T(p.theta)
    cutoff = T(p.depth_cutoff)
    des_eps = p.desing_eps
    slope_eps = T(p.flux_slope_eps)
    two_g = T(2.0) * g
    north, east_bc, south, west = p.bc
    nX, nY = T(p.north[0]), T(p.north[1])
    eX, eY = nY, -nX  # east = (north.y, -north.x), CDKLM16_kernel.cu:681
    dt = T(dt)
    flag = T(DRY_FLAG)

    eta = np.array(Q_in[0], dtype=T, copy=True)
    hu = np.array(Q_in[1], dtype=T, copy=True)
    hv = np.array(Q_in[2], dtype=T, copy=True)
    _mirror_walls(eta, hu, hv, p.bc, nx, ny)

    Hi_f = np.array(Hi, dtype=np.float32, copy=True)
    Hi_f[np.abs(Hi_f - np.float32(p.land_value)) < np.float32(DRY_EPS)] = np.float32(DRY_FLAG)
    Hi_t = Hi_f.astype(T)
    Bm_t = np.asarray(Bm, dtype=np.float32).astype(T)
    f = np.asarray(f_rows, dtype=np.float32).astype(T)

    # --- cell state (eta, u, v), CDKLM16_kernel.cu:551-593 -------------------
    land = np.abs(np.asarray(Bm, np.float32) - np.float32(p.land_value)) <= np.float32(DRY_EPS)
    h = eta + Bm_t
    with np.errstate(divide="ignore", invalid="ignore"):
        u_wet = hu / h
        v_wet = hv / h
    shallow = h < T(des_eps)
    dry = h <= cutoff
    u_des = desingularize(h, hu, des_eps)
    v_des = desingularize(h, hv, des_eps)
    R0 = np.where(land, flag, np.where(shallow & dry, -Bm_t + cutoff, eta)).astype(T)
    R1 = np.where(land, 0, np.where(shallow, np.where(dry, 0, u_des), u_wet)).astype(T)
    R2 = np.where(land, 0, np.where(shallow, np.where(dry, 0, v_des), v_wet)).astype(T)

    J = slice(2, ny + 2)
    I = slice(2, nx + 2)

    # own-cell Hm from the four corners (CDKLM16_kernel.cu:547)
    Hm = T(0.25) * (((Hi_t[2:ny + 2, 2:nx + 2] + Hi_t[3:ny + 3, 2:nx + 2])
                     + Hi_t[2:ny + 2, 3:nx + 3]) + Hi_t[3:ny + 3, 3:nx + 3])
    h_own = R0[J, I] + Hm
    hu_own = np.where(h_own > cutoff, R1[J, I] * h_own, 0).astype(T)
    hv_own = np.where(h_own > cutoff, R2[J, I] * h_own, 0).astype(T)

    # --- x reconstruction on rows J, cells cols 1..nx+2 (:610-673) ----------
    cols = np.arange(nx + 4)
    vflip = np.where(((west == WALL) & (cols < 2)) | ((east_bc == WALL) & (cols > nx + 1)),
                     -1, 1).astype(T)
    C = slice(1, nx + 3)
    L = slice(0, nx + 2)
    Rr = slice(2, nx + 4)
    fJ = f[J][:, None]
    eta_c, eta_l, eta_r = R0[J, C], R0[J, L], R0[J, Rr]
    ux = minmod_slope(R1[J, L], R1[J, C], R1[J, Rr], theta)
    vx = minmod_slope(R2[J, L], R2[J, C], R2[J, Rr], theta)
    vfx = R2[J, :] * vflip[None, :]
    fv = (nX * R1[J, :] + nY * vfx) * fJ
    fv_l, fv_c, fv_r = fv[:, L], fv[:, C], fv[:, Rr]
    V = DX / two_g
    backward = (theta * g) * ((eta_c - eta_l) - V * (fv_c + fv_l))
    central = (T(0.5) * g) * ((eta_r - eta_l) - V * ((fv_r + T(2.0) * fv_c) + fv_l))
    forward = (theta * g) * ((eta_r - eta_c) - V * (fv_c + fv_r))
    Kx = minmod_raw(backward, central, forward).astype(T)
    # adjustSlopes_x (:148-191); east flip uses col > NX+2 as the reference
    vadj = R2[J, C] * np.where(((west == WALL) & (cols[C] < 2)) | ((east_bc == WALL) & (cols[C] > nx + 2)),
                               -1, 1).astype(T)[None, :]
    dxfv = (DX * fJ) * vadj
    H_w = T(0.5) * (Hi_t[2:ny + 2, 1:nx + 3] + Hi_t[3:ny + 3, 1:nx + 3])
    H_e = T(0.5) * (Hi_t[2:ny + 2, 2:nx + 4] + Hi_t[3:ny + 3, 2:nx + 4])
    h_w = (eta_c + H_w) - (Kx + dxfv) / two_g
    h_e = (eta_c + H_e) + (Kx + dxfv) / two_g
    Kx = np.where(h_w > 0, Kx, -dxfv + two_g * (eta_c + H_w)).astype(T)
    Kx = np.where(h_e > 0, Kx, -dxfv - two_g * (eta_c + H_e)).astype(T)

    # --- F fluxes at faces between cols c and c+1, c = 1..nx+1 (:246-304) --
    # arrays over slope-cells index s = col-1 (0..nx+1); face s <-> (s, s+1)
    m = slice(0, nx + 1)
    pp = slice(1, nx + 2)
    Rm_u = R1[J, 1:nx + 2] + T(0.5) * ux[:, m]
    Rm_v = R2[J, 1:nx + 2] + T(0.5) * vx[:, m]
    Rp_u = R1[J, 2:nx + 3] - T(0.5) * ux[:, pp]
    Rp_v = R2[J, 2:nx + 3] - T(0.5) * vx[:, pp]
    gp = cols[2:nx + 3]
    vm = R2[J, 1:nx + 2] * np.where((west == WALL) & (gp == 2), -1, 1).astype(T)[None, :]
    vp = R2[J, 2:nx + 3] * np.where((east_bc == WALL) & (gp == nx + 2), -1, 1).astype(T)[None, :]
    vp_n = R1[J, 2:nx + 3] * nX + vp * nY
    vm_n = R1[J, 1:nx + 2] * nX + vm * nY
    H_face = T(0.5) * (Hi_t[2:ny + 2, 2:nx + 3] + Hi_t[3:ny + 3, 2:nx + 3])
    hp = np.maximum(0, (R0[J, 2:nx + 3] + H_face) - (Kx[:, pp] + (DX * fJ) * vp_n) / two_g)
    hm = np.maximum(0, (R0[J, 1:nx + 2] + H_face) + (Kx[:, m] + (DX * fJ) * vm_n) / two_g)
    F0, F1, F2 = central_upwind_flux(hm.astype(T), Rm_u, Rm_v, hp.astype(T), Rp_u, Rp_v,
                                     g, cutoff, slope_eps)
    dryf = (R0[J, 2:nx + 3] == flag) | (R0[J, 1:nx + 2] == flag)
    F0 = np.where(dryf, 0, F0).astype(T)
    F1 = np.where(dryf, 0, F1).astype(T)
    F2 = np.where(dryf, 0, F2).astype(T)
    # flux difference for interior cells: east face index c-1 (c=2..nx+1)
    fdx0 = (F0[:, 1:nx + 1] - F0[:, 0:nx]) / DX
    fdx1 = (F1[:, 1:nx + 1] - F1[:, 0:nx]) / DX
    fdx2 = (F2[:, 1:nx + 1] - F2[:, 0:nx]) / DX

    fc = f[J][:, None]
    Kx_own = Kx[:, 1:nx + 1]
    eta_own = R0[J, I]
    tmp = (Kx_own + (DX * fc) * R2[J, I]) / two_g
    eta_west = eta_own - tmp
    eta_east = eta_own + tmp

    # --- y reconstruction on rows 1..ny+2, interior cols (:715-777) --------
    rows = np.arange(ny + 4)
    uflip = np.where(((south == WALL) & (rows < 2)) | ((north == WALL) & (rows > ny + 1)),
                     -1, 1).astype(T)
    Ry = slice(1, ny + 3)
    Lo = slice(0, ny + 2)
    Up = slice(2, ny + 4)
    uy = minmod_slope(R1[Lo, I], R1[Ry, I], R1[Up, I], theta)
    vy = minmod_slope(R2[Lo, I], R2[Ry, I], R2[Up, I], theta)
    ufy = R1[:, I] * uflip[:, None]
    fu = (eX * ufy + eY * R2[:, I]) * f[:, None]
    fu_lo, fu_c, fu_up = fu[Lo], fu[Ry], fu[Up]
    U = DY / two_g
    e_c, e_lo, e_up = R0[Ry, I], R0[Lo, I], R0[Up, I]
    backward = (theta * g) * ((e_c - e_lo) + U * (fu_c + fu_lo))
    central = (T(0.5) * g) * ((e_up - e_lo) + U * ((fu_up + T(2.0) * fu_c) + fu_lo))
    forward = (theta * g) * ((e_up - e_c) + U * (fu_c + fu_up))
    Ly = minmod_raw(backward, central, forward).astype(T)
    fR = f[Ry][:, None]
    uadj = R1[Ry, I] * np.where(((south == WALL) & (rows[Ry] < 2)) | ((north == WALL) & (rows[Ry] > ny + 2)),
                                -1, 1).astype(T)[:, None]
    dyfu = (DY * fR) * uadj
    H_s = T(0.5) * (Hi_t[1:ny + 3, 2:nx + 2] + Hi_t[1:ny + 3, 3:nx + 3])
    H_n = T(0.5) * (Hi_t[2:ny + 4, 2:nx + 2] + Hi_t[2:ny + 4, 3:nx + 3])
    h_s = (e_c + H_s) - (Ly - dyfu) / two_g
    h_n = (e_c + H_n) + (Ly - dyfu) / two_g
    Ly = np.where(h_s > 0, Ly, dyfu + two_g * (e_c + H_s)).astype(T)
    Ly = np.where(h_n > 0, Ly, dyfu - two_g * (e_c + H_n)).astype(T)

    # --- G fluxes at faces between rows r and r+1, r = 1..ny+1 (:309-370) ---
    m = slice(0, ny + 1)
    pp = slice(1, ny + 2)
    Rm_u = R1[1:ny + 2, I] + T(0.5) * uy[m]
    Rm_v = R2[1:ny + 2, I] + T(0.5) * vy[m]
    Rp_u = R1[2:ny + 3, I] - T(0.5) * uy[pp]
    Rp_v = R2[2:ny + 3, I] - T(0.5) * vy[pp]
    gpr = rows[2:ny + 3]
    um_ = R1[1:ny + 2, I] * np.where((south == WALL) & (gpr == 2), -1, 1).astype(T)[:, None]
    up_ = R1[2:ny + 3, I] * np.where((north == WALL) & (gpr == ny + 2), -1, 1).astype(T)[:, None]
    up_e = up_ * eX + R2[2:ny + 3, I] * eY
    um_e = um_ * eX + R2[1:ny + 2, I] * eY
    H_face = T(0.5) * (Hi_t[2:ny + 3, 2:nx + 2] + Hi_t[2:ny + 3, 3:nx + 3])
    fp = f[2:ny + 3][:, None]
    fm = f[1:ny + 2][:, None]
    hp = np.maximum(0, (R0[2:ny + 3, I] + H_face) - (Ly[pp] - (DY * fp) * up_e) / two_g)
    hm = np.maximum(0, (R0[1:ny + 2, I] + H_face) + (Ly[m] - (DY * fm) * um_e) / two_g)
    G0, G2, G1 = central_upwind_flux(hm.astype(T), Rm_v, Rm_u, hp.astype(T), Rp_v, Rp_u,
                                     g, cutoff, slope_eps)
    dryg = (R0[2:ny + 3, I] == flag) | (R0[1:ny + 2, I] == flag)
    G0 = np.where(dryg, 0, G0).astype(T)
    G1 = np.where(dryg, 0, G1).astype(T)
    G2 = np.where(dryg, 0, G2).astype(T)
    fd0 = fdx0 + (G0[1:ny + 1] - G0[0:ny]) / DY
    fd1 = fdx1 + (G1[1:ny + 1] - G1[0:ny]) / DY
    fd2 = fdx2 + (G2[1:ny + 1] - G2[0:ny]) / DY

    Ly_own = Ly[1:ny + 1]
    tmp = (Ly_own - (DY * fc) * R1[J, I]) / two_g
    eta_south = eta_own - tmp
    eta_north = eta_own + tmp

    # --- source terms (:817-867) --------------------------------------------
    X, Y = wind
    X = np.asarray(X, dtype=T)
    Y = np.asarray(Y, dtype=T)
    if X.ndim == 2:
        X = X[J, I]
        Y = Y[J, I]
    Hc = Hi_t
    RHxp = T(0.5) * (Hc[2:ny + 2, 3:nx + 3] + Hc[3:ny + 3, 3:nx + 3])
    RHxm = T(0.5) * (Hc[2:ny + 2, 2:nx + 2] + Hc[3:ny + 3, 2:nx + 2])
    RHyp = T(0.5) * (Hc[3:ny + 3, 2:nx + 2] + Hc[3:ny + 3, 3:nx + 3])
    RHym = T(0.5) * (Hc[2:ny + 2, 2:nx + 2] + Hc[2:ny + 2, 3:nx + 3])
    H_x = RHxp - RHxm
    H_y = RHyp - RHym
    eta_sn = T(0.5) * (eta_north + eta_south)
    eta_we = T(0.5) * (eta_west + eta_east)
    bath1 = (g * (eta_we + Hm)) * H_x
    bath2 = (g * (eta_sn + Hm)) * H_y
    hu_east = hu_own * eX + hv_own * eY
    hv_north = hu_own * nX + hv_own * nY
    hu_east_cor = fc * hv_north
    hv_north_cor = -fc * hu_east
    upX, upY = -nX, nY
    rX, rY = upY, -upX
    hu_cor = rX * hu_east_cor + rY * hv_north_cor
    hv_cor = upX * hu_east_cor + upY * hv_north_cor
    src = (h_own >= cutoff) & (eta_own != flag)
    st1 = np.where(src, (X + hu_cor) + bath1 / DX, 0).astype(T)
    st2 = np.where(src, (Y + hv_cor) + bath2 / DY, 0).astype(T)

    L1 = -fd0
    L2 = -fd1 + st1
    L3 = -fd2 + st2

    # --- friction and RK update (:870-1004) ---------------------------------
    r = T(p.r)
    if p.linear_friction:
        C = (T(2.0) * r * dt) / (eta_own + Hm)
    elif p.r > 0.0:
        with np.errstate(divide="ignore", invalid="ignore"):
            us = desingularize(h_own, hu_own, des_eps)
            vs = desingularize(h_own, hv_own, des_eps)
            Cs = (dt * r) * desingularize(h_own, np.sqrt(us * us + vs * vs).astype(T), des_eps)
            uw = hu_own / h_own
            vw = hv_own / h_own
            Cw = ((dt * r) * np.sqrt(uw * uw + vw * vw)) / h_own
        C = np.where(h_own < T(des_eps), Cs, Cw).astype(T)
    else:
        C = np.zeros_like(h_own)

    if rk_order == 2 or rk_order == 1:
        if rk_step == 0:
            new_eta = eta_own + dt * L1
            new_hu = (hu_own + dt * L2) / (T(1.0) + C)
            new_hv = (hv_own + dt * L3) / (T(1.0) + C)
        else:
            eta_a = np.asarray(Q_n[0], T)[J, I]
            hu_a = np.asarray(Q_n[1], T)[J, I]
            hv_a = np.asarray(Q_n[2], T)[J, I]
            new_eta = T(0.5) * (eta_a + (eta_own + dt * L1))
            new_hu = (T(0.5) * (hu_a + (hu_own + dt * L2))) / (T(1.0) + T(0.5) * C)
            new_hv = (T(0.5) * (hv_a + (hv_own + dt * L3))) / (T(1.0) + T(0.5) * C)
    else:
        raise NotImplementedError("rk_order 3 is not part of the oracle")

    dry_new = (new_eta + Hm) <= cutoff
    floor = -Hm + cutoff
    new_eta = np.where(dry_new, floor, new_eta)
    new_hu = np.where(dry_new, 0, new_hu)
    new_hv = np.where(dry_new, 0, new_hv)
    new_eta = np.maximum(floor, new_eta)
    return new_eta.astype(T), new_hu.astype(T), new_hv.astype(T)


# ---------------------------------------------------------------------------
# Time stepping (CDKLM16.step, CDKLM16.py:494-598)
# ---------------------------------------------------------------------------

class OracleSim:
    """Host-side restatement of ``CDKLM16`` for the RK2 path: two state
    buffers (h0 = Q^n, h1 = Q*), periodic ghost refresh after each stage."""

    def __init__(self, eta0, hu0, hv0, Hi, nx, ny, dx, dy, dt, g, f, r,
                 coriolis_beta=0.0, theta=1.3, bc=(1, 1, 1, 1),
                 wind=(0.0, 0.0), dtype=np.float64, linear_friction=False):
        self.p = Params(nx, ny, dx, dy, g, r, theta=theta, bc=bc,
                        linear_friction=linear_friction)
        self.dtype = dtype
        self.Hi = fix_bi_ghost_corners(Hi, nx, ny, self.p.bc)
        self.Bm = init_bm(self.Hi)
        eta0 = np.maximum(np.asarray(eta0, np.float32), -self.Bm)   # CDKLM16.py:237-238
        self.h0 = [np.array(a, dtype=np.float32).astype(dtype) for a in (eta0, hu0, hv0)]
        self.h1 = [a.copy() for a in self.h0]
        self.f_rows = coriolis_rows(f, coriolis_beta, ny, dy)
        self.dt = dt
        self.wind = wind
        self.t = 0.0
        self.num_iterations = 0

    def _bc(self, Q):
        apply_periodic_bc(Q[0], Q[1], Q[2], self.p.bc, self.p.nx, self.p.ny)

    def _stage(self, Qin, Qout, dt, k):
        J = slice(2, self.p.ny + 2)
        I = slice(2, self.p.nx + 2)
        e, u, v = rk_stage(self.p, Qin, Qout, self.Hi, self.Bm, self.f_rows, dt, k,
                           wind=self.wind, dtype=self.dtype)
        Qout[0][J, I] = e
        Qout[1][J, I] = u
        Qout[2][J, I] = v

    def rk2_step(self, local_dt):
        self._stage(self.h0, self.h1, local_dt, 0)
        self._bc(self.h1)
        self._stage(self.h1, self.h0, local_dt, 1)
        self._bc(self.h0)

    def step(self, t_end):
        if self.t == 0:
            self._bc(self.h0)
        t_now = 0.0
        while t_now < t_end:
            local_dt = np.float32(min(self.dt, np.float32(t_end - t_now)))
            self.rk2_step(float(local_dt))
            self.t += np.float64(local_dt)
            t_now += np.float64(local_dt)
            self.num_iterations += 1
        return self.t

    def download(self):
        return tuple(a.copy() for a in self.h0)


def max_dt(eta, hu, hv, Bm, nx, ny, dx, dy, g, land_value=LAND_VALUE, dtype=np.float64):
    """Exact CFL limit over interior cells: min of 0.25*dx/|u +- c| and
    0.25*dy/|v +- c|, c = sqrt(g h), skipping dry and land cells
    (max_dt.cu:72-99; the minimum here is exact)."""
    T = dtype
    J = slice(2, ny + 2)
    I = slice(2, nx + 2)
    H = np.asarray(Bm, np.float32)[J, I]
    e = np.asarray(eta, T)[J, I]
    h = e + H.astype(T)
    skip = (h <= 0) | (np.abs(H - np.float32(land_value)) < np.float32(DRY_EPS))
    with np.errstate(divide="ignore", invalid="ignore"):
        u = np.asarray(hu, T)[J, I] / h
        v = np.asarray(hv, T)[J, I] / h
        c = np.sqrt(T(g) * h)
        d = np.minimum(np.minimum(T(0.25) * T(dx) / np.abs(u + c), T(0.25) * T(dx) / np.abs(u - c)),
                       np.minimum(T(0.25) * T(dy) / np.abs(v + c), T(0.25) * T(dy) / np.abs(v - c)))
    d = np.where(skip, np.inf, d)
    return float(np.min(d))
