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
# Array namespace: the same restatement runs on NumPy arrays (CPU) or on
# torch tensors (float64 on a GPU, and under autograd for the adjoint
# checks).  Only elementwise operations and slicing are used.
# ---------------------------------------------------------------------------

class _NP:
    name = "numpy"

    @staticmethod
    def where(c, a, b):
        return np.where(c, a, b)

    minimum = staticmethod(np.minimum)
    maximum = staticmethod(np.maximum)
    abs = staticmethod(np.abs)
    sqrt = staticmethod(np.sqrt)

    @staticmethod
    def sign1(x):
        return np.copysign(1.0, x).astype(x.dtype)

    @staticmethod
    def cast(a, dtype):
        return np.asarray(a).astype(dtype)

    @staticmethod
    def errstate():
        return np.errstate(divide="ignore", invalid="ignore", over="ignore")


class _Torch:
    name = "torch"

    def __init__(self, device):
        import torch
        self.t = torch
        self.device = device

    def where(self, c, a, b):
        t = self.t
        if not t.is_tensor(c):
            c = t.as_tensor(c, device=self.device)
        return t.where(c, a, b)

    def minimum(self, a, b):
        t = self.t
        if not t.is_tensor(b):
            return t.clamp(a, max=float(b))
        if not t.is_tensor(a):
            return t.clamp(b, max=float(a))
        return t.minimum(a, b)

    def maximum(self, a, b):
        t = self.t
        if not t.is_tensor(b):
            return t.clamp(a, min=float(b))
        if not t.is_tensor(a):
            return t.clamp(b, min=float(a))
        return t.maximum(a, b)

    def abs(self, a):
        return self.t.abs(a)

    def sqrt(self, a):
        return self.t.sqrt(a)

    def sign1(self, x):
        return self.t.copysign(self.t.ones_like(x), x)

    def cast(self, a, dtype):
        t = self.t
        tdt = {np.float64: t.float64, np.float32: t.float32}[dtype]
        if t.is_tensor(a):
            return a.to(device=self.device, dtype=tdt)
        return t.as_tensor(np.asarray(a), device=self.device, dtype=tdt)

    def errstate(self):
        import contextlib
        return contextlib.nullcontext()


def namespace_for(a):
    """_NP for NumPy arrays, a torch namespace for tensors."""
    if isinstance(a, np.ndarray):
        return _NP
    return _Torch(a.device)


# ---------------------------------------------------------------------------
# Kernel helpers
# ---------------------------------------------------------------------------

# ---------------------------------------------------------------------------
# Branch recording (for finite-difference checks of the adjoint: a direction
# is only usable when no branch of the scheme changes along it)
# ---------------------------------------------------------------------------

_REC = None


class record_branches:
    """Context manager: every branch decision of rk_stage inside it is
    appended (as a boolean or small-integer array) to ``self.masks``."""

    def __enter__(self):
        global _REC
        self.masks = []
        self._prev = _REC
        _REC = self.masks
        return self

    def __exit__(self, *exc):
        global _REC
        _REC = self._prev
        return False


def _rec(*arrays):
    if _REC is not None:
        for a in arrays:
            _REC.append(a.detach().clone() if hasattr(a, "detach") else np.array(a, copy=True))


def minmod_raw(xp, backward, central, forward):
    """common.cu:544-551"""
    sb = xp.sign1(backward)
    sc = xp.sign1(central)
    sf = xp.sign1(forward)
    m = xp.minimum(xp.minimum(xp.abs(backward), xp.abs(central)), xp.abs(forward))
    if _REC is not None:
        ab, ac, af = xp.abs(backward), xp.abs(central), xp.abs(forward)
        same = (sb == sc) & (sc == sf)
        _rec(same, same & (ab <= ac) & (ab <= af), same & (ac <= af))
    return 0.25 * sb * (sb + sc) * (sc + sf) * m


def minmod_slope(xp, left, center, right, theta):
    """common.cu:532-542"""
    backward = (center - left) * theta
    central = (right - left) * 0.5
    forward = (right - center) * theta
    return minmod_raw(xp, backward, central, forward)


def desingularize(xp, h, hu, eps, f32=False):
    """common.cu:822-824.  ``0.5*eps`` is a double literal in the reference;
    the float32 path emulates that promotion."""
    if f32:
        a = (h * h / np.float32(2.0 * eps)).astype(np.float64) + 0.5 * eps
        a = a.astype(np.float32)
        den = np.maximum(np.minimum(a, np.float32(eps)), np.abs(h))
    else:
        den = xp.maximum(xp.minimum(h * h / (2.0 * eps) + 0.5 * eps, eps), xp.abs(h))
    return hu / den


def central_upwind_flux(xp, hm, um, vm, hp, up_, vp, g, cutoff, slope_eps):
    """CDKLM16_flux (CDKLM16_kernel.cu:101-140) on arrays.  Inputs are the
    face states (h, u, v) from the minus (m) and plus (p) side."""
    wetp = hp > cutoff
    wetm = hm > cutoff
    Fp0 = xp.where(wetp, hp * up_, 0.0)
    Fp1 = xp.where(wetp, hp * up_ * up_ + (0.5 * g) * hp * hp, 0.0)
    Fp2 = xp.where(wetp, hp * up_ * vp, 0.0)
    Fm0 = xp.where(wetm, hm * um, 0.0)
    Fm1 = xp.where(wetm, hm * um * um + (0.5 * g) * hm * hm, 0.0)
    Fm2 = xp.where(wetm, hm * um * vm, 0.0)
    cp = xp.where(wetp, xp.sqrt(xp.where(wetp, g * hp, 1.0)), 0.0)
    cm = xp.where(wetm, xp.sqrt(xp.where(wetm, g * hm, 1.0)), 0.0)
    upw = xp.where(wetp, up_, 0.0)
    umw = xp.where(wetm, um, 0.0)
    am = xp.minimum(xp.minimum(umw - cm, upw - cp), 0.0)
    ap = xp.maximum(xp.maximum(umw + cm, upw + cp), 0.0)
    zero = xp.abs(ap - am) < slope_eps
    _rec(wetp, wetm, (umw - cm) <= (upw - cp), am < 0.0, (umw + cm) >= (upw + cp), ap > 0.0, zero,
         (um + up_) > 0)
    den = xp.where(zero, 1.0, ap - am)
    F0 = ((ap * Fm0 - am * Fp0) + ap * am * (hp - hm)) / den
    F1 = ((ap * Fm1 - am * Fp1) + ap * am * (Fp0 - Fm0)) / den
    F2 = xp.where(um + up_ > 0, Fm2, Fp2)
    return xp.where(zero, 0.0, F0), xp.where(zero, 0.0, F1), xp.where(zero, 0.0, F2)


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


def periodic_wrap(xp, a, bc, nx, ny):
    """Out-of-place version of apply_periodic_bc for one array (keeps
    autograd graphs intact)."""
    north, east, south, west = bc
    if north == PERIODIC:
        a = _cat0(xp, [a[ny:ny + 2], a[2:ny + 2], a[2:4]])
    if east == PERIODIC:
        a = _cat1(xp, [a[:, nx:nx + 2], a[:, 2:nx + 2], a[:, 2:4]])
    return a


def _cat0(xp, parts):
    if xp is _NP:
        return np.concatenate(parts, axis=0)
    return xp.t.cat(parts, dim=0)


def _cat1(xp, parts):
    if xp is _NP:
        return np.concatenate(parts, axis=1)
    return xp.t.cat(parts, dim=1)


def _mirror_walls(xp, eta, hu, hv, bc, nx, ny):
    """handleWallBC (CDKLM16_kernel.cu:373-424): the two ghost rows/columns
    next to a wall take the interior values, normal momentum negated.
    Out of place: returns new arrays."""
    north, east, south, west = bc
    out = []
    for a, sns, sew in ((eta, 1.0, 1.0), (hu, 1.0, -1.0), (hv, -1.0, 1.0)):
        if north == WALL or south == WALL:
            top = [a[ny + 1:ny + 2] * sns, a[ny:ny + 1] * sns] if north == WALL else [a[ny + 2:ny + 4]]
            bot = [a[3:4] * sns, a[2:3] * sns] if south == WALL else [a[0:2]]
            a = _cat0(xp, bot + [a[2:ny + 2]] + top)
        if east == WALL or west == WALL:
            right = [a[:, nx + 1:nx + 2] * sew, a[:, nx:nx + 1] * sew] if east == WALL else [a[:, nx + 2:nx + 4]]
            left = [a[:, 3:4] * sew, a[:, 2:3] * sew] if west == WALL else [a[:, 0:2]]
            a = _cat1(xp, left + [a[:, 2:nx + 2]] + right)
        out.append(a)
    return out


# ---------------------------------------------------------------------------
# Static per-domain arrays (bathymetry-derived, Coriolis, wall flips)
# ---------------------------------------------------------------------------

class Static:
    """Everything in a stage that depends only on Hi, Bm, f and the
    boundary codes, prepared once in float32 on the host (as the kernel
    reads it) and held in the working dtype/array library."""

    def __init__(self, p, Hi, Bm, f_rows, dtype=np.float64, like=None):
        nx, ny = p.nx, p.ny
        north, east, south, west = p.bc
        xp = _NP if like is None else namespace_for(like)
        self.xp = xp
        self.dtype = dtype
        T = lambda a: xp.cast(a, dtype)  # noqa: E731
        Hf = np.array(Hi, dtype=np.float32, copy=True)
        Hf[np.abs(Hf - np.float32(p.land_value)) < np.float32(DRY_EPS)] = np.float32(DRY_FLAG)
        H = Hf.astype(np.float64) if dtype == np.float64 else Hf
        Bm32 = np.asarray(Bm, np.float32)
        self.land = xp.cast(np.abs(Bm32 - np.float32(p.land_value)) <= np.float32(DRY_EPS), np.float32) > 0.5
        self.Bm = T(Bm32)
        self.f = T(np.asarray(f_rows, np.float32))
        # own-cell Hm (CDKLM16_kernel.cu:547)
        c = np.float32(0.25) if dtype == np.float32 else 0.25
        Hm = c * (((H[2:ny + 2, 2:nx + 2] + H[3:ny + 3, 2:nx + 2]) + H[2:ny + 2, 3:nx + 3]) + H[3:ny + 3, 3:nx + 3])
        self.Hm = T(Hm)
        half = np.float32(0.5) if dtype == np.float32 else 0.5
        # x-face depths for rows J: face west of column c = 0.5(H[r,c] + H[r+1,c])
        Hx = half * (H[2:ny + 2, :] + H[3:ny + 3, :])          # (ny, nx+5)
        self.H_w = T(Hx[:, 1:nx + 3])      # adjust_x, cells 1..nx+2
        self.H_e = T(Hx[:, 2:nx + 4])
        self.Hface_x = T(Hx[:, 2:nx + 3])  # faces with p-col 2..nx+2
        self.RHxm = T(Hx[:, 2:nx + 2])
        self.RHxp = T(Hx[:, 3:nx + 3])
        # y-face depths for columns I: face south of row r = 0.5(H[r,c] + H[r,c+1])
        Hy = half * (H[:, 2:nx + 2] + H[:, 3:nx + 3])          # (ny+5, nx)
        self.H_s = T(Hy[1:ny + 3])         # adjust_y, cells rows 1..ny+2
        self.H_n = T(Hy[2:ny + 4])
        self.Hface_y = T(Hy[2:ny + 3])     # faces with p-row 2..ny+2
        self.RHym = T(Hy[2:ny + 2])
        self.RHyp = T(Hy[3:ny + 3])
        cols = np.arange(nx + 4)
        rows = np.arange(ny + 4)
        fl = lambda m: T(np.where(m, -1.0, 1.0))  # noqa: E731
        self.vflip_kx = fl(((west == WALL) & (cols < 2)) | ((east == WALL) & (cols > nx + 1)))[None, :]
        self.vflip_adj = fl(((west == WALL) & (cols[1:nx + 3] < 2)) | ((east == WALL) & (cols[1:nx + 3] > nx + 2)))[None, :]
        gp = cols[2:nx + 3]
        self.flip_vm = fl((west == WALL) & (gp == 2))[None, :]
        self.flip_vp = fl((east == WALL) & (gp == nx + 2))[None, :]
        self.uflip_ly = fl(((south == WALL) & (rows < 2)) | ((north == WALL) & (rows > ny + 1)))[:, None]
        self.uflip_adj = fl(((south == WALL) & (rows[1:ny + 3] < 2)) | ((north == WALL) & (rows[1:ny + 3] > ny + 2)))[:, None]
        gpr = rows[2:ny + 3]
        self.flip_um = fl((south == WALL) & (gpr == 2))[:, None]
        self.flip_up = fl((north == WALL) & (gpr == ny + 2))[:, None]


# ---------------------------------------------------------------------------
# One RK sub-step
# ---------------------------------------------------------------------------

def rk_stage(p, Q_in, Q_n, S, dt, rk_step, wind=(0.0, 0.0)):
    """One call of ``cdklm_swe_2D`` (CDKLM16_kernel.cu:429-1006).

    Q_in  : (eta, hu, hv) input of this stage, each (ny+4, nx+4).  Ghost
            cells of periodic sides must already hold the wrapped values.
    Q_n   : (eta, hu, hv) of the output buffer (read at the own cell by
            stage 1, as the reference reads Q^n from its output buffer);
            interior-only (ny, nx) arrays are accepted too.
    S     : ``Static`` of the domain (bathymetry, Coriolis, flips).
    wind  : (X, Y) scalars or (ny, nx) arrays of the wind at each interior
            cell, already interpolated in time.
    Returns (eta, hu, hv) new interior values, each (ny, nx).
    """
    xp = S.xp
    f32 = S.dtype == np.float32
    T = (lambda x: np.float32(x)) if f32 else float
    nx, ny = p.nx, p.ny
    g = T(p.g)
    DX, DY = T(p.dx), T(p.dy)
    theta = T(p.theta)
    cutoff = T(p.depth_cutoff)
    des_eps = p.desing_eps
    slope_eps = T(p.flux_slope_eps)
    two_g = T(2.0) * g
    theta_g = theta * g
    half_g = T(0.5) * g
    nX, nY = T(p.north[0]), T(p.north[1])
    eX, eY = nY, -nX  # east = (north.y, -north.x), CDKLM16_kernel.cu:681
    dt = T(dt)
    flag = T(DRY_FLAG)
    J = slice(2, ny + 2)
    I = slice(2, nx + 2)

    eta, hu, hv = _mirror_walls(xp, Q_in[0], Q_in[1], Q_in[2], p.bc, nx, ny)

    with xp.errstate():
        # --- cell state (eta, u, v), CDKLM16_kernel.cu:551-593 ---------------
        Bm = S.Bm
        land = S.land
        h = eta + Bm
        shallow = h < T(des_eps)
        dry = h <= cutoff
        _rec(shallow, dry)
        h_safe = xp.where(shallow, 1.0, h)
        u_des = desingularize(xp, h, hu, des_eps, f32)
        v_des = desingularize(xp, h, hv, des_eps, f32)
        R0 = xp.where(land, flag, xp.where(shallow & dry, -Bm + cutoff, eta))
        R1 = xp.where(land, 0.0, xp.where(shallow, xp.where(dry, 0.0, u_des), hu / h_safe))
        R2 = xp.where(land, 0.0, xp.where(shallow, xp.where(dry, 0.0, v_des), hv / h_safe))

        Hm = S.Hm
        h_own = R0[J, I] + Hm
        hu_own = xp.where(h_own > cutoff, R1[J, I] * h_own, 0.0)
        hv_own = xp.where(h_own > cutoff, R2[J, I] * h_own, 0.0)

        # --- x reconstruction on rows J, cells cols 1..nx+2 (:610-673) ------
        C = slice(1, nx + 3)
        L = slice(0, nx + 2)
        Rr = slice(2, nx + 4)
        fJ = S.f[J][:, None]
        eta_c, eta_l, eta_r = R0[J, C], R0[J, L], R0[J, Rr]
        ux = minmod_slope(xp, R1[J, L], R1[J, C], R1[J, Rr], theta)
        vx = minmod_slope(xp, R2[J, L], R2[J, C], R2[J, Rr], theta)
        vfx = R2[J, :] * S.vflip_kx
        fv = (nX * R1[J, :] + nY * vfx) * fJ
        fv_l, fv_c, fv_r = fv[:, L], fv[:, C], fv[:, Rr]
        V = DX / two_g
        backward = theta_g * ((eta_c - eta_l) - V * (fv_c + fv_l))
        central = half_g * ((eta_r - eta_l) - V * ((fv_r + T(2.0) * fv_c) + fv_l))
        forward = theta_g * ((eta_r - eta_c) - V * (fv_c + fv_r))
        Kx = minmod_raw(xp, backward, central, forward)
        # adjustSlopes_x (:148-191); east flip uses col > NX+2 as the reference
        vadj = R2[J, C] * S.vflip_adj
        dxfv = (DX * fJ) * vadj
        h_w = (eta_c + S.H_w) - (Kx + dxfv) / two_g
        h_e = (eta_c + S.H_e) + (Kx + dxfv) / two_g
        _rec(h_w > 0, h_e > 0)
        Kx = xp.where(h_w > 0, Kx, -dxfv + two_g * (eta_c + S.H_w))
        Kx = xp.where(h_e > 0, Kx, -dxfv - two_g * (eta_c + S.H_e))

        # --- F fluxes at faces between cols c and c+1, c = 1..nx+1 (:246-304)
        m = slice(0, nx + 1)
        pp = slice(1, nx + 2)
        Rm_u = R1[J, 1:nx + 2] + T(0.5) * ux[:, m]
        Rm_v = R2[J, 1:nx + 2] + T(0.5) * vx[:, m]
        Rp_u = R1[J, 2:nx + 3] - T(0.5) * ux[:, pp]
        Rp_v = R2[J, 2:nx + 3] - T(0.5) * vx[:, pp]
        vm = R2[J, 1:nx + 2] * S.flip_vm
        vp = R2[J, 2:nx + 3] * S.flip_vp
        vp_n = R1[J, 2:nx + 3] * nX + vp * nY
        vm_n = R1[J, 1:nx + 2] * nX + vm * nY
        Hfx = S.Hface_x
        hp = xp.maximum((R0[J, 2:nx + 3] + Hfx) - (Kx[:, pp] + (DX * fJ) * vp_n) / two_g, 0.0)
        hm = xp.maximum((R0[J, 1:nx + 2] + Hfx) + (Kx[:, m] + (DX * fJ) * vm_n) / two_g, 0.0)
        _rec(hp > 0, hm > 0)
        F0, F1, F2 = central_upwind_flux(xp, hm, Rm_u, Rm_v, hp, Rp_u, Rp_v, g, cutoff, slope_eps)
        dryf = (R0[J, 2:nx + 3] == flag) | (R0[J, 1:nx + 2] == flag)
        F0 = xp.where(dryf, 0.0, F0)
        F1 = xp.where(dryf, 0.0, F1)
        F2 = xp.where(dryf, 0.0, F2)
        fdx0 = (F0[:, 1:nx + 1] - F0[:, 0:nx]) / DX
        fdx1 = (F1[:, 1:nx + 1] - F1[:, 0:nx]) / DX
        fdx2 = (F2[:, 1:nx + 1] - F2[:, 0:nx]) / DX

        fc = S.f[J][:, None]
        Kx_own = Kx[:, 1:nx + 1]
        eta_own = R0[J, I]
        tmp = (Kx_own + (DX * fc) * R2[J, I]) / two_g
        eta_west = eta_own - tmp
        eta_east = eta_own + tmp

        # --- y reconstruction on rows 1..ny+2, interior cols (:715-777) -----
        Ry = slice(1, ny + 3)
        Lo = slice(0, ny + 2)
        Up = slice(2, ny + 4)
        uy = minmod_slope(xp, R1[Lo, I], R1[Ry, I], R1[Up, I], theta)
        vy = minmod_slope(xp, R2[Lo, I], R2[Ry, I], R2[Up, I], theta)
        ufy = R1[:, I] * S.uflip_ly
        fu = (eX * ufy + eY * R2[:, I]) * S.f[:, None]
        fu_lo, fu_c, fu_up = fu[Lo], fu[Ry], fu[Up]
        U = DY / two_g
        e_c, e_lo, e_up = R0[Ry, I], R0[Lo, I], R0[Up, I]
        backward = theta_g * ((e_c - e_lo) + U * (fu_c + fu_lo))
        central = half_g * ((e_up - e_lo) + U * ((fu_up + T(2.0) * fu_c) + fu_lo))
        forward = theta_g * ((e_up - e_c) + U * (fu_c + fu_up))
        Ly = minmod_raw(xp, backward, central, forward)
        fR = S.f[Ry][:, None]
        uadj = R1[Ry, I] * S.uflip_adj
        dyfu = (DY * fR) * uadj
        h_s = (e_c + S.H_s) - (Ly - dyfu) / two_g
        h_n = (e_c + S.H_n) + (Ly - dyfu) / two_g
        _rec(h_s > 0, h_n > 0)
        Ly = xp.where(h_s > 0, Ly, dyfu + two_g * (e_c + S.H_s))
        Ly = xp.where(h_n > 0, Ly, dyfu - two_g * (e_c + S.H_n))

        # --- G fluxes at faces between rows r and r+1, r = 1..ny+1 (:309-370)
        m = slice(0, ny + 1)
        pp = slice(1, ny + 2)
        Rm_u = R1[1:ny + 2, I] + T(0.5) * uy[m]
        Rm_v = R2[1:ny + 2, I] + T(0.5) * vy[m]
        Rp_u = R1[2:ny + 3, I] - T(0.5) * uy[pp]
        Rp_v = R2[2:ny + 3, I] - T(0.5) * vy[pp]
        um_ = R1[1:ny + 2, I] * S.flip_um
        up_ = R1[2:ny + 3, I] * S.flip_up
        up_e = up_ * eX + R2[2:ny + 3, I] * eY
        um_e = um_ * eX + R2[1:ny + 2, I] * eY
        Hfy = S.Hface_y
        fp = S.f[2:ny + 3][:, None]
        fm = S.f[1:ny + 2][:, None]
        hp = xp.maximum((R0[2:ny + 3, I] + Hfy) - (Ly[pp] - (DY * fp) * up_e) / two_g, 0.0)
        hm = xp.maximum((R0[1:ny + 2, I] + Hfy) + (Ly[m] - (DY * fm) * um_e) / two_g, 0.0)
        _rec(hp > 0, hm > 0)
        G0, G2, G1 = central_upwind_flux(xp, hm, Rm_v, Rm_u, hp, Rp_v, Rp_u, g, cutoff, slope_eps)
        dryg = (R0[2:ny + 3, I] == flag) | (R0[1:ny + 2, I] == flag)
        G0 = xp.where(dryg, 0.0, G0)
        G1 = xp.where(dryg, 0.0, G1)
        G2 = xp.where(dryg, 0.0, G2)
        fd0 = fdx0 + (G0[1:ny + 1] - G0[0:ny]) / DY
        fd1 = fdx1 + (G1[1:ny + 1] - G1[0:ny]) / DY
        fd2 = fdx2 + (G2[1:ny + 1] - G2[0:ny]) / DY

        Ly_own = Ly[1:ny + 1]
        tmp = (Ly_own - (DY * fc) * R1[J, I]) / two_g
        eta_south = eta_own - tmp
        eta_north = eta_own + tmp

        # --- source terms (:817-867) -----------------------------------------
        X, Y = wind
        H_x = S.RHxp - S.RHxm
        H_y = S.RHyp - S.RHym
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
        st1 = xp.where(src, (X + hu_cor) + bath1 / DX, 0.0)
        st2 = xp.where(src, (Y + hv_cor) + bath2 / DY, 0.0)

        L1 = -fd0
        L2 = -fd1 + st1
        L3 = -fd2 + st2

        # --- friction and RK update (:870-1004) ------------------------------
        r = T(p.r)
        if p.linear_friction:
            Cf = (T(2.0) * r * dt) / (eta_own + Hm)
        elif p.r > 0.0:
            hs = xp.where(h_own < T(des_eps), h_own, 1.0)
            us = desingularize(xp, hs, hu_own, des_eps, f32)
            vs = desingularize(xp, hs, hv_own, des_eps, f32)
            Cs = (dt * r) * desingularize(xp, hs, xp.sqrt(us * us + vs * vs + 1e-300), des_eps, f32)
            hw = xp.where(h_own < T(des_eps), 1.0, h_own)
            uw = hu_own / hw
            vw = hv_own / hw
            Cw = ((dt * r) * xp.sqrt(uw * uw + vw * vw + 1e-300)) / hw
            Cf = xp.where(h_own < T(des_eps), Cs, Cw)
        else:
            Cf = 0.0 * h_own

        if rk_step == 0:
            new_eta = eta_own + dt * L1
            new_hu = (hu_own + dt * L2) / (T(1.0) + Cf)
            new_hv = (hv_own + dt * L3) / (T(1.0) + Cf)
        else:
            qa = [a[J, I] if a.shape[0] == ny + 4 else a for a in Q_n]
            new_eta = T(0.5) * (qa[0] + (eta_own + dt * L1))
            new_hu = (T(0.5) * (qa[1] + (hu_own + dt * L2))) / (T(1.0) + T(0.5) * Cf)
            new_hv = (T(0.5) * (qa[2] + (hv_own + dt * L3))) / (T(1.0) + T(0.5) * Cf)

        dry_new = (new_eta + Hm) <= cutoff
        _rec(dry_new)
        floor = -Hm + cutoff
        new_eta = xp.where(dry_new, floor, new_eta)
        new_hu = xp.where(dry_new, 0.0, new_hu)
        new_hv = xp.where(dry_new, 0.0, new_hv)
        new_eta = xp.maximum(floor, new_eta)
    return new_eta, new_hu, new_hv


# ---------------------------------------------------------------------------
# Time stepping (CDKLM16.step, CDKLM16.py:494-598)
# ---------------------------------------------------------------------------

class OracleSim:
    """Host-side restatement of ``CDKLM16`` for the RK2 path: two state
    buffers (h0 = Q^n, h1 = Q*), periodic ghost refresh after each stage.
    ``device=None`` runs on NumPy arrays; a torch device runs the same code
    on torch tensors of ``dtype``."""

    def __init__(self, eta0, hu0, hv0, Hi, nx, ny, dx, dy, dt, g, f, r,
                 coriolis_beta=0.0, theta=1.3, bc=(1, 1, 1, 1),
                 wind=(0.0, 0.0), dtype=np.float64, linear_friction=False, device=None,
                 f_rows=None):
        self.p = Params(nx, ny, dx, dy, g, r, theta=theta, bc=bc,
                        linear_friction=linear_friction)
        self.dtype = dtype
        self.Hi = fix_bi_ghost_corners(Hi, nx, ny, self.p.bc)
        self.Bm = init_bm(self.Hi)
        eta0 = np.maximum(np.asarray(eta0, np.float32), -self.Bm)   # CDKLM16.py:237-238
        host = [np.array(a, dtype=np.float32).astype(dtype) for a in (eta0, hu0, hv0)]
        if device is None:
            self.h0 = host
        else:
            import torch
            tdt = {np.float64: torch.float64, np.float32: torch.float32}[dtype]
            self.h0 = [torch.as_tensor(a, dtype=tdt, device=device) for a in host]
        self.h1 = [a.copy() if isinstance(a, np.ndarray) else a.clone() for a in self.h0]
        self.f_rows = coriolis_rows(f, coriolis_beta, ny, dy) if f_rows is None else np.asarray(f_rows, np.float32)
        self.S = Static(self.p, self.Hi, self.Bm, self.f_rows, dtype, like=None if device is None else self.h0[0])
        T = np.float32 if dtype == np.float32 else float
        if np.ndim(wind[0]) == 0:
            self.wind = (T(wind[0]), T(wind[1]))
        else:
            self.wind = (self.S.xp.cast(np.asarray(wind[0], np.float32), dtype),
                         self.S.xp.cast(np.asarray(wind[1], np.float32), dtype))
        self.dt = dt
        self.t = 0.0
        self.num_iterations = 0

    def _bc(self, Q):
        apply_periodic_bc(Q[0], Q[1], Q[2], self.p.bc, self.p.nx, self.p.ny)

    def _stage(self, Qin, Qout, dt, k):
        J = slice(2, self.p.ny + 2)
        I = slice(2, self.p.nx + 2)
        e, u, v = rk_stage(self.p, Qin, Qout, self.S, dt, k, wind=self.wind)
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
        return tuple(a.copy() if isinstance(a, np.ndarray) else a.detach().cpu().numpy() for a in self.h0)


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
