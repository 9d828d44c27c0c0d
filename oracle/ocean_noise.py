"""CPU restatement of the reference's stochastic model error (test oracle
only: tests and smoke() import it, the product never does).

Follows the reference's own CPU twins of OceanStateNoise
(gpu_ocean/SWESimulators/OceanStateNoise.py:572-937), vectorised with
NumPy in float64, with three corrections where the twins and the kernels
disagree; the oracle follows the kernels (ocean_noise.cu), since those are
what the reference runs:

* H at the cell centre is read at the ghost-inclusive cell, Hi[j+gy ...]
  (ocean_noise.cu:418-438); the twin reads H[j ...] (OceanStateNoise.py:
  686-689), the same only for the constant H of the reference's tests.
* The Coriolis parameter is f + beta ((i+0.5) dx north_x + (j+0.5) dy
  north_y) (ocean_noise.cu:471-476); the twin uses f + beta j dy.
* Land: the direct kernel zeroes eta, hu, hv in a cell with a land corner,
  the bicubic kernel leaves it unchanged (ocean_noise.cu:495-503, 758-770).

Pinned: tests/test_ocean_noise_host.py checks these functions against the
reference tests' known answers (OceanStateNoise_test.py, RandomNumbers_
test.py: sizes, statistics, coarse-versus-fine values, grid offsets) and
the GPU tests compare the reference's own kernels (oracle/_ref) with it.
"""

import numpy as np

CUTOFF = 2
LCG_A, LCG_C, LCG_M = 1103515245, 12345, 2147483647


def lcg(seed):
    """One ANSI C LCG draw per seed (OceanStateNoise.py:630-633,
    ocean_noise.cu:81-99): (new seed, seed / 2^31)."""
    s = (np.asarray(seed, dtype=np.uint64) * np.uint64(LCG_A) + np.uint64(LCG_C)) % np.uint64(LCG_M)
    return s, s / 2147483648.0


def fill_random(host_seed, rand_nx, normal=True):
    """Random numbers from the seeds (OceanStateNoise.py:646-680): two
    draws per seed, Box-Muller for normal numbers, written to columns 2i,
    2i+1 while 2i+1 < rand_nx, and column 2i alone when 2i == rand_nx (a
    condition no seed meets, so an odd width keeps its last column at 0).
    Returns (numbers, seeds)."""
    s, u1 = lcg(host_seed)
    s, u2 = lcg(s)
    if normal:
        r = np.sqrt(-2.0 * np.log(u1))
        n1, n2 = r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)
    else:
        n1, n2 = u1, u2
    seed_ny, seed_nx = s.shape
    out = np.zeros((seed_ny, rand_nx))
    for x in range(seed_nx):
        if 2 * x + 1 < rand_nx:
            out[:, 2 * x], out[:, 2 * x + 1] = n1[:, x], n2[:, x]
        elif 2 * x == rand_nx:
            out[:, 2 * x] = n1[:, x]
    return out, s


def soar_weight(ox, oy, cdx, cdy, q0, L):
    """SOAR covariance for the offset (ox, oy) cells (OceanStateNoise.py:
    682-690)."""
    dist = np.sqrt(float(cdx) ** 2 * ox * ox + float(cdy) ** 2 * oy * oy)
    return float(q0) * (1.0 + dist / float(L)) * np.exp(-dist / float(L))


def apply_q(random, coarse_nx, coarse_ny, cdx, cdy, q0, L, periodic_ns, periodic_ew, scale=1.0):
    """Q xi on all (coarse_ny + 4) x (coarse_nx + 4) coarse cells
    (OceanStateNoise.py:692-729): the random field with a 4-cell halo
    (wrapped when periodic), 5 x 5 taps."""
    random = np.asarray(random, dtype=np.float64)
    rny, rnx = random.shape
    nyh, nxh = coarse_ny + 8, coarse_nx + 8
    rows = (np.arange(nyh) - 4) % rny if periodic_ns else np.minimum(np.arange(nyh), rny - 1)
    cols = (np.arange(nxh) - 4) % rnx if periodic_ew else np.minimum(np.arange(nxh), rnx - 1)
    local = random[np.ix_(rows, cols)]
    out = np.zeros((coarse_ny + 4, coarse_nx + 4))
    for ky in range(2 * CUTOFF + 1):
        for kx in range(2 * CUTOFF + 1):
            w = soar_weight(CUTOFF - kx, CUTOFF - ky, cdx, cdy, q0, L)
            out += w * local[ky:ky + coarse_ny + 4, kx:kx + coarse_nx + 4]
    return scale * out


_B = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [-3, 3, -2, -1], [2, -2, 1, 1]], dtype=np.float64)


def interpolate(coarse, nx, ny, dx, dy, cdx, cdy, offset_i=0, offset_j=0, gx=2, gy=2):
    """Bicubic interpolation of the coarse buffer onto the model grid with a
    one-cell halo, (ny + 4) x (nx + 4) with zeros outside
    (OceanStateNoise.py:746-835, ocean_noise.cu:610-705): the coarse cell
    below-left of each cell centre, central differences for the
    derivatives, reads clamped to the coarse array."""
    coarse = np.asarray(coarse, dtype=np.float64)
    cny4, cnx4 = coarse.shape
    cnx, cny = cnx4 - 4, cny4 - 4
    out = np.zeros((ny + 4, nx + 4))
    for j in range(gy - 1, ny + gy + 1):
        for i in range(gx - 1, nx + gx + 1):
            x = (i - gx + 0.5 + offset_i) * dx
            y = (j - gy + 0.5 + offset_j) * dy
            ci = int(np.floor(x / cdx + gx - 0.5))
            cj = int(np.floor(y / cdy + gy - 0.5))
            if ci > cnx + 1:
                ci -= 1
            if cj > cny + 1:
                cj -= 1

            def c(di, dj):
                return coarse[min(max(cj + dj, 0), cny + 3), min(max(ci + di, 0), cnx + 3)]

            f = np.array([
                [c(0, 0), c(0, 1), (c(0, 1) - c(0, -1)) / 2, (c(0, 2) - c(0, 0)) / 2],
                [c(1, 0), c(1, 1), (c(1, 1) - c(1, -1)) / 2, (c(1, 2) - c(1, 0)) / 2],
                [(c(1, 0) - c(-1, 0)) / 2, (c(1, 1) - c(-1, 1)) / 2, 0.0, 0.0],
                [(c(2, 0) - c(0, 0)) / 2, (c(2, 1) - c(0, 1)) / 2, 0.0, 0.0]])
            fy_10 = (c(-1, 1) - c(-1, -1)) / 2
            fy_11 = (c(-1, 2) - c(-1, 0)) / 2
            fy20 = (c(2, 1) - c(2, -1)) / 2
            fy21 = (c(2, 2) - c(2, 0)) / 2
            f[2, 2] = (f[1, 2] - fy_10) / 2
            f[2, 3] = (f[1, 3] - fy_11) / 2
            f[3, 2] = (fy20 - f[0, 2]) / 2
            f[3, 3] = (fy21 - f[0, 3]) / 2
            a = _B @ f @ _B.T
            rx = (x - (ci - gx + 0.5) * cdx) / cdx
            ry = (y - (cj - gy + 0.5) * cdy) / cdy
            out[j, i] = np.array([1, rx, rx * rx, rx ** 3]) @ a @ np.array([1, ry, ry * ry, ry ** 3])
    return out


def geostrophic(d_eta, eta, hu, hv, Hi, nx, ny, dx, dy, g, f, beta=0.0, north=(0.0, 1.0), land=1e20,
                gx=2, gy=2, add_eta_to_depth=True, zero_land=True):
    """(eta, hu, hv) + the perturbation d_eta and its geostrophic balance in
    the interior cells (OceanStateNoise.py:747-773, ocean_noise.cu:440-508
    and 707-770).  The direct kernel counts eta in the depth and zeroes
    land cells; the bicubic one does neither."""
    eta, hu, hv = (np.array(a, dtype=np.float64) for a in (eta, hu, hv))
    Hi = np.asarray(Hi, dtype=np.float64)
    for j in range(gy, ny + gy):
        for i in range(gx, nx + gx):
            h4 = Hi[j:j + 2, i:i + 2]
            dry = bool(np.any(h4 == land))
            H_mid = 0.25 * h4.sum()
            cor = f + beta * ((i + 0.5) * dx * north[0] + (j + 0.5) * dy * north[1])
            d = d_eta[j, i]
            h_mid = d + H_mid + (eta[j, i] if add_eta_to_depth else 0.0)
            ex = (d_eta[j, i + 1] - d_eta[j, i - 1]) / (2 * dx)
            ey = (d_eta[j + 1, i] - d_eta[j - 1, i]) / (2 * dy)
            d_hu, d_hv = -(g / cor) * h_mid * ey, (g / cor) * h_mid * ex
            if dry:
                if zero_land:
                    eta[j, i] = hu[j, i] = hv[j, i] = 0.0
                continue
            eta[j, i] += d
            hu[j, i] += d_hu
            hv[j, i] += d_hv
    return eta, hu, hv


def perturb_ocean_state(random, eta, hu, hv, Hi, nx, ny, dx, dy, factor, q0, L, periodic_ns, periodic_ew, g, f,
                        beta=0.0, offset_i=0, offset_j=0, perturbation_scale=1.0, land=1e20):
    """The whole perturbation (OceanStateNoise.py:399-496): SOAR on the
    coarse grid, then the direct or bicubic balance.  Returns (coarse,
    eta, hu, hv)."""
    cnx, cny = nx // factor, ny // factor
    cdx, cdy = np.float32(dx * factor), np.float32(dy * factor)
    coarse = apply_q(random, cnx, cny, cdx, cdy, q0, L, periodic_ns, periodic_ew, perturbation_scale)
    if factor > 1:
        d_eta = interpolate(coarse, nx, ny, dx, dy, float(cdx), float(cdy), offset_i, offset_j)
        out = geostrophic(d_eta, eta, hu, hv, Hi, nx, ny, dx, dy, g, f, beta, land=land, add_eta_to_depth=False,
                          zero_land=False)
    else:
        out = geostrophic(coarse, eta, hu, hv, Hi, nx, ny, dx, dy, g, f, beta, land=land)
    return (coarse,) + tuple(out)
