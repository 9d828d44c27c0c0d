"""Model-error host logic and the CPU oracle (no GPU).

* Buffer sizes and the reference's launch grids for the cases of the
  reference's tests (gpu_ocean/tests/stochastic/OceanStateNoise_test.py:
  33-112, OceanStateNoise_parent.py:40-70): 30 x 40 cells, periodic or not.
* The LCG and Box-Muller oracle against the statistics the reference's
  RandomNumbers tests demand of its CPU generator (RandomNumbers_test.py).
* SOAR, bicubic interpolation and geostrophic balance of the oracle against
  properties with exact answers: a unit impulse gives the SOAR weights, the
  interpolation reproduces quadratics and the coarse values at coarse cell
  centres (OceanStateNoise_test.py:231-245), the grid offsets of the
  reference's alignment test (:253-310).
"""

import numpy as np
import pytest

from oracle import ocean_noise as on
from SWESimulators.Common import BoundaryConditions
from SWESimulators.OceanStateNoise import coarse_grid_offset, noise_layout


@pytest.mark.parametrize("pns, pew, rand, seed, soar_grid, rand_grid", [
    (True, True, (30, 40), (15, 40), (3, 3), (1, 3)),
    (False, False, (38, 48), (19, 48), (3, 3), (2, 3)),
    (True, False, (38, 40), (19, 40), (3, 3), (2, 3)),
    (False, True, (30, 48), (15, 48), (3, 3), (1, 3)),
])
def test_layout_matches_reference_tests(pns, pew, rand, seed, soar_grid, rand_grid):
    n, s = (2, 2) if pns else (1, 1)
    e, w = (2, 2) if pew else (1, 1)
    L = noise_layout(30, 40, 7.0, BoundaryConditions(n, e, s, w))
    assert (L["rand_nx"], L["rand_ny"]) == rand
    assert (L["seed_nx"], L["seed_ny"]) == seed
    assert L["global_size_SOAR"] == soar_grid
    assert L["global_size_random_numbers"] == rand_grid


def test_layout_rejects_even_or_misaligned_factor():
    with pytest.raises(AssertionError):
        noise_layout(30, 40, 7.0, BoundaryConditions(2, 2, 2, 2), interpolation_factor=2)
    with pytest.raises(AssertionError):
        noise_layout(31, 40, 7.0, BoundaryConditions(2, 2, 2, 2), interpolation_factor=3)
    L = noise_layout(150, 200, 7.0, BoundaryConditions(2, 2, 2, 2), interpolation_factor=5)
    assert (L["coarse_nx"], L["coarse_ny"]) == (30, 40)


def test_grid_offsets_of_alignment_test():
    # OceanStateNoise_test.py:309-310: cells 6, 7, 8 with factor 5 -> 1, 0, -1
    assert [coarse_grid_offset(5, a, a) for a in (6, 7, 8)] == [(1, 1), (0, 0), (-1, -1)]
    assert coarse_grid_offset(5, None, None) == (0, 0)


def _seeds(ny, nx, seed=3):
    return (np.random.RandomState(seed).rand(ny, nx) * 2147483648.0).astype(np.uint64)


def test_lcg_known_values():
    s, u = on.lcg(np.array([1], dtype=np.uint64))
    assert int(s[0]) == (1103515245 + 12345) % 2147483647 and u[0] == int(s[0]) / 2 ** 31
    s2, _ = on.lcg(s)
    assert int(s2[0]) == (int(s[0]) * 1103515245 + 12345) % 2147483647


def test_uniform_and_normal_statistics():
    # RandomNumbers_test.py: 400 x 400 large_noise, CPU generators
    seeds = _seeds(400, 200)
    U, s1 = on.fill_random(seeds, 400, normal=False)
    assert abs(U.mean() - 0.5) < 0.005 and abs(U.var() - 1 / 12) < 0.001
    N, s2 = on.fill_random(seeds, 400, normal=True)
    assert abs(N.mean()) < 0.01 and abs(N.var() - 1.0) < 0.01
    assert np.array_equal(s1, s2) and not np.array_equal(s1, seeds)


def test_odd_width_leaves_last_column():
    # The reference writes a lone first draw only when 2 i == random_nx
    # (ocean_noise.cu:150-156, OceanStateNoise.py:676-680), which no thread
    # meets: with an odd width the last column is never written.
    seeds = _seeds(3, 4)
    out7, _ = on.fill_random(seeds, 7, normal=False)
    out8, _ = on.fill_random(seeds, 8, normal=False)
    assert np.array_equal(out7[:, :6], out8[:, :6]) and not out7[:, 6].any()


def test_soar_of_impulse_is_the_covariance():
    cnx = cny = 12
    xi = np.zeros((cny, cnx))
    xi[5, 6] = 1.0
    q = on.apply_q(xi, cnx, cny, 7.0, 7.0, 1e-4, 5.25, True, True)
    # coarse cell (a_y, a_x) holds Q(a - b) for the impulse at b = (5, 6)
    # shifted by the two ghost cells
    for oy in range(-2, 3):
        for ox in range(-2, 3):
            assert q[5 + 2 + oy, 6 + 2 + ox] == pytest.approx(on.soar_weight(ox, oy, 7.0, 7.0, 1e-4, 5.25))
    assert np.count_nonzero(q) == 25


def test_soar_periodic_wraps():
    cnx, cny = 10, 8
    xi = np.random.RandomState(1).standard_normal((cny, cnx))
    q = on.apply_q(xi, cnx, cny, 7.0, 7.0, 1e-4, 5.25, True, True)
    # ghost rows/cols repeat the opposite interior ones
    assert np.allclose(q[:2], q[cny:cny + 2]) and np.allclose(q[:, :2], q[:, cnx:cnx + 2])


def test_bicubic_reproduces_quadratics_and_coarse_centres():
    factor, cnx, cny = 5, 8, 6
    nx, ny, dx, dy = cnx * factor, cny * factor, 7.0, 7.0
    cdx, cdy = dx * factor, dy * factor
    cx = (np.arange(cnx + 4) - 2 + 0.5) * cdx
    cy = (np.arange(cny + 4) - 2 + 0.5) * cdy
    X, Y = np.meshgrid(cx, cy)
    quad = lambda x, y: 0.3 + 1e-3 * x - 2e-3 * y + 1e-5 * x * x + 3e-6 * x * y - 2e-6 * y * y  # noqa: E731
    fine = on.interpolate(quad(X, Y), nx, ny, dx, dy, cdx, cdy)
    fx = (np.arange(nx + 4) - 2 + 0.5) * dx
    fy = (np.arange(ny + 4) - 2 + 0.5) * dy
    FX, FY = np.meshgrid(fx, fy)
    # away from the clamped edge the central differences are exact for quadratics
    inner = (slice(4, -4), slice(4, -4))
    assert np.allclose(fine[inner], quad(FX, FY)[inner], rtol=0, atol=1e-9)
    # the coarse values reappear at the coarse cell centres
    rnd = np.random.RandomState(2).standard_normal((cny + 4, cnx + 4))
    fine = on.interpolate(rnd, nx, ny, dx, dy, cdx, cdy)
    c0 = (factor - 1) // 2
    assert np.allclose(fine[2:-2, 2:-2][c0::factor, c0::factor], rnd[2:-2, 2:-2], atol=1e-12)


def test_geostrophic_balance_of_a_slope():
    nx, ny, dx, dy, g, f = 6, 5, 7.0, 7.0, 9.81, 0.02
    j, i = np.mgrid[0:ny + 4, 0:nx + 4]
    d_eta = 1e-3 * i + 2e-3 * j
    z = np.zeros((ny + 4, nx + 4))
    Hi = np.full((ny + 5, nx + 5), 5.0)
    eta, hu, hv = on.geostrophic(d_eta, z, z, z, Hi, nx, ny, dx, dy, g, f)
    h = d_eta[2:-2, 2:-2] + 5.0
    assert np.allclose(eta[2:-2, 2:-2], d_eta[2:-2, 2:-2])
    assert np.allclose(hu[2:-2, 2:-2], -(g / f) * h * 2e-3 / dy)
    assert np.allclose(hv[2:-2, 2:-2], (g / f) * h * 1e-3 / dx)
    Hi[3, 3] = 1e20
    eta, hu, hv = on.geostrophic(d_eta, z + 0.5, z, z, Hi, nx, ny, dx, dy, g, f)
    assert eta[3, 3] == 0 and eta[2, 2] == 0 and hu[2, 3] == 0 and eta[4, 4] != 0
