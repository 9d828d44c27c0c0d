"""Seeded synthetic inputs for the benchmark and parity workloads.

No public dataset is involved: these are the workloads the CDKLM16
throughput numbers are quoted on, generated deterministically.

* ``bump256``   256 x 256, dx = dy = 200 m, flat Hi = 60 m, f-plane 1.2e-4,
                no friction or wind, walls; eta0 = 0.5 exp(-r^2/(10 dx)^2)
                centred in the domain; 1000 steps at CFL 0.7.
* ``grf4096``   4096 x 4096, dx = dy = 500 m, walls north/south, periodic
                east/west, beta-plane f = 1e-4 + 2e-11 y, Hi = 100 + 40 G
                (G a unit-variance Gaussian random field, squared-
                exponential correlation of 20 cells) clipped at 10 m,
                eta0 = 8 seeded Gaussian bumps, uniform wind stress
                0.1 N/m^2 at 45 degrees, quadratic friction r = 3e-3;
                2000 steps at CFL 0.7.
* ``grf(n)``    the grf4096 physics on an n x n grid (dx = 1 km for the
                ensemble and adjoint sizes).
"""

import numpy as np

RHO_WATER = 1025.0


def gaussian_random_field(shape, corr_cells, seed, periodic_x=True):
    """Unit-variance Gaussian random field by FFT filtering of seeded white
    noise with a squared-exponential covariance exp(-d^2 / (2 L^2)).  The
    field is periodic in x; in y a margin of 4L is generated and cut off so
    the field is not periodic there."""
    ny, nx = shape
    pad = int(4 * corr_cells)
    Ny = ny + pad
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((Ny, nx))
    ky = np.fft.fftfreq(Ny)[:, None]
    kx = np.fft.rfftfreq(nx)[None, :]
    L = float(corr_cells)
    # spectrum of exp(-d^2/(2L^2)) ~ exp(-2 pi^2 L^2 k^2); the filter is its sqrt
    filt = np.exp(-np.pi ** 2 * L ** 2 * (kx ** 2 + ky ** 2))
    g = np.fft.irfft2(np.fft.rfft2(w) * filt, s=(Ny, nx))[:ny]
    g -= g.mean()
    g /= g.std()
    return g


def gaussian_bumps(nx, ny, n, seed, amp=(0.1, 1.0), radius=(5.0, 30.0)):
    """Sum of n Gaussian bumps a*exp(-r^2/R^2) on the ghost-inclusive
    (ny+4) x (nx+4) grid; centres uniform over the interior, r and R in
    cells."""
    rng = np.random.default_rng(seed)
    cx = rng.uniform(0, nx, n)
    cy = rng.uniform(0, ny, n)
    a = rng.uniform(amp[0], amp[1], n)
    R = rng.uniform(radius[0], radius[1], n)
    x = np.arange(nx + 4) - 2 + 0.5
    y = np.arange(ny + 4) - 2 + 0.5
    eta = np.zeros((ny + 4, nx + 4))
    for k in range(n):
        ex = np.exp(-((x - cx[k]) ** 2) / R[k] ** 2)
        ey = np.exp(-((y - cy[k]) ** 2) / R[k] ** 2)
        eta += a[k] * np.outer(ey, ex)
    return eta.astype(np.float32)


class Case:
    """Everything a CDKLM16 constructor needs, plus the step count."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    def kwargs(self):
        """Keyword arguments of CDKLM16(...) apart from gpu_ctx and dt."""
        from .Common import BoundaryConditions
        from .WindStress import WindStress
        kw = dict(eta0=self.eta0, hu0=self.hu0, hv0=self.hv0, H=self.Hi, nx=self.nx, ny=self.ny,
                  dx=self.dx, dy=self.dy, g=self.g, f=self.f, r=self.r, coriolis_beta=self.beta,
                  boundary_conditions=BoundaryConditions(*self.bc))
        if self.wind != (0.0, 0.0):
            kw["wind_stress"] = WindStress(t=[0], X=[np.array([[self.wind[0]]], np.float32)],
                                           Y=[np.array([[self.wind[1]]], np.float32)])
        return kw


def cfl_dt(case, courant=0.7):
    """courant * exact CFL limit at t = 0, in float64 on the host, from the
    case's state (hu = hv = 0 here so u = v = 0): 0.25*min(dx,dy)/sqrt(g h)
    over wet interior cells, with Bm = mean of the four corners."""
    H = case.Hi.astype(np.float64)
    Bm = 0.25 * (H[:-1, :-1] + H[1:, :-1] + H[:-1, 1:] + H[1:, 1:])
    J = slice(2, case.ny + 2)
    I = slice(2, case.nx + 2)
    eta = np.maximum(case.eta0.astype(np.float64), -Bm)
    h = (eta + Bm)[J, I]
    u = case.hu0.astype(np.float64)[J, I] / h
    v = case.hv0.astype(np.float64)[J, I] / h
    c = np.sqrt(case.g * h)
    lim = min(np.min(0.25 * case.dx / (np.abs(u) + c)), np.min(0.25 * case.dy / (np.abs(v) + c)))
    return float(np.float32(courant * lim))


def bump256():
    nx = ny = 256
    dx = dy = 200.0
    Hi = np.full((ny + 5, nx + 5), 60.0, dtype=np.float32)
    x = (np.arange(nx + 4) - 2 + 0.5) * dx
    y = (np.arange(ny + 4) - 2 + 0.5) * dy
    X, Y = np.meshgrid(x, y)
    r2 = (X - 128 * dx) ** 2 + (Y - 128 * dy) ** 2
    eta0 = (0.5 * np.exp(-r2 / (10 * dx) ** 2)).astype(np.float32)
    z = np.zeros_like(eta0)
    c = Case(name="bump256", nx=nx, ny=ny, dx=dx, dy=dy, g=9.81, f=1.2e-4, beta=0.0, r=0.0,
             bc=(1, 1, 1, 1), wind=(0.0, 0.0), eta0=eta0, hu0=z, hv0=z.copy(), Hi=Hi, steps=1000)
    c.dt = cfl_dt(c)
    return c


def grf(n, dx=1000.0, seed_bathy=20241, seed_bumps=20242, steps=2000, f0=1.0e-4, beta=2.0e-11, ny=None,
        bc=(1, 2, 1, 2), r=3.0e-3):
    """The headline physics on an n x n grid (n x ny if ny is given);
    bc = (north, east, south, west) codes, r the friction coefficient."""
    nx = int(n)
    ny = nx if ny is None else int(ny)
    dy = dx
    G = gaussian_random_field((ny + 1, nx), 20, seed_bathy)
    Hi = np.zeros((ny + 5, nx + 5), dtype=np.float64)
    Hi[2:ny + 3, 2:nx + 2] = np.maximum(100.0 + 40.0 * G, 10.0)
    # ghost corners by the reference's rule (walls north/south, periodic east/west)
    for j in range(2):
        Hi[j, :] = Hi[4 - j, :]
        Hi[ny + 4 - j, :] = Hi[ny + j, :]
    Hi[:, nx + 2] = Hi[:, 2]
    for i in range(2):
        Hi[:, i] = Hi[:, i + nx]
    for i in range(nx + 2, nx + 5):
        Hi[:, i] = Hi[:, i - nx]
    Hi = Hi.astype(np.float32)
    eta0 = gaussian_bumps(nx, ny, 8, seed_bumps)
    Hf = Hi.astype(np.float64)
    Bm = (0.25 * (Hf[:-1, :-1] + Hf[1:, :-1] + Hf[:-1, 1:] + Hf[1:, 1:])).astype(np.float32)
    eta0 = np.maximum(eta0, -Bm)
    z = np.zeros_like(eta0)
    tau = 0.1 * np.cos(np.pi / 4) / RHO_WATER
    c = Case(name="grf%d" % n, nx=nx, ny=ny, dx=dx, dy=dy, g=9.81, f=f0 + 2 * beta * dy, beta=beta, r=float(r),
             bc=tuple(int(b) for b in bc), wind=(np.float32(tau), np.float32(tau)), eta0=eta0, hu0=z, hv0=z.copy(),
             Hi=Hi, steps=steps)
    c.dt = cfl_dt(c)
    return c


def grf4096():
    return grf(4096, dx=500.0, steps=2000)
