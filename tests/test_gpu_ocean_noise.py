"""Stochastic model error on the GPU (SWESimulators.OceanStateNoise,
go_noise_*).

* Against the reference's own kernels (oracle/_ref: ocean_noise.cu built
  with --use_fast_math): LCG normal and uniform numbers and seeds, SOAR on
  the four boundary combinations, the direct geostrophic balance (f-plane,
  beta plane, land, the Coriolis texture), the bicubic interpolation with
  factors 3, 5, 7 and grid offsets, the perpendicular field.  Bit for bit.
* Against the CPU oracle with the reference tests' tolerances
  (gpu_ocean/tests/stochastic/OceanStateNoise_test.py): perturbations of
  eta, of the ocean state, interpolation (with the coarse-versus-fine check)
  and the alignment offsets.
* The XORWOW path, the norms, the perpendicular pair and the simulator's
  small_scale_perturbation against their defining properties
  (RandomNumbers_test.py).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from SWESimulators import CDKLM16, Common  # noqa: E402
from SWESimulators.OceanStateNoise import OceanStateNoise  # noqa: E402
from oracle import build_ref, ocean_noise as on, ref_kernel  # noqa: E402

CFG = build_ref.CONFIGS["small_beta"]      # every reference library holds the noise kernels
BCS = [(True, True), (False, False), (True, False), (False, True)]
NX, NY, DX, F, G = 30, 40, 7.0, 0.02, 9.81   # OceanStateNoise_parent.py:40-50


@pytest.fixture(scope="module")
def ctx():
    return Common.CUDAContext()


def _ref(angle=((0.0,),), coriolis=((0.0,),)):
    if not ref_kernel.available(CFG):
        pytest.skip("reference kernel library not built")
    return ref_kernel.RefNoise(CFG, angle, coriolis)


def _bc(pns, pew):
    n = 2 if pns else 1
    e = 2 if pew else 1
    return Common.BoundaryConditions(n, e, n, e)


def _noise(ctx, nx=NX, ny=NY, pns=True, pew=True, factor=1, lcg=True, seed=7, **kw):
    n = OceanStateNoise(ctx, torch.cuda.current_stream(), nx, ny, DX, DX, _bc(pns, pew), False,
                        interpolation_factor=factor, use_lcg=lcg, **kw)
    if lcg:
        n.random_state = np.random.RandomState(seed)
        n.resetSeed()
    return n


def _pitched(a, extra_rows=16, extra_cols=32, dtype=np.float32):
    """A device copy of a 2-D array with spare rows and columns (the
    reference's SOAR tile reads past a non-periodic random field)."""
    a = np.ascontiguousarray(a, dtype=dtype)
    ny, nx = a.shape
    pe = ((nx + extra_cols + 31) // 32) * 32
    t = torch.zeros((ny + extra_rows, pe), dtype=torch.int64 if dtype == np.int64 else torch.float32, device="cuda")
    t[:ny, :nx] = torch.from_numpy(a).cuda()
    return t, pe * a.itemsize


def _host(tp, shape):
    torch.cuda.synchronize()
    return tp[0][:shape[0], :shape[1]].cpu().numpy()


def _state(nx, ny, land=None, eta0=None):
    eta = np.zeros((ny + 4, nx + 4), np.float32) if eta0 is None else eta0.astype(np.float32)
    Hi = np.full((ny + 5, nx + 5), 5.0, np.float32)
    if land is not None:
        for (j, i) in land:
            Hi[j, i] = 1e20
    return eta, Hi


def _arrays(ctx, nx, ny, eta, Hi):
    s = torch.cuda.current_stream()
    z = np.zeros_like(eta)
    return (Common.CUDAArray2D(s, nx, ny, 2, 2, eta), Common.CUDAArray2D(s, nx, ny, 2, 2, z),
            Common.CUDAArray2D(s, nx, ny, 2, 2, z), Common.CUDAArray2D(s, nx + 1, ny + 1, 2, 2, Hi))


# ---- against the reference's kernels ------------------------------------------

@pytest.mark.parametrize("normal", [True, False])
@pytest.mark.parametrize("pns, pew", BCS)
def test_lcg_vs_reference(ctx, normal, pns, pew):
    ref = _ref()
    n = _noise(ctx, pns=pns, pew=pew)
    seeds = n.getSeed().astype(np.int64)
    rs, rr = _pitched(seeds, dtype=np.int64), _pitched(np.zeros((n.rand_ny, n.rand_nx)))
    for _ in range(3):
        (n.generateNormalDistribution if normal else n.generateUniformDistribution)()
        ref.lcg(normal, int(n.seed_nx), int(n.seed_ny), int(n.rand_nx), rs, rr)
    mine = n.getRandomNumbers()
    theirs = _host(rr, mine.shape)
    assert np.array_equal(mine, theirs)
    assert np.array_equal(n.getSeed().astype(np.int64), _host(rs, seeds.shape))
    assert np.abs(mine).max() > 0


@pytest.mark.parametrize("factor", [1, 3])
@pytest.mark.parametrize("pns, pew", BCS)
def test_soar_vs_reference(ctx, pns, pew, factor):
    ref = _ref()
    n = _noise(ctx, NX * factor, NY * factor, pns, pew, factor)
    n.generateNormalDistribution()
    xi = n.getRandomNumbers()
    rr = _pitched(xi)
    shape = (n.coarse_ny + 4, n.coarse_nx + 4)
    rc = _pitched(np.zeros(shape))
    eta, Hi = _state(n.nx, n.ny)
    a = _arrays(ctx, n.nx, n.ny, eta, Hi)
    n.perturbOceanState(*a, F, update_random_field=False, ghost_cells_x=2, ghost_cells_y=2)
    ref.soar(int(n.coarse_nx), int(n.coarse_ny), n.coarse_dx, n.coarse_dy, n.soar_q0, n.soar_L, 1.0, pns, pew,
             rr, rc)
    mine, theirs = n.getCoarseBuffer(), _host(rc, shape)
    print("max |mine - reference| %.3g" % np.abs(mine - theirs).max())
    assert np.array_equal(mine, theirs)
    # additive second field (perpendicular_scale > 0)
    n.generateNormalDistributionPerpendicular()
    nu = n.getPerpendicularRandomNumbers()
    n.perturbOceanState(*a, F, update_random_field=False, perpendicular_scale=0.5)
    ref.soar(int(n.coarse_nx), int(n.coarse_ny), n.coarse_dx, n.coarse_dy, n.soar_q0, n.soar_L, 1.0, pns, pew,
             rr, rc)
    ref.soar(int(n.coarse_nx), int(n.coarse_ny), n.coarse_dx, n.coarse_dy, n.soar_q0, n.soar_L, 0.5, pns, pew,
             _pitched(nu), rc, additive=1)
    assert np.array_equal(n.getCoarseBuffer(), _host(rc, shape))


@pytest.mark.parametrize("case", ["fplane", "beta", "land", "coriolis_texture", "angle"])
def test_geostrophic_vs_reference(ctx, case):
    f, beta, land, angle, cor = F, 0.0, None, ((0.0,),), ((0.0,),)
    if case == "beta":
        beta = 1e-4
    if case == "land":
        land = [(5, 7), (12, 12), (30, 3)]
    if case == "coriolis_texture":
        f = 0.0
        cor = (0.01 + 1e-4 * np.arange(NY + 4, dtype=np.float32)).reshape(-1, 1)
    if case == "angle":
        beta, angle = 2e-4, ((0.3,),)
    ref = _ref(angle, cor)
    n = _noise(ctx, angle=np.asarray(angle, np.float32), coriolis_f=np.asarray(cor, np.float32))
    eta0 = np.random.RandomState(3).uniform(-0.1, 0.1, (NY + 4, NX + 4)).astype(np.float32)
    eta, Hi = _state(NX, NY, land, eta0)
    a = _arrays(ctx, NX, NY, eta, Hi)
    re, rhu, rhv, rH = _pitched(eta), _pitched(np.zeros_like(eta)), _pitched(np.zeros_like(eta)), _pitched(Hi)
    for _ in range(3):    # repeated: hu, hv non-zero from the second on
        n.perturbOceanState(*a, f, beta=beta, g=G, ghost_cells_x=2, ghost_cells_y=2)
        ref.geostrophic(NX, NY, DX, DX, G, f, beta, _pitched(n.getCoarseBuffer()), re, rhu, rhv, rH)
    for mine, theirs in zip((a[0], a[1], a[2]), (re, rhu, rhv)):
        m = mine.download(torch.cuda.current_stream())
        t = _host(theirs, m.shape)
        assert np.array_equal(m, t), np.abs(m - t).max()
    assert np.abs(a[1].download(torch.cuda.current_stream())).max() > 0


@pytest.mark.parametrize("factor, align", [(3, None), (5, None), (7, None), (5, 6), (5, 8)])
def test_bicubic_vs_reference(ctx, factor, align):
    ref = _ref()
    nx, ny = (NX, NY) if align else (NX * factor, NY * factor)
    n = _noise(ctx, nx, ny, factor=factor)
    eta, Hi = _state(nx, ny, land=[(7, 9)])
    a = _arrays(ctx, nx, ny, eta, Hi)
    oi, oj = n._obtain_coarse_grid_offset(align, align)
    re, rhu, rhv, rH = _pitched(eta), _pitched(np.zeros_like(eta)), _pitched(np.zeros_like(eta)), _pitched(Hi)
    for _ in range(3):
        n.perturbOceanState(*a, F, g=G, ghost_cells_x=2, ghost_cells_y=2, align_with_cell_i=align,
                            align_with_cell_j=align)
        ref.bicubic(nx, ny, DX, DX, int(n.coarse_nx), int(n.coarse_ny), n.coarse_dx, n.coarse_dy, oi, oj, G, F,
                    0.0, _pitched(n.getCoarseBuffer()), re, rhu, rhv, rH)
    for mine, theirs in zip(a[:3], (re, rhu, rhv)):
        m = mine.download(torch.cuda.current_stream())
        t = _host(theirs, m.shape)
        assert np.array_equal(m, t), np.abs(m - t).max()


def test_make_perpendicular_vs_reference(ctx):
    ref = _ref()
    n = _noise(ctx, 64, 48)
    n.generatePerpendicularNormalDistributions()
    xi = n.getRandomNumbers()
    # replay the last step on the reference's kernel from the same inputs
    n.generateNormalDistributionPerpendicular()
    nu0 = n.getPerpendicularRandomNumbers()
    n.findDoubleNormAndDot()
    red = torch.from_numpy(n.getReductionBuffer().reshape(-1).copy()).cuda()
    n._makePerpendicular()
    rx, rn = _pitched(xi), _pitched(nu0)
    ref.make_perpendicular(int(n.rand_nx), int(n.rand_ny), rx, rn, red)
    assert np.array_equal(n.getPerpendicularRandomNumbers(), _host(rn, nu0.shape))


# ---- against the CPU oracle (the reference tests' tolerances) --------------------

def _assert_places(a, b, places):
    # assert2DListAlmostEqual of the reference's testUtils: |a - b| < 0.5 10^-places
    assert np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max() < 0.5 * 10.0 ** (-places)


@pytest.mark.parametrize("pns, pew", BCS)
def test_perturb_ocean_vs_oracle(ctx, pns, pew):
    n = _noise(ctx, pns=pns, pew=pew)
    eta, Hi = _state(NX, NY)
    a = _arrays(ctx, NX, NY, eta, Hi)
    n.perturbOceanState(*a, F, 0.0, G)        # ghost cells 0, as the reference's perturb_ocean test
    xi = n.getRandomNumbers()
    eta2, Hi2 = _state(NX, NY)
    b = _arrays(ctx, NX, NY, eta2, Hi2)
    n.perturbOceanState(*b, F, 0.0, G, ghost_cells_x=2, ghost_cells_y=2, update_random_field=False)
    _, e, hu, hv = on.perturb_ocean_state(xi, eta2, np.zeros_like(eta2), np.zeros_like(eta2), Hi2, NX, NY, DX, DX,
                                          1, n.soar_q0, n.soar_L, pns, pew, G, F)
    s = torch.cuda.current_stream()
    me, mhu, mhv = (x.download(s) for x in b[:3])
    _assert_places(me / e.max(), e / e.max(), 5)
    _assert_places(mhu / hu.max(), hu / hu.max(), 5)
    _assert_places(mhv / hu.max(), hv / hu.max(), 5)


@pytest.mark.parametrize("factor", [3, 5, 7])
def test_interpolation_vs_oracle(ctx, factor):
    nx, ny = NX * factor, NY * factor
    n = _noise(ctx, nx, ny, factor=factor)
    eta, Hi = _state(nx, ny)
    a = _arrays(ctx, nx, ny, eta, Hi)
    n.perturbOceanState(*a, F, 0.0, G, ghost_cells_x=2, ghost_cells_y=2)
    xi = n.getRandomNumbers()
    coarse, e, hu, hv = on.perturb_ocean_state(xi, eta, np.zeros_like(eta), np.zeros_like(eta), Hi, nx, ny, DX, DX,
                                               factor, n.soar_q0, n.soar_L, True, True, G, F)
    s = torch.cuda.current_stream()
    me, mhu, mhv = (x.download(s) for x in a[:3])
    mx = e.max()
    _assert_places(me / mx, e / mx, 6)
    _assert_places(mhu / hu.max(), hu / hu.max(), 5)
    _assert_places(mhv / hu.max(), hv / hu.max(), 5)
    # coarse values reappear at the coarse cell centres of the fine field
    c0 = (factor - 1) // 2
    _assert_places(n.getCoarseBuffer()[2:-2, 2:-2] / mx, (me / mx)[2:-2, 2:-2][c0::factor, c0::factor], 5)


def test_alignment_offsets_shift_the_field(ctx):
    # OceanStateNoise_test.py:253-310: aligning with cells 6, 7, 8 (factor 5)
    # shifts the interpolated field by 1, 0, -1 cells on a periodic grid
    n = _noise(ctx, factor=5)
    n.generateNormalDistribution()
    eta, Hi = _state(NX, NY)
    base = None
    for align, shift in zip((7, 6, 8), (0, 1, -1)):
        a = _arrays(ctx, NX, NY, eta, Hi)
        n.perturbOceanState(*a, F, 0.0, G, ghost_cells_x=2, ghost_cells_y=2, update_random_field=False,
                            align_with_cell_i=align, align_with_cell_j=align)
        e = a[0].download(torch.cuda.current_stream())[2:-2, 2:-2]
        if base is None:
            base = e
            continue
        _assert_places(e / base.max(), np.roll(np.roll(base, -shift, 0), -shift, 1) / base.max(), 5)


# ---- generators, norms, simulator ------------------------------------------------

def test_xorwow_statistics_and_seed_rules(ctx):
    n = _noise(ctx, 400, 400, lcg=False, xorwow_seed=11)
    n.generateNormalDistribution()
    x = n.getRandomNumbers()
    assert abs(x.mean()) < 0.01 and abs(x.var() - 1.0) < 0.01
    n.generateUniformDistribution()
    u = n.getRandomNumbers()
    assert abs(u.mean() - 0.5) < 0.005 and abs(u.var() - 1 / 12) < 0.001
    n.generateNormalDistributionPerpendicular()
    v = n.getPerpendicularRandomNumbers()
    assert abs(v.mean()) < 0.01 and abs(v.var() - 1.0) < 0.01
    assert n.seed is None and n.host_seed is None
    with pytest.raises(AssertionError):
        n.getSeed()
    with pytest.raises(AssertionError):
        n.resetSeed()
    m = _noise(ctx, 400, 400, lcg=False, xorwow_seed=11)
    m.generateNormalDistribution()
    assert np.array_equal(m.getRandomNumbers(), x)      # same seed, same draws


@pytest.mark.parametrize("lcg", [True, False])
def test_norms_and_perpendicular(ctx, lcg):
    n = _noise(ctx, 400, 400, lcg=lcg, xorwow_seed=5)
    assert n.getReductionBuffer().shape == (1, 3) and not n.getReductionBuffer().any()
    n.generateNormalDistribution()
    xi = n.getRandomNumbers().astype(np.float64)
    gamma = n.getRandomNorm()
    assert abs((np.sum(xi * xi) - gamma) / np.sum(xi * xi)) < 5e-6
    n.generatePerpendicularNormalDistributions()
    xi = n.getRandomNumbers().astype(np.float64)
    nu = n.getPerpendicularRandomNumbers().astype(np.float64)
    rel = np.sum(xi * xi)
    pre = n.getReductionBuffer()
    n.findDoubleNormAndDot()
    post = n.getReductionBuffer()
    assert abs(post[0, 0] / rel - np.sum(xi * xi) / rel) < 5e-7
    assert abs(post[0, 1] / rel - np.sum(nu * nu) / rel) < 5e-6
    assert abs(post[0, 0] - pre[0, 0]) / rel < 5e-7
    assert abs(post[0, 1] - pre[0, 1]) / rel < 5e-6
    assert abs(post[0, 2] / rel) < 5e-4 and abs(np.sum(xi * nu)) < 5e-3
    assert abs(nu.mean()) < 0.01 and abs(nu.var() - 1.0) < 0.01


def test_seed_advances(ctx):
    n = _noise(ctx)
    s0 = n.getSeed()
    n.generateNormalDistribution()
    s1 = n.getSeed()
    n.generateUniformDistribution()
    s2 = n.getSeed()
    assert not np.array_equal(s0, s1) and not np.array_equal(s1, s2)
    assert np.array_equal(s1, on.fill_random(s0, int(n.rand_nx))[1])


def test_simulator_small_scale_perturbation(ctx):
    """CDKLM16 with small_scale_perturbation perturbs after every step:
    bit-identical to stepping without it and calling perturbSim and the
    boundary conditions by hand with the same seeds."""
    nx, ny, dx = 64, 48, 1000.0
    H = np.full((ny + 5, nx + 5), 60.0, np.float32)
    z = np.zeros((ny + 4, nx + 4), np.float32)
    kw = dict(eta0=z, hu0=z, hv0=z, H=H, nx=nx, ny=ny, dx=dx, dy=dx, dt=5.0, g=G, f=1.2e-4, r=0.0,
              boundary_conditions=Common.BoundaryConditions(2, 2, 2, 2))
    a = CDKLM16.CDKLM16(ctx, small_scale_perturbation=True, small_scale_perturbation_amplitude=1e-3,
                        use_lcg=True, **kw)
    b = CDKLM16.CDKLM16(ctx, **kw)
    nb = OceanStateNoise.fromsim(b, soar_q0=1e-3, use_lcg=True)
    seeds = a.small_scale_model_error.getSeed()
    nb.host_seed = seeds.copy()
    nb.seed.upload(b.gpu_stream, seeds)
    a.step(20.0)
    for _ in range(4):
        b.step(5.0)
        nb.perturbSim(b)
        b.applyBoundaryConditions()
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y)
    eta = a.download()[0]
    assert np.abs(eta).max() > 0
    a.perturbState(q0_scale=0.5)
    assert not np.array_equal(a.download()[0], eta)


@pytest.mark.parametrize("pns, pew", [(True, True), (False, False)])
def test_large_grid_vs_reference_with_timing(ctx, pns, pew):
    """2048 x 2048 model grid: three draws, SOAR and balance against the
    reference's kernels on copies of the same seeds and state, bit for bit;
    prints both sides' device times (CUDA events, 10 repetitions)."""
    n_cells = 2048
    ref = _ref()
    n = _noise(ctx, n_cells, n_cells, pns, pew)
    eta, Hi = _state(n_cells, n_cells, land=[(100, 200), (1500, 7)])
    a = _arrays(ctx, n_cells, n_cells, eta, Hi)
    rs = _pitched(n.getSeed().astype(np.int64), dtype=np.int64)
    rr = _pitched(np.zeros((n.rand_ny, n.rand_nx)))
    rc = _pitched(np.zeros((n.coarse_ny + 4, n.coarse_nx + 4)))
    re, rhu, rhv, rH = _pitched(eta), _pitched(np.zeros_like(eta)), _pitched(np.zeros_like(eta)), _pitched(Hi)

    def mine():
        n.perturbOceanState(*a, F, 0.0, G, ghost_cells_x=2, ghost_cells_y=2)

    def theirs():
        ref.lcg(True, int(n.seed_nx), int(n.seed_ny), int(n.rand_nx), rs, rr)
        ref.soar(int(n.coarse_nx), int(n.coarse_ny), n.coarse_dx, n.coarse_dy, n.soar_q0, n.soar_L, 1.0, pns, pew,
                 rr, rc)
        ref.geostrophic(n_cells, n_cells, DX, DX, G, F, 0.0, rc, re, rhu, rhv, rH)

    def timed(fn, reps=10):
        s = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            fn()
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    for _ in range(3):
        mine()
        theirs()
    for x, y in zip(a[:3], (re, rhu, rhv)):
        m = x.download(torch.cuda.current_stream())
        assert np.array_equal(m, _host(y, m.shape))
    t_mine, t_ref = timed(mine), timed(theirs)
    print("2048^2 perturbation (draws + SOAR + balance): ours %.3f ms, reference kernels %.3f ms (x%.2f)"
          % (t_mine, t_ref, t_ref / t_mine))


@pytest.mark.parametrize("ghost", [0, 1, 2])
@pytest.mark.parametrize("n, factor", [(47, 1), (63, 3)])
def test_ghost_offsets_vs_reference(ctx, ghost, n, factor):
    """Ghost offsets 0 and 1 (the reference's defaults of perturbOceanState)
    on grids of 16k - 1 cells, where the reference's 16 x 16 launch stops
    short of the last interior cells: the same cells change, bit for bit,
    through the direct (factor 1) and bicubic (factor 3) balance."""
    ref = _ref()
    nn = _noise(ctx, n, n, factor=factor)
    eta, Hi = _state(n, n)
    a = _arrays(ctx, n, n, eta, Hi)
    re, rhu, rhv, rH = _pitched(eta), _pitched(np.zeros_like(eta)), _pitched(np.zeros_like(eta)), _pitched(Hi)
    for _ in range(2):
        nn.perturbOceanState(*a, F, 0.0, G, ghost_cells_x=ghost, ghost_cells_y=ghost)
        rc = _pitched(nn.getCoarseBuffer())
        if factor == 1:
            ref.geostrophic(n, n, DX, DX, G, F, 0.0, rc, re, rhu, rhv, rH, gx=ghost, gy=ghost)
        else:
            ref.bicubic(n, n, DX, DX, int(nn.coarse_nx), int(nn.coarse_ny), nn.coarse_dx, nn.coarse_dy, 0, 0, G, F,
                        0.0, rc, re, rhu, rhv, rH, gx=ghost, gy=ghost)
    s = torch.cuda.current_stream()
    for x, y in zip(a[:3], (re, rhu, rhv)):
        m = x.download(s)
        assert np.array_equal(m, _host(y, m.shape))
    if ghost == 0:
        assert not a[1].download(s)[2:-2, -3].any()      # column n + 1 untouched, as in the reference
