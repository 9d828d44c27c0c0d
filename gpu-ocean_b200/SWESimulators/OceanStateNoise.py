"""Stochastic model error: small-scale, geostrophically balanced
perturbations of an ocean state (the reference's
gpu_ocean/SWESimulators/OceanStateNoise.py:40-571).

A random field xi ~ N(0, I) on a coarse grid (LCG or XORWOW), the SOAR
covariance Q applied to it with a cut-off of two cells, d_eta = Q xi added
to eta, and d_hu, d_hv from the geostrophic balance of d_eta added to hu,
hv.  A coarse grid interpolation_factor times coarser than the model grid
is interpolated bicubically.  Every kernel is in the in-tree CUDA library
(csrc/ocean_noise.cu, go_noise_*); this class keeps the reference's
interface: the constructor, fromsim, perturbSim, perturbOceanState, the
random-number generators, the norms and the perpendicular field.

The reference's CPU twins of these methods (OceanStateNoise.py:572-937) are
test code and live with the other CPU restatements, outside this package.
"""

import ctypes

import numpy as np

from . import Common, _native

SOAR_CUTOFF = 2     # gpu_ocean/SWESimulators/config.py:31


def noise_layout(nx, ny, dx, boundaryConditions, interpolation_factor=1, block_width=16, block_height=16):
    """Sizes of the random, seed and coarse buffers for an nx x ny model
    grid (OceanStateNoise.py:93-152), and the reference's launch grids for
    its block size (OceanStateNoise.py:250-282)."""
    assert interpolation_factor > 0 and interpolation_factor % 2 == 1, \
        'interpolation_factor must be a positive odd integer'
    assert nx % interpolation_factor == 0, 'nx must be divisible by the interpolation factor'
    assert ny % interpolation_factor == 0, 'ny must be divisible by the interpolation factor'
    L = {}
    L["interpolation_factor"] = np.int32(interpolation_factor)
    L["coarse_nx"] = np.int32(nx / interpolation_factor)
    L["coarse_ny"] = np.int32(ny / interpolation_factor)
    L["periodicNorthSouth"] = np.int32(boundaryConditions.isPeriodicNorthSouth())
    L["periodicEastWest"] = np.int32(boundaryConditions.isPeriodicEastWest())
    gx = 0 if L["periodicEastWest"] else 2 + SOAR_CUTOFF
    gy = 0 if L["periodicNorthSouth"] else 2 + SOAR_CUTOFF
    L["rand_ghost_cells_x"], L["rand_ghost_cells_y"] = np.int32(gx), np.int32(gy)
    L["rand_nx"] = np.int32(L["coarse_nx"] + 2 * gx)
    L["rand_ny"] = np.int32(L["coarse_ny"] + 2 * gy)
    L["seed_ny"] = np.int32(L["rand_ny"])
    L["seed_nx"] = np.int32(np.ceil(L["rand_nx"] / 2))
    bw, bh = block_width, block_height
    L["local_size"] = (bw, bh, 1)
    L["global_size_random_numbers"] = (int(np.ceil(L["seed_nx"] / float(bw))), int(np.ceil(L["seed_ny"] / float(bh))))
    L["global_size_perpendicular"] = (int(np.ceil(L["rand_nx"] / float(bw))), int(np.ceil(L["rand_ny"] / float(bh))))
    L["global_size_SOAR"] = (int(np.ceil((L["coarse_nx"] + 4) / float(bw))),
                             int(np.ceil((L["coarse_ny"] + 4) / float(bh))))
    L["global_size_geo_balance"] = (int(np.ceil(nx / float(bw))), int(np.ceil(ny / float(bh))))
    return L


def coarse_grid_offset(interpolation_factor, fine_index_i, fine_index_j):
    """Shift of the coarse grid that centres a coarse cell on model cell
    (fine_index_i, fine_index_j) (OceanStateNoise.py:498-513)."""
    default_offset = interpolation_factor // 2
    offset_i, offset_j = 0, 0
    if fine_index_i is not None:
        offset_i = -int(fine_index_i % interpolation_factor - default_offset)
    if fine_index_j is not None:
        offset_j = -int(fine_index_j % interpolation_factor - default_offset)
    return offset_i, offset_j


class _SeedArray:
    """seed_ny x seed_nx 64-bit LCG seeds on the device, rows padded to 128
    bytes (the reference's integer CUDAArray2D)."""

    def __init__(self, host_seed):
        torch = _native.require_cuda()
        self.ny, self.nx = host_seed.shape
        self.pitch_elems = Common.round_up(self.nx, 16)
        self.pitch = self.pitch_elems * 8
        self.tensor = torch.zeros((self.ny, self.pitch_elems), dtype=torch.int64, device="cuda")

    def upload(self, gpu_stream, host_seed):
        torch = _native.require_cuda()
        src = torch.from_numpy(np.ascontiguousarray(host_seed.astype(np.int64)))
        with torch.cuda.stream(gpu_stream):
            self.tensor[:, :self.nx].copy_(src, non_blocking=False)

    def download(self, gpu_stream):
        gpu_stream.synchronize()
        return self.tensor[:, :self.nx].cpu().numpy().astype(np.uint64)


class OceanStateNoise(object):
    """Small-scale, geostrophically balanced perturbations of an ocean state
    (OceanStateNoise.py:40-571)."""

    def __init__(self, gpu_ctx, gpu_stream, nx, ny, dx, dy, boundaryConditions, staggered,
                 soar_q0=None, soar_L=None, interpolation_factor=1, use_lcg=False, xorwow_seed=None,
                 angle=np.array([[0]], dtype=np.float32), coriolis_f=np.array([[0]], dtype=np.float32),
                 block_width=16, block_height=16):
        torch = _native.require_cuda()
        self.lib = _native.load()
        self.use_lcg = use_lcg
        self.random_state = np.random.RandomState()
        self.random_numbers = None
        self.perpendicular_random_numbers = None
        self.coarse_buffer = None
        self.reduction_buffer = None
        self.rng = None
        self.seed = None
        self.host_seed = None
        self._textures = []
        self.gpu_ctx = gpu_ctx
        self.gpu_stream = gpu_stream
        self.nx, self.ny = np.int32(nx), np.int32(ny)
        self.dx, self.dy = np.float32(dx), np.float32(dy)
        self.staggered = 1 if staggered else 0
        self.cutoff = np.int32(SOAR_CUTOFF)
        L = noise_layout(int(nx), int(ny), dx, boundaryConditions, interpolation_factor, block_width, block_height)
        for k, v in L.items():
            setattr(self, k, v)
        self.coarse_dx = np.float32(dx * self.interpolation_factor)
        self.coarse_dy = np.float32(dy * self.interpolation_factor)

        self.floatMax = 2147483648.0
        if self.use_lcg:
            self.host_seed = (self.random_state.rand(self.seed_ny, self.seed_nx) * self.floatMax).astype(
                np.uint64, order='C')
            self.seed = _SeedArray(self.host_seed)
            self.seed.upload(gpu_stream, self.host_seed)
        else:
            if xorwow_seed is None:
                xorwow_seed = int(np.random.randint(0, 2 ** 31 - 1))
            n_random = int(self.rand_nx) * int(self.rand_ny)
            self._n_generators = int(min(148 * 8 * 128, max(1, (n_random + 1) // 2)))
            nbytes = self._n_generators * int(self.lib.go_noise_xorwow_state_bytes())
            self.rng = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
            _native.check(self.lib.go_noise_xorwow_init(self._s(), ctypes.c_uint64(int(xorwow_seed)),
                                                        self._n_generators, _native.ptr(self.rng)))

        self.soar_q0 = np.float32(self.dx / 100000)
        if soar_q0 is not None:
            self.soar_q0 = np.float32(soar_q0)
        self.soar_L = np.float32(0.75 * self.coarse_dx)
        if soar_L is not None:
            self.soar_L = np.float32(soar_L)

        zeros_rand = np.zeros((self.rand_ny, self.rand_nx), dtype=np.float32)
        self.random_numbers_host = zeros_rand.copy()
        self.random_numbers = Common.CUDAArray2D(gpu_stream, self.rand_nx, self.rand_ny, 0, 0, zeros_rand)
        self.perpendicular_random_numbers_host = zeros_rand.copy()
        self.perpendicular_random_numbers = Common.CUDAArray2D(gpu_stream, self.rand_nx, self.rand_ny, 0, 0,
                                                               zeros_rand)
        self.coarse_buffer_host = np.zeros((self.coarse_ny + 4, self.coarse_nx + 4), dtype=np.float32)
        self.coarse_buffer = Common.CUDAArray2D(gpu_stream, self.coarse_nx, self.coarse_ny, 2, 2,
                                                self.coarse_buffer_host)
        self.reduction_buffer = Common.CUDAArray2D(gpu_stream, 3, 1, 0, 0, np.zeros((1, 3), dtype=np.float32))
        self._red_scratch = torch.zeros(int(self.lib.go_noise_reduce_scratch_bytes()), dtype=torch.uint8,
                                        device="cuda")
        self._angle_tex = self._texture(angle)
        self._coriolis_tex = self._texture(coriolis_f)

    def _texture(self, field):
        arr = np.ascontiguousarray(np.asarray(field, dtype=np.float32))
        if arr.ndim != 2:
            arr = arr.reshape(1, -1) if arr.size > 1 else arr.reshape(1, 1)
        h = ctypes.c_uint64()
        _native.check(self.lib.go_wind_texture_create(arr.ctypes.data_as(ctypes.c_void_p), arr.shape[1],
                                                      arr.shape[0], ctypes.byref(h)))
        self._textures.append(h.value)
        return h.value

    def _s(self, stream=None):
        return _native.stream_handle(self.gpu_stream if stream is None else stream)

    def __del__(self):
        self.cleanUp()

    def cleanUp(self):
        lib = getattr(self, "lib", None)
        for h in getattr(self, "_textures", []):
            lib.go_wind_texture_destroy(h)
        self._textures = []
        for name in ("random_numbers", "perpendicular_random_numbers", "coarse_buffer", "reduction_buffer"):
            a = getattr(self, name, None)
            if a is not None:
                a.release()
                setattr(self, name, None)
        self.rng = None
        self.seed = None
        self.gpu_ctx = None

    @classmethod
    def fromsim(cls, sim, soar_q0=None, soar_L=None, interpolation_factor=1, use_lcg=False, xorwow_seed=None,
                block_width=16, block_height=16):
        """The perturbation for a simulator, with its grid, boundary
        conditions, angle and Coriolis textures (OceanStateNoise.py:318-333)."""
        return cls(sim.gpu_ctx, sim.gpu_stream, sim.nx, sim.ny, sim.dx, sim.dy, sim.boundary_conditions, False,
                   soar_q0=soar_q0, soar_L=soar_L, interpolation_factor=interpolation_factor,
                   angle=sim.angle_texture_field(), coriolis_f=sim.coriolis_texture_field(),
                   use_lcg=use_lcg, xorwow_seed=xorwow_seed, block_width=block_width, block_height=block_height)

    # ---- seeds and random numbers -------------------------------------------

    def getSeed(self):
        assert self.use_lcg, "getSeed is only valid if LCG is used as pseudo-random generator."
        return self.seed.download(self.gpu_stream)

    def resetSeed(self):
        assert self.use_lcg, "resetSeed is only valid if LCG is used as pseudo-random generator."
        self.host_seed = (self.random_state.rand(self.seed_ny, self.seed_nx) * self.floatMax).astype(
            np.uint64, order='C')
        self.seed.upload(self.gpu_stream, self.host_seed)

    def getRandomNumbers(self):
        return self.random_numbers.download(self.gpu_stream)

    def getPerpendicularRandomNumbers(self):
        return self.perpendicular_random_numbers.download(self.gpu_stream)

    def getCoarseBuffer(self):
        return self.coarse_buffer.download(self.gpu_stream)

    def getReductionBuffer(self):
        return self.reduction_buffer.download(self.gpu_stream)

    def _fill(self, target, normal):
        if self.use_lcg:
            _native.check(self.lib.go_noise_lcg(self._s(), int(normal), int(self.seed_nx), int(self.seed_ny),
                                                int(self.rand_nx), _native.ptr(self.seed.tensor), self.seed.pitch,
                                                _native.ptr(target.tensor), int(target.pitch)))
        else:
            _native.check(self.lib.go_noise_xorwow_fill(self._s(), int(normal), self._n_generators,
                                                        _native.ptr(self.rng), int(self.rand_nx),
                                                        int(self.rand_ny), _native.ptr(target.tensor),
                                                        int(target.pitch)))

    def generateNormalDistribution(self):
        self._fill(self.random_numbers, True)

    def generateNormalDistributionPerpendicular(self):
        self._fill(self.perpendicular_random_numbers, True)

    def generateUniformDistribution(self):
        self._fill(self.random_numbers, False)

    # ---- perturbations ------------------------------------------------------

    def perturbSim(self, sim, q0_scale=1.0, update_random_field=True, perturbation_scale=1.0,
                   perpendicular_scale=0.0, align_with_cell_i=None, align_with_cell_j=None, stream=None):
        """Adds a perturbation to the simulator's current state
        (OceanStateNoise.py:376-397)."""
        self.perturbOceanState(sim.gpu_data.h0, sim.gpu_data.hu0, sim.gpu_data.hv0, sim.bathymetry.Bi,
                               sim.f, beta=sim.coriolis_beta, g=sim.g,
                               y0_reference_cell=sim.y_zero_reference_cell,
                               ghost_cells_x=sim.ghost_cells_x, ghost_cells_y=sim.ghost_cells_y,
                               q0_scale=q0_scale, update_random_field=update_random_field,
                               perturbation_scale=perturbation_scale, perpendicular_scale=perpendicular_scale,
                               align_with_cell_i=align_with_cell_i, align_with_cell_j=align_with_cell_j,
                               land_mask_value=sim.bathymetry.mask_value, stream=stream)

    def perturbOceanState(self, eta, hu, hv, H, f, beta=0.0, g=9.81, y0_reference_cell=0, ghost_cells_x=0,
                          ghost_cells_y=0, q0_scale=1.0, update_random_field=True, perturbation_scale=1.0,
                          perpendicular_scale=0.0, align_with_cell_i=None, align_with_cell_j=None,
                          land_mask_value=np.float32(1.0e20), stream=None):
        """eta += Q xi, (hu, hv) += their geostrophic balance, on the stream
        (OceanStateNoise.py:399-496)."""
        if stream is None:
            stream = self.gpu_stream
        if update_random_field:
            self.generateNormalDistribution()
        s = self._s(stream)
        # q0 x q0_scale in double, then float (the reference's NumPy 1
        # scalar arithmetic; go_noise_batch_perturb forms it the same way)
        soar_q0 = np.float32(np.float64(self.soar_q0) * np.float64(q0_scale))
        offset_i, offset_j = coarse_grid_offset(int(self.interpolation_factor), align_with_cell_i,
                                                align_with_cell_j)
        rn, cb = self.random_numbers, self.coarse_buffer
        phys = (float(np.float32(g)), float(np.float32(f)), float(np.float32(beta)),
                float(np.float32(y0_reference_cell)))
        tail = (_native.ptr(cb.tensor), int(cb.pitch), _native.ptr(eta.tensor), int(eta.pitch),
                _native.ptr(hu.tensor), int(hu.pitch), _native.ptr(hv.tensor), int(hv.pitch),
                _native.ptr(H.tensor), int(H.pitch), float(np.float32(land_mask_value)),
                ctypes.c_uint64(self._angle_tex), ctypes.c_uint64(self._coriolis_tex))
        _native.check(self.lib.go_noise_soar(s, int(self.coarse_nx), int(self.coarse_ny), float(self.coarse_dx),
                                             float(self.coarse_dy), float(soar_q0), float(self.soar_L),
                                             float(np.float32(perturbation_scale)), int(self.periodicNorthSouth),
                                             int(self.periodicEastWest), _native.ptr(rn.tensor), int(rn.pitch),
                                             _native.ptr(cb.tensor), int(cb.pitch), 0))
        if perpendicular_scale > 0:
            pn = self.perpendicular_random_numbers
            _native.check(self.lib.go_noise_soar(s, int(self.coarse_nx), int(self.coarse_ny),
                                                 float(self.coarse_dx), float(self.coarse_dy), float(soar_q0),
                                                 float(self.soar_L), float(np.float32(perpendicular_scale)),
                                                 int(self.periodicNorthSouth), int(self.periodicEastWest),
                                                 _native.ptr(pn.tensor), int(pn.pitch), _native.ptr(cb.tensor),
                                                 int(cb.pitch), 1))
        if self.interpolation_factor > 1:
            _native.check(self.lib.go_noise_bicubic(s, int(self.nx), int(self.ny), int(ghost_cells_x),
                                                    int(ghost_cells_y), float(self.dx), float(self.dy),
                                                    int(self.coarse_nx), int(self.coarse_ny), int(ghost_cells_x),
                                                    int(ghost_cells_y), float(self.coarse_dx),
                                                    float(self.coarse_dy), int(offset_i), int(offset_j),
                                                    *phys, *tail))
        else:
            _native.check(self.lib.go_noise_geostrophic(s, int(self.nx), int(self.ny), float(self.dx),
                                                        float(self.dy), int(ghost_cells_x), int(ghost_cells_y),
                                                        *phys, *tail))

    def member_desc(self, sim):
        """The go_noise_member descriptor of this perturbation applied to
        sim's state (for go_noise_batch_create)."""
        m = _native.GoNoiseMember()
        if self.use_lcg:
            m.seed, m.seed_pitch = int(self.seed.tensor.data_ptr()), int(self.seed.pitch)
        else:
            m.xorwow_states, m.n_generators = int(self.rng.data_ptr()), int(self._n_generators)
        m.random, m.random_pitch = int(self.random_numbers.tensor.data_ptr()), int(self.random_numbers.pitch)
        m.coarse, m.coarse_pitch = int(self.coarse_buffer.tensor.data_ptr()), int(self.coarse_buffer.pitch)
        g = sim.gpu_data
        m.eta, m.eta_pitch = int(g.h0.tensor.data_ptr()), int(g.h0.pitch)
        m.hu, m.hu_pitch = int(g.hu0.tensor.data_ptr()), int(g.hu0.pitch)
        m.hv, m.hv_pitch = int(g.hv0.tensor.data_ptr()), int(g.hv0.pitch)
        Bi = sim.bathymetry.Bi
        m.Hi, m.Hi_pitch = int(Bi.tensor.data_ptr()), int(Bi.pitch)
        m.angle_texture, m.coriolis_texture = self._angle_tex, self._coriolis_tex
        m.soar_q0 = float(self.soar_q0)
        m.g, m.f, m.beta = float(np.float32(sim.g)), float(np.float32(sim.f)), float(np.float32(sim.coriolis_beta))
        m.land_value = float(np.float32(sim.bathymetry.mask_value))
        return m

    def _obtain_coarse_grid_offset(self, fine_index_i, fine_index_j):
        return coarse_grid_offset(int(self.interpolation_factor), fine_index_i, fine_index_j)

    # ---- norms and the perpendicular field ----------------------------------

    def _square_sums(self, b=None):
        a = self.random_numbers
        _native.check(self.lib.go_noise_square_sums(
            self._s(), int(self.rand_nx), int(self.rand_ny), _native.ptr(a.tensor), int(a.pitch),
            _native.ptr(b.tensor) if b is not None else None, int(b.pitch) if b is not None else 0,
            _native.ptr(self.reduction_buffer.tensor), _native.ptr(self._red_scratch),
            self._red_scratch.numel()))

    def getRandomNorm(self):
        """sum(xi^2) over the random buffer (OceanStateNoise.py:515-528)."""
        self._square_sums()
        return self.getReductionBuffer()[0, 0]

    def findDoubleNormAndDot(self):
        """[sum(xi^2), sum(nu^2), sum(xi nu)] into the reduction buffer
        (OceanStateNoise.py:530-543)."""
        self._square_sums(self.perpendicular_random_numbers)

    def _makePerpendicular(self):
        """nu made perpendicular to xi with its norm kept
        (OceanStateNoise.py:545-557)."""
        xi, nu = self.random_numbers, self.perpendicular_random_numbers
        _native.check(self.lib.go_noise_make_perpendicular(
            self._s(), int(self.rand_nx), int(self.rand_ny), _native.ptr(xi.tensor), int(xi.pitch),
            _native.ptr(nu.tensor), int(nu.pitch), _native.ptr(self.reduction_buffer.tensor)))

    def generatePerpendicularNormalDistributions(self):
        """xi, nu ~ N(0, I) with nu perpendicular to xi
        (OceanStateNoise.py:559-571)."""
        self.generateNormalDistribution()
        self.generateNormalDistributionPerpendicular()
        self.findDoubleNormAndDot()
        self._makePerpendicular()
