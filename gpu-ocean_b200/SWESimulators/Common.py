"""Device arrays, boundary conditions and bathymetry for the CDKLM16 path.

Mirrors the parts of gpu_ocean/SWESimulators/Common.py that the CDKLM16
simulator and its callers use:

* ``CUDAContext``                  (Common.py:285-495)  -- device handle, no JIT
* ``CUDAArray2D``                  (Common.py:503-631)  -- torch-backed, padded pitch
* ``SWEDataArakawaA``              (Common.py:634-690)
* ``BoundaryConditions`` / ``BoundaryConditionsData`` (Common.py:824-1014)
* ``BoundaryConditionsArakawaA``   (Common.py:1019-1309) -- wall, periodic and open (3/4)
* ``Bathymetry``                   (Common.py:1313-1459)

Device memory is allocated by PyTorch; every kernel is the in-tree CUDA
library reached through ``_native`` (no CPU fallback).
"""

import logging

import ctypes

import re

import numpy as np

from . import _native


def _torch():
    return _native.require_cuda()


def round_up(n, m):
    return ((int(n) + m - 1) // m) * m


class CUDAContext:
    """Device selection and synchronisation (Common.py:285-331).  Kernels are
    prebuilt for sm_100a, so there is no runtime compiler or cache."""

    def __init__(self, device=0, blocking=False, use_cache=True, autotuning=False):
        torch = _torch()
        self.logger = logging.getLogger(__name__)
        self.device_index = int(device)
        torch.cuda.set_device(self.device_index)
        self.device = torch.device("cuda", self.device_index)
        self.blocking = blocking
        _native.load()

    def __str__(self):
        torch = _torch()
        return "CUDAContext id %d (%s)" % (self.device_index, torch.cuda.get_device_name(self.device_index))

    def synchronize(self):
        _torch().cuda.synchronize(self.device)

    def get_kernel(self, *args, **kwargs):
        raise NotImplementedError("kernels are prebuilt for sm_100a; there is no runtime compilation")


class _DeviceData:
    """Stand-in for the pycuda GPUArray held in ``CUDAArray2D.data``: exposes
    the device pointer as ``gpudata`` / ``ptr`` and the torch tensor."""

    def __init__(self, tensor):
        self.tensor = tensor

    @property
    def gpudata(self):
        return int(self.tensor.data_ptr())

    @property
    def ptr(self):
        return int(self.tensor.data_ptr())

    @property
    def shape(self):
        return tuple(self.tensor.shape)


class CUDAArray2D:
    """A (ny + 2*halo_y) x (nx + 2*halo_x) float32 array on the device.

    Rows are padded to a multiple of 32 floats (128 bytes) so every row
    starts on a cache-line boundary; ``pitch`` is the row stride in bytes,
    as in the reference (which uses an unpadded pitch, Common.py:546).
    """

    PAD_FLOATS = 32

    def __init__(self, gpu_stream, nx, ny, halo_x, halo_y, data, asymHalo=None,
                 double_precision=False, integers=False):
        torch = _torch()
        if double_precision or integers:
            raise NotImplementedError("only float32 device arrays are used on the CDKLM16 path")
        self.double_precision = False
        self.integers = False
        self.nx, self.ny = int(nx), int(ny)
        self.nx_halo = int(nx) + 2 * int(halo_x)
        self.ny_halo = int(ny) + 2 * int(halo_y)
        if asymHalo is not None and len(asymHalo) == 4:
            self.nx_halo = int(nx) + int(asymHalo[1]) + int(asymHalo[3])
            self.ny_halo = int(ny) + int(asymHalo[0]) + int(asymHalo[2])
        host = self.convert_to_float32(data)
        assert host.shape == (self.ny_halo, self.nx_halo), \
            str(host.shape) + " vs " + str((self.ny_halo, self.nx_halo))
        self.bytes_per_float = 4
        self.pitch_floats = round_up(self.nx_halo, self.PAD_FLOATS)
        self.pitch = np.int32(self.pitch_floats * 4)
        self.tensor = torch.zeros((self.ny_halo, self.pitch_floats), dtype=torch.float32, device="cuda")
        self.data = _DeviceData(self.tensor)
        self.holds_data = True
        self.mask = data.mask if np.ma.is_masked(data) else None
        self.upload(gpu_stream, data)

    @property
    def view(self):
        """The (ny_halo, nx_halo) torch view without the row padding."""
        return self.tensor[:, :self.nx_halo]

    def upload(self, gpu_stream, data):
        torch = _torch()
        if not self.holds_data:
            raise RuntimeError("The buffer has been freed before upload is called")
        if torch.is_tensor(data):
            # host tensor (pinned for an asynchronous copy) or device tensor
            assert tuple(data.shape) == (self.ny_halo, self.nx_halo), \
                str(tuple(data.shape)) + " vs " + str((self.ny_halo, self.nx_halo))
            with torch.cuda.stream(gpu_stream) if gpu_stream is not None else _null():
                self.view.copy_(data.to(torch.float32), non_blocking=True)
            return
        if np.ma.is_masked(data):
            self.mask = data.mask
        host = self.convert_to_float32(data)
        assert host.shape == (self.ny_halo, self.nx_halo), \
            str(host.shape) + " vs " + str((self.ny_halo, self.nx_halo))
        src = torch.from_numpy(np.ascontiguousarray(host))
        with torch.cuda.stream(gpu_stream) if gpu_stream is not None else _null():
            self.view.copy_(src.to(self.tensor.device, non_blocking=False))

    def copyBuffer(self, gpu_stream, buffer):
        torch = _torch()
        if not self.holds_data:
            raise RuntimeError("The buffer has been freed before copying buffer")
        if not buffer.holds_data:
            raise RuntimeError("The provided buffer is either not allocated, or has been freed before copying buffer")
        assert buffer.nx_halo == self.nx_halo and buffer.ny_halo == self.ny_halo
        with torch.cuda.stream(gpu_stream) if gpu_stream is not None else _null():
            self.view.copy_(buffer.view)

    def download(self, gpu_stream):
        """Host copy (numpy, ny_halo x nx_halo) of the array after the work
        queued on gpu_stream.  The copy lands in page-locked memory (one
        asynchronous device-to-host copy on the stream, then a wait); a
        pageable destination took 44 ms per 4096^2 field on a B200, the
        page-locked one a few."""
        torch = _torch()
        if not self.holds_data:
            raise RuntimeError("CUDA buffer has been freed")
        host_t = torch.empty((self.ny_halo, self.nx_halo), dtype=torch.float32, pin_memory=True)
        stream = gpu_stream if gpu_stream is not None else torch.cuda.current_stream()
        with torch.cuda.stream(stream):
            host_t.copy_(self.view, non_blocking=True)
        stream.synchronize()
        host = host_t.numpy()
        if self.mask is not None:
            host = np.ma.array(host, mask=self.mask)
        return host

    def release(self):
        if self.holds_data:
            self.tensor = None
            self.data = None
            self.holds_data = False

    @staticmethod
    def convert_to_float32(data):
        data = np.ma.getdata(data) if np.ma.isMaskedArray(data) else data
        if not np.issubdtype(np.asarray(data).dtype, np.float32) or np.isfortran(data):
            return np.asarray(data).astype(np.float32, order="C")
        return np.asarray(data)


class _null:
    def __enter__(self):
        return None

    def __exit__(self, *a):
        return False


class SWEDataArakawaA:
    """Double-buffered (eta, hu, hv) on an unstaggered grid (Common.py:634-690)."""

    def __init__(self, gpu_stream, nx, ny, halo_x, halo_y, h0, hu0, hv0):
        self.h0 = CUDAArray2D(gpu_stream, nx, ny, halo_x, halo_y, h0)
        self.hu0 = CUDAArray2D(gpu_stream, nx, ny, halo_x, halo_y, hu0)
        self.hv0 = CUDAArray2D(gpu_stream, nx, ny, halo_x, halo_y, hv0)
        self.h1 = CUDAArray2D(gpu_stream, nx, ny, halo_x, halo_y, h0)
        self.hu1 = CUDAArray2D(gpu_stream, nx, ny, halo_x, halo_y, hu0)
        self.hv1 = CUDAArray2D(gpu_stream, nx, ny, halo_x, halo_y, hv0)

    def swap(self):
        self.h1, self.h0 = self.h0, self.h1
        self.hu1, self.hu0 = self.hu0, self.hu1
        self.hv1, self.hv0 = self.hv0, self.hv1

    def download(self, gpu_stream):
        return self.h0.download(gpu_stream), self.hu0.download(gpu_stream), self.hv0.download(gpu_stream)

    def downloadPrevTimestep(self, gpu_stream):
        return self.h1.download(gpu_stream), self.hu1.download(gpu_stream), self.hv1.download(gpu_stream)

    def release(self):
        for a in (self.h0, self.hu0, self.hv0, self.h1, self.hu1, self.hv1):
            a.release()


class BoundaryConditions:
    """Boundary codes per side (Common.py:824-946): 1 wall, 2 periodic,
    3 flow relaxation, 4 linear interpolation."""

    def __init__(self, north=1, east=1, south=1, west=1,
                 spongeCells={'north': 0, 'south': 0, 'east': 0, 'west': 0}):
        self.north = np.int32(north)
        self.east = np.int32(east)
        self.south = np.int32(south)
        self.west = np.int32(west)
        self.spongeCells = dict(spongeCells)
        for key in self.spongeCells.keys():
            self.spongeCells[key] = np.int32(self.spongeCells[key])
        assert not ((self.north == 2 or self.south == 2) and (self.north != self.south)), \
            'The given periodic boundary conditions are not periodically (north/south)'
        assert not ((self.east == 2 or self.west == 2) and (self.east != self.west)), \
            'The given periodic boundary conditions are not periodically (east/west)'

    def get(self):
        raise NotImplementedError("get() implementation changed! Change calling code")

    def getSponge(self):
        return self.spongeCells

    def isDefault(self):
        return self.north == 1 and self.east == 1 and self.south == 1 and self.east == 1

    def isSponge(self):
        return any(b in (3, 4) for b in (self.north, self.east, self.south, self.west))

    def isPeriodicNorthSouth(self):
        return self.north == 2 and self.south == 2

    def isPeriodicEastWest(self):
        return self.east == 2 and self.west == 2

    def _toString(self, cond):
        return {1: "Wall", 2: "Periodic", 3: "Flow_Relaxation_Scheme",
                4: "Open_Linear_Interpolation"}.get(int(cond), "Invalid_:|")

    def __str__(self):
        # plain ints in the sponge dict, so the string reads back with
        # fromstring (NumPy 2 would print np.int32(..))
        sponge = {k: int(v) for k, v in self.spongeCells.items()}
        return ("north: " + self._toString(self.north) + ", east: " + self._toString(self.east) +
                ", south: " + self._toString(self.south) + ", west: " + self._toString(self.west) +
                ", spongeCells: " + str(sponge))

    @classmethod
    def fromstring(cls, bc_string):
        """Inverse of __str__, the form SimWriter stores in NetCDF files
        (Common.py:908-946): four side keywords, then the sponge widths as
        a dict or as four numbers in north, east, south, west order."""
        codes = {"Wall": 1, "Periodic": 2, "Flow_Relaxation_Scheme": 3, "Open_Linear_Interpolation": 4}
        words = [w for w in re.split(r"[\s,:{}\[\]']+", str(bc_string)) if w]
        sides = [codes.get(words[k], -1) for k in (1, 3, 5, 7)]
        rest = words[9:]
        if len(rest) >= 8:
            sponge = {rest[k]: int(rest[k + 1]) for k in range(0, 8, 2)}
        else:
            sponge = dict(zip(("north", "east", "south", "west"), (int(w) for w in rest[:4])))
        return cls(*sides, spongeCells=sponge)

    def codes(self):
        return (int(self.north), int(self.east), int(self.south), int(self.west))


class SingleBoundaryConditionData:
    """External solution on one side (Common.py:949-978)."""

    def __init__(self, h=None, hu=None, hv=None):
        self.h = [np.zeros((1, 2), dtype=np.float32)]
        self.hu = [np.zeros((1, 2), dtype=np.float32)]
        self.hv = [np.zeros((1, 2), dtype=np.float32)]
        self.numSteps = 1
        self.shape = self.h[0].shape
        if h is not None:
            self.shape = h[0].shape
            self.numSteps = len(h)
            self.h, self.hu, self.hv = h, hu, hv


class BoundaryConditionsData:
    """External solutions for the sponge boundaries (Common.py:980-1014)."""

    def __init__(self, t=None, north=None, south=None, east=None, west=None):
        self.t = [0] if t is None else t
        self.numSteps = len(self.t)
        self.north = north or SingleBoundaryConditionData()
        self.south = south or SingleBoundaryConditionData()
        self.east = east or SingleBoundaryConditionData()
        self.west = west or SingleBoundaryConditionData()


class BoundaryConditionsArakawaA:
    """Ghost-cell refresh for unstaggered grids (Common.py:1019-1309): north-
    south first, then east-west; per axis the periodic copy, or the open
    kinds of its two sides (3: flow relaxation towards the exterior solution
    in ``bc_data``, 4: linear interpolation over the sponge).  Wall sides are
    mirrored inside the step kernel and need no launch here.  With open
    boundaries the simulator's own step domain is attached (``use_domain``)
    so that its RK stages apply the same sequence."""

    def __init__(self, gpu_ctx, nx, ny, halo_x, halo_y, boundary_conditions,
                 bc_data=None, block_width=16, block_height=16):
        self.boundary_conditions = boundary_conditions
        self.nx, self.ny = np.int32(nx), np.int32(ny)
        self.halo_x, self.halo_y = np.int32(halo_x), np.int32(halo_y)
        self.bc_data = bc_data if bc_data is not None else BoundaryConditionsData()
        self._domain = _native.Domain(nx, ny, 1.0, 1.0, 1.0, bc=boundary_conditions.codes())
        self._domains = [self._domain]
        self.bc_timestamps = [None, None]
        self.bc_t = np.float32(0.0)
        self._textures = None
        if boundary_conditions.isSponge():
            sp = boundary_conditions.getSponge()
            self._domain.set_sponge(sp["north"], sp["east"], sp["south"], sp["west"])

    def use_domain(self, domain):
        """Also keep `domain` (the simulator's step domain) up to date with
        the sponge widths and the exterior solution."""
        if self.boundary_conditions.isSponge():
            sp = self.boundary_conditions.getSponge()
            domain.set_sponge(sp["north"], sp["east"], sp["south"], sp["west"])
            if self._textures is not None:
                domain.set_open_bc(self._textures, self.bc_t)
        self._domains.append(domain)

    def _relaxes(self):
        bc = self.boundary_conditions
        return 3 in (int(bc.north), int(bc.south), int(bc.east), int(bc.west))

    @staticmethod
    def _pack(side_a, side_b, t_index, along_x):
        """Texels (h, hu, hv, 0) of two sides at one time: rows (south,
        north) of one texel per column, or columns (west, east) of one texel
        per row (Common.py:1105-1137)."""
        def rgba(side):
            h = np.squeeze(side.h[t_index])
            hu = np.squeeze(side.hu[t_index])
            hv = np.squeeze(side.hv[t_index])
            if h.ndim != 1:
                raise ValueError("boundary data of a side must be one row or column")
            return np.stack([h, hu, hv, np.zeros_like(h)], axis=1).astype(np.float32)
        a, b = rgba(side_a), rgba(side_b)
        if along_x:
            return np.ascontiguousarray(np.stack([a, b], axis=0))      # 2 x L x 4
        return np.ascontiguousarray(np.stack([a, b], axis=1))          # L x 2 x 4

    def update_bc_values(self, gpu_stream, t):
        """Exterior solution of the interval around t as textures (rebuilt
        when the interval changes) and the time weight of this step
        (Common.py:1073-1216)."""
        if not self._relaxes():
            return
        d = self.bc_data
        t1_index = min(len(d.t) - 1, int(np.searchsorted(d.t, t)))
        t0_index = max(0, int(np.searchsorted(d.t, t)) - 1)
        new_t0, new_t1 = d.t[t0_index], d.t[t1_index]
        if [new_t0, new_t1] != self.bc_timestamps or self._textures is None:
            lib = _native.load()
            handles = []
            for k in (t0_index, t1_index):
                for along_x, (a, b) in ((True, (d.south, d.north)), (False, (d.west, d.east))):
                    texels = self._pack(a, b, k, along_x)
                    h = ctypes.c_uint64(0)
                    _native.check(lib.go_bc_texture_create(texels.ctypes.data_as(ctypes.c_void_p),
                                                           int(texels.shape[1]), int(texels.shape[0]),
                                                           ctypes.byref(h)))
                    handles.append(h.value)
            # order: NS current, NS next, EW current, EW next
            new = (handles[0], handles[2], handles[1], handles[3])
            if gpu_stream is not None:
                gpu_stream.synchronize()
            self._release()
            self._textures = new
            self.bc_timestamps = [new_t0, new_t1]
        interval = max(1.0e-10, new_t1 - new_t0)
        self.bc_t = np.float32(max(0.0, min(1.0, (t - new_t0) / interval)))
        for dom in self._domains:
            dom.set_open_bc(self._textures, self.bc_t)

    def _release(self):
        if self._textures is not None:
            lib = _native.load()
            for h in self._textures:
                lib.go_wind_texture_destroy(ctypes.c_uint64(h))
            self._textures = None

    def __del__(self):
        try:
            self._release()
        except Exception:
            pass

    def boundaryCondition(self, gpu_stream, h, u, v):
        assert h.pitch == u.pitch == v.pitch
        _native.check(_native.load().go_boundary_condition(
            self._domain.handle, _native.stream_handle(gpu_stream),
            _native.ptr(h.tensor), _native.ptr(u.tensor), _native.ptr(v.tensor), int(h.pitch)))


class Bathymetry:
    """Corner bathymetry Bi and cell bathymetry Bm (Common.py:1313-1459)."""

    def __init__(self, gpu_ctx, gpu_stream, nx, ny, halo_x, halo_y, Bi_host,
                 boundary_conditions=None, block_width=16, block_height=16):
        if boundary_conditions is None:
            boundary_conditions = BoundaryConditions()
        self.gpu_stream = gpu_stream
        self.nx, self.ny = np.int32(nx), np.int32(ny)
        self.halo_x, self.halo_y = np.int32(halo_x), np.int32(halo_y)
        self.halo_nx = np.int32(nx + 2 * halo_x)
        self.halo_ny = np.int32(ny + 2 * halo_y)
        self.boundary_conditions = boundary_conditions
        self.mask_value = np.float32(1.0e20)
        self.use_mask = False
        if np.ma.is_masked(Bi_host):
            Bi_host = Bi_host.copy().filled(self.mask_value).astype(np.float32)
            self.use_mask = True
        BiShapeY, BiShapeX = Bi_host.shape
        assert BiShapeX == nx + 1 + 2 * halo_x and BiShapeY == ny + 1 + 2 * halo_y, \
            "Wrong size of bottom bathymetry, should be defined on cell intersections, not cell centers. " + \
            str((BiShapeX, BiShapeY)) + " vs " + str((nx + 1 + 2 * halo_x, ny + 1 + 2 * halo_y))
        self.Bi = CUDAArray2D(gpu_stream, nx + 1, ny + 1, halo_x, halo_y, Bi_host)
        Bm_host = np.zeros((self.halo_ny, self.halo_nx), dtype=np.float32)
        self.Bm = CUDAArray2D(gpu_stream, nx, ny, halo_x, halo_y, Bm_host)
        codes = boundary_conditions.codes()
        codes = tuple(c if c in (1, 2) else 1 for c in codes)
        self._domain = _native.Domain(nx, ny, 1.0, 1.0, 1.0, bc=codes)
        _native.check(_native.load().go_init_bathymetry(
            self._domain.handle, _native.stream_handle(gpu_stream),
            _native.ptr(self.Bi.tensor), int(self.Bi.pitch),
            _native.ptr(self.Bm.tensor), int(self.Bm.pitch), float(self.mask_value)))

    def download(self, gpu_stream):
        Bm_cpu = self.Bm.download(gpu_stream)
        Bi_cpu = self.Bi.download(gpu_stream)
        if self.use_mask:
            Bi_cpu = np.ma.array(data=Bi_cpu, mask=(Bi_cpu == self.mask_value), fill_value=0.0)
            Bm_cpu = np.ma.array(data=Bm_cpu, mask=(Bm_cpu == self.mask_value), fill_value=0.0)
        return Bi_cpu, Bm_cpu

    def release(self):
        self.Bm.release()
        self.Bi.release()
