"""Drifters on the GPU (gpu_ocean/SWESimulators/GPUDrifterCollection.py).

Positions live in a device array of (numDrifters + 1) rows of (x, y)
float32, the last row the observation's position.  ``drift`` advances every
row one Euler step with the flow velocity interpolated bilinearly between
cell centres (plus optional wind drift) through ``go_drift_passive``; the
simulator calls it after every time step once the collection is attached
(``CDKLM16.attachDrifters``).  ``observeUnderlyingFlow`` samples (hu, hv)
under each drifter (the observation operator of the reference's
ensembles, ``go_observe_flow``).
"""

import ctypes

import numpy as np

from . import Common, WindStress, _native
from .BaseDrifterCollection import BaseDrifterCollection


class GPUDrifterCollection(BaseDrifterCollection):

    def __init__(self, gpu_ctx, numDrifters, observation_variance=0.01, wind=None, wind_drift_factor=0.0,
                 boundaryConditions=None, initialization_cov_drifters=None, domain_size_x=1.0,
                 domain_size_y=1.0, gpu_stream=None, block_width=64):
        super(GPUDrifterCollection, self).__init__(
            numDrifters, observation_variance=observation_variance,
            boundaryConditions=boundaryConditions if boundaryConditions is not None else Common.BoundaryConditions(),
            domain_size_x=domain_size_x, domain_size_y=domain_size_y)
        torch = _native.require_cuda()
        self.gpu_ctx = gpu_ctx
        self.block_width = block_width
        self.block_height = 1
        self.wind = wind if wind is not None else WindStress.WindStress()
        self.wind_drift_factor = np.float32(wind_drift_factor)
        self.gpu_stream = gpu_stream if gpu_stream is not None else torch.cuda.Stream()
        self.sensitivity = 1.0
        self.driftersHost = np.zeros((self.getNumDrifters() + 1, 2), dtype=np.float32)
        self.driftersDevice = Common.CUDAArray2D(self.gpu_stream, 2, self.getNumDrifters() + 1, 0, 0,
                                                 self.driftersHost)
        self._wind_tex = None          # handles (X cur, X next, Y cur, Y next)
        self._wind_interval = None
        if self.wind_drift_factor:
            self.update_wind(0.0)
        self.uniformly_distribute_drifters(initialization_cov_drifters=initialization_cov_drifters)

    def copy(self):
        """An independent collection with the same positions, observation,
        boundary conditions and domain (GPUDrifterCollection.py:99-116)."""
        c = GPUDrifterCollection(self.gpu_ctx, self.getNumDrifters(),
                                 observation_variance=self.observation_variance,
                                 boundaryConditions=self.boundaryConditions,
                                 domain_size_x=self.domain_size_x, domain_size_y=self.domain_size_y,
                                 gpu_stream=self.gpu_stream, block_width=self.block_width)
        c.setDrifterPositions(self.getDrifterPositions())
        c.setObservationPosition(self.getObservationPosition())
        return c

    # -- wind drift ------------------------------------------------------------
    def update_wind(self, t):
        """Binds the wind interval around t as textures (rebuilt when the
        interval changes) and returns the time weight in [0, 1]
        (GPUDrifterCollection.py:120-190)."""
        times = self.wind.t
        t1 = min(len(times) - 1, int(np.searchsorted(times, t)))
        t0 = max(0, int(np.searchsorted(times, t)) - 1)
        interval = (times[t0], times[t1])
        if interval != self._wind_interval:
            self._release_wind()
            lib = _native.load()
            handles = []
            for field in (self.wind.X[t0], self.wind.X[t1], self.wind.Y[t0], self.wind.Y[t1]):
                a = np.ascontiguousarray(np.asarray(field, dtype=np.float32).reshape(np.shape(field)[-2:]))
                h = ctypes.c_uint64(0)
                _native.check(lib.go_wind_texture_create(a.ctypes.data_as(ctypes.c_void_p), int(a.shape[1]),
                                                         int(a.shape[0]), ctypes.byref(h)))
                handles.append(h.value)
            self._wind_tex = (ctypes.c_uint64 * 4)(*handles)
            self._wind_interval = interval
        span = max(1.0e-10, interval[1] - interval[0])
        return max(0.0, min(1.0, (t - interval[0]) / span))

    def _release_wind(self):
        if self._wind_tex is not None:
            lib = _native.load()
            self.gpu_stream.synchronize()
            for h in self._wind_tex:
                lib.go_wind_texture_destroy(ctypes.c_uint64(h))
            self._wind_tex = None
            self._wind_interval = None

    def cleanUp(self):
        if getattr(self, "_wind_tex", None) is not None:
            self._release_wind()

    # -- positions ---------------------------------------------------------------
    def setDrifterPositions(self, newDrifterPositions):
        rows = np.concatenate((np.asarray(newDrifterPositions, dtype=np.float64).reshape(-1, 2),
                               np.array([self.getObservationPosition()], dtype=np.float64)), axis=0)
        self.driftersDevice.upload(self.gpu_stream, rows.astype(np.float32))

    def setObservationPosition(self, newObservationPosition):
        rows = np.concatenate((np.asarray(self.getDrifterPositions(), dtype=np.float64),
                               np.asarray(newObservationPosition, dtype=np.float64).reshape(1, 2)), axis=0)
        self.driftersDevice.upload(self.gpu_stream, rows.astype(np.float32))

    def setSensitivity(self, sensitivity):
        self.sensitivity = sensitivity

    def getDrifterPositions(self):
        return self.driftersDevice.download(self.gpu_stream)[:-1, :]

    def getObservationPosition(self):
        return self.driftersDevice.download(self.gpu_stream)[self.obs_index, :]

    def setGPUStream(self, gpu_stream):
        self.gpu_stream = gpu_stream

    # -- device work ---------------------------------------------------------------
    def drift(self, eta, hu, hv, Hm, nx, ny, t, dx, dy, dt, x_zero_ref, y_zero_ref):
        """One Euler step of every drifter and the observation through the
        flow (eta, hu, hv with cell depths Hm, CUDAArray2D of the
        ghost-inclusive grid), x_zero_ref/y_zero_ref the ghost-inclusive
        cell of the origin (2 for CDKLM16) (GPUDrifterCollection.py:209-232)."""
        wind_t = np.float32(self.update_wind(t)) if self.wind_drift_factor else np.float32(0.0)
        bc = self.boundaryConditions
        P = _native.ptr
        _native.check(_native.load().go_drift_passive(
            _native.stream_handle(self.gpu_stream), int(nx), int(ny), float(dx), float(dy), float(dt),
            int(x_zero_ref), int(y_zero_ref), P(eta.tensor), int(eta.pitch), P(hu.tensor), int(hu.pitch),
            P(hv.tensor), int(hv.pitch), P(Hm.tensor), int(Hm.pitch), int(bc.isPeriodicNorthSouth()),
            int(bc.isPeriodicEastWest()), self.getNumDrifters(), P(self.driftersDevice.tensor),
            int(self.driftersDevice.pitch), float(np.float32(self.sensitivity)), float(wind_t),
            float(self.wind_drift_factor), self._wind_tex if self.wind_drift_factor else None))

    def enforceBoundaryConditions(self):
        """Periodic wrap of every position on the device
        (GPUDrifterCollection.py:236-248)."""
        bc = self.boundaryConditions
        if not (bc.isPeriodicNorthSouth() or bc.isPeriodicEastWest()):
            return
        _native.check(_native.load().go_drift_enforce_bc(
            _native.stream_handle(self.gpu_stream), float(self.domain_size_x), float(self.domain_size_y),
            int(bc.isPeriodicNorthSouth()), int(bc.isPeriodicEastWest()), self.getNumDrifters(),
            _native.ptr(self.driftersDevice.tensor), int(self.driftersDevice.pitch)))

    def observeUnderlyingFlow(self, hu, hv, nx, ny, dx, dy, x_zero_ref=2, y_zero_ref=2):
        """(hu, hv) of the cell under each drifter, numDrifters x 2 numpy
        (observeUnderlyingFlow, observationKernels.cu:29-81, as the
        reference's ensembles call it, BaseOceanStateEnsemble.py:110-125)."""
        torch = _native.require_cuda()
        n = self.getNumDrifters()
        out = torch.empty((max(n, 1), 2), dtype=torch.float32, device="cuda")
        _native.check(_native.load().go_observe_flow(
            _native.stream_handle(self.gpu_stream), int(nx), int(ny), float(dx), float(dy), int(x_zero_ref),
            int(y_zero_ref), _native.ptr(hu.tensor), int(hu.pitch), _native.ptr(hv.tensor), int(hv.pitch), n,
            _native.ptr(self.driftersDevice.tensor), int(self.driftersDevice.pitch), _native.ptr(out), 8))
        self.gpu_stream.synchronize()
        return out[:n].cpu().numpy()
