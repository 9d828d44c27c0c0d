"""Base class of the simulators, gpu_ocean/SWESimulators/Simulator.py:43-349.

Keeps the reference's attributes (float32 scalars as the kernels see them,
``gpu_stream``, ``t``, ``num_iterations``) and methods (``download``,
``downloadPrevTimestep``, ``copyState``, ``upload``, ``attachDrifters``,
``update_wind_stress``).  ``gpu_stream`` is a ``torch.cuda.Stream``.
"""

import logging

import numpy as np

from . import _native
from .WindStress import sample_at_cells


class Simulator(object):

    def __init__(self, gpu_ctx, nx, ny, ghost_cells_x, ghost_cells_y, dx, dy, dt, g, f, r, A,
                 t, theta, rk_order, coriolis_beta, y_zero_reference_cell, wind_stress,
                 write_netcdf, ignore_ghostcells, offset_x, offset_y, comm,
                 block_width, block_height, local_particle_id=0):
        torch = _native.require_cuda()
        self.gpu_stream = torch.cuda.Stream()
        self.logger = logging.getLogger(__name__)
        self.gpu_ctx = gpu_ctx
        self.nx = np.int32(nx)
        self.ny = np.int32(ny)
        self.ghost_cells_x = np.int32(ghost_cells_x)
        self.ghost_cells_y = np.int32(ghost_cells_y)
        self.dx = np.float32(dx)
        self.dy = np.float32(dy)
        self.dt = dt
        self.g = np.float32(g)
        self.f = np.float32(f)
        self.r = np.float32(r)
        self.coriolis_beta = np.float32(coriolis_beta)
        self.wind_stress = wind_stress
        self.y_zero_reference_cell = np.float32(y_zero_reference_cell)
        self.offset_x = offset_x
        self.offset_y = offset_y
        self.t = t
        self.num_iterations = 0
        self.wind_stress_timestamps = {}
        self.A = 'NA' if A is None else np.float32(A)
        self.theta = 'NA' if theta is None else np.float32(theta)
        self.rk_order = 'NA' if rk_order is None else np.int32(rk_order)
        self.hasDrifters = False
        self.drifters = None
        self.write_netcdf = write_netcdf
        self.ignore_ghostcells = ignore_ghostcells
        self.sim_writer = None
        self.comm = comm
        self.local_particle_id = local_particle_id
        self.local_size = (block_width, block_height, 1)
        self.global_size = (int(np.ceil(self.nx / float(block_width))),
                            int(np.ceil(self.ny / float(block_height))))
        self._wind_field_tensors = None

    # -- wind (Simulator.py:145-223) ---------------------------------------
    def _wind_interval(self):
        ws = self.wind_stress
        t_max_index = len(ws.t) - 1
        t0_index = max(0, np.searchsorted(ws.t, self.t) - 1)
        t1_index = min(t_max_index, np.searchsorted(ws.t, self.t))
        return t0_index, t1_index

    def update_wind_stress(self, domain=None):
        """Selects the wind interval around ``self.t``, hands the current and
        next wind to the kernel and returns the time-interpolation weight."""
        domain = domain if domain is not None else self._domain
        ws = self.wind_stress
        t0_index, t1_index = self._wind_interval()
        new_t0, new_t1 = ws.t[t0_index], ws.t[t1_index]
        old = self.wind_stress_timestamps.get("cdklm")
        if old != [new_t0, new_t1]:
            self.wind_stress_timestamps["cdklm"] = [new_t0, new_t1]
            if ws.is_uniform():
                domain.set_wind_uniform(np.asarray(ws.X[t0_index]).reshape(-1)[0],
                                        np.asarray(ws.X[t1_index]).reshape(-1)[0],
                                        np.asarray(ws.Y[t0_index]).reshape(-1)[0],
                                        np.asarray(ws.Y[t1_index]).reshape(-1)[0])
            else:
                tens = [sample_at_cells(a, int(self.nx), int(self.ny), self.gpu_stream)
                        for a in (ws.X[t0_index], ws.X[t1_index], ws.Y[t0_index], ws.Y[t1_index])]
                self._wind_field_tensors = tens
                domain.set_wind_field(*tens)
        elapsed_since_t0 = (self.t - new_t0)
        time_interval = max(1.0e-10, (new_t1 - new_t0))
        return max(0.0, min(1.0, elapsed_since_t0 / time_interval))

    # -- state access -------------------------------------------------------
    def attachDrifters(self, drifters):
        self.drifters = drifters
        self.hasDrifters = True
        if hasattr(self.drifters, "setGPUStream"):
            self.drifters.setGPUStream(self.gpu_stream)
        self.drifter_t = 0.0

    def download(self, interior_domain_only=False):
        eta, hu, hv = self.gpu_data.download(self.gpu_stream)
        if interior_domain_only:
            idx = self.interior_domain_indices
            return (eta[idx[2]:idx[0], idx[3]:idx[1]],
                    hu[idx[2]:idx[0], idx[3]:idx[1]],
                    hv[idx[2]:idx[0], idx[3]:idx[1]])
        return eta, hu, hv

    def downloadPrevTimestep(self):
        return self.gpu_data.downloadPrevTimestep(self.gpu_stream)

    def copyState(self, otherSim):
        assert type(otherSim) is type(self), "A simulator can only copy the state from another simulator of the same class."
        assert (self.ny, self.nx) == (otherSim.ny, otherSim.nx), "Simulators differ in computational domain."
        otherSim.gpu_stream.synchronize()
        for dst, src in ((self.gpu_data.h0, otherSim.gpu_data.h0), (self.gpu_data.hu0, otherSim.gpu_data.hu0),
                         (self.gpu_data.hv0, otherSim.gpu_data.hv0), (self.gpu_data.h1, otherSim.gpu_data.h1),
                         (self.gpu_data.hu1, otherSim.gpu_data.hu1), (self.gpu_data.hv1, otherSim.gpu_data.hv1)):
            dst.copyBuffer(self.gpu_stream, src)
        self.wind_stress = otherSim.wind_stress
        self.wind_stress_timestamps = {}
        if otherSim.hasDrifters and self.hasDrifters:
            self.drifters.setDrifterPositions(otherSim.drifters.getDrifterPositions())
            self.drifters.setObservationPosition(otherSim.drifters.getObservationPosition())

    def upload(self, eta0, hu0, hv0, eta1=None, hu1=None, hv1=None):
        """Sets the state (Simulator.py:upload of the reference).  Without a
        separate second state, the second buffers get a device-side copy of
        the first instead of a second host-to-device transfer of the same
        arrays (same contents, half the bus traffic)."""
        self.gpu_data.h0.upload(self.gpu_stream, eta0)
        self.gpu_data.hu0.upload(self.gpu_stream, hu0)
        self.gpu_data.hv0.upload(self.gpu_stream, hv0)
        if eta1 is None:
            for dst, src in ((self.gpu_data.h1, self.gpu_data.h0), (self.gpu_data.hu1, self.gpu_data.hu0),
                             (self.gpu_data.hv1, self.gpu_data.hv0)):
                dst.copyBuffer(self.gpu_stream, src)
                dst.mask = src.mask
        else:
            self.gpu_data.h1.upload(self.gpu_stream, eta1)
            self.gpu_data.hu1.upload(self.gpu_stream, hu1)
            self.gpu_data.hv1.upload(self.gpu_stream, hv1)

    def closeNetCDF(self):
        if self.write_netcdf and self.sim_writer is not None:
            self.sim_writer.__exit__(0, 0, 0)
            self.write_netcdf = False

    def __del__(self):
        try:
            self.cleanUp()
        except Exception:
            pass

    def cleanUp(self):
        pass
