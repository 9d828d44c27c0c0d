"""CDKLM16 simulator on the B200-native kernels.

Drop-in for gpu_ocean/SWESimulators/CDKLM16.py:44-794: same constructor
(CDKLM16.py:49-85), same ``step`` loop semantics (CDKLM16.py:494-598),
``updateDt`` (:712-739), ``dataAssimilationStep`` (:650-704) and the
attributes other modules read (``gpu_data.h0 ...``, ``bathymetry``,
``gpu_stream``, ``t``, ``num_iterations``, ...).

What is not built raises ``NotImplementedError`` at construction:
a spatially varying grid angle, ``latitude``, ``rk_order`` other than 2.
The stochastic model error (``small_scale_perturbation``) runs on
OceanStateNoise after each step; NetCDF output (``write_netcdf``) and
``fromfilename`` use SimWriter and SimReader.
The Coriolis table is always full-resolution
(``subsample_f``/``subsample_angle`` are accepted and ignored; the
reference's subsampler calls ``scipy.interpolate.interp2d``, which the
installed SciPy no longer provides).
"""

import logging

import numpy as np

from . import Common, OceanStateNoise, SimReader, Simulator, SimWriter, WindStress, _native


class CDKLM16(Simulator.Simulator):

    def __init__(self, gpu_ctx, eta0, hu0, hv0, H, nx, ny, dx, dy, dt, g, f, r,
                 subsample_f=10, angle=np.array([[0]], dtype=np.float32), subsample_angle=10,
                 latitude=None, t=0.0, theta=1.3, rk_order=2, coriolis_beta=0.0,
                 max_wind_direction_perturbation=0, wind_stress=WindStress.WindStress(),
                 boundary_conditions=Common.BoundaryConditions(),
                 boundary_conditions_data=Common.BoundaryConditionsData(),
                 small_scale_perturbation=False, small_scale_perturbation_amplitude=None,
                 small_scale_perturbation_interpolation_factor=1, model_time_step=None,
                 reportGeostrophicEquilibrium=False, use_lcg=False, xorwow_seed=None,
                 write_netcdf=False, comm=None, local_particle_id=0, super_dir_name=None,
                 netcdf_filename=None, ignore_ghostcells=False, courant_number=0.8,
                 offset_x=0, offset_y=0, flux_slope_eps=1.0e-1, desingularization_eps=1.0e-1,
                 depth_cutoff=1.0e-5, block_width=12, block_height=32, num_threads_dt=256,
                 block_width_model_error=16, block_height_model_error=16,
                 linear_friction=False):
        self.logger = logging.getLogger(__name__)
        if rk_order != 2:
            raise NotImplementedError("only rk_order=2 (Heun) is built")
        if latitude is not None:
            raise NotImplementedError("a latitude field (2-D Coriolis) is not built")
        angle = np.asarray(angle)
        if angle.size != 1 and not np.all(angle == angle.reshape(-1)[0]):
            raise NotImplementedError("a spatially varying grid angle is not built")

        ghost_cells_x = 2
        ghost_cells_y = 2
        x_zero_reference_cell = ghost_cells_x
        y_zero_reference_cell = ghost_cells_y
        self.boundary_conditions = boundary_conditions

        # CDKLM16.py:146-148 -- f compensated to the first interior cell
        a0 = float(angle.reshape(-1)[0])
        self._angle0 = np.float32(a0)
        north = np.array([np.sin(a0), np.cos(a0)])
        f = f - coriolis_beta * (x_zero_reference_cell * dx * north[0] + y_zero_reference_cell * dy * north[1])
        x_zero_reference_cell = 0
        y_zero_reference_cell = 0

        self.max_wind_direction_perturbation = max_wind_direction_perturbation
        super(CDKLM16, self).__init__(gpu_ctx, nx, ny, ghost_cells_x, ghost_cells_y, dx, dy, dt, g, f, r, None,
                                      t, theta, rk_order, coriolis_beta, y_zero_reference_cell, wind_stress,
                                      write_netcdf, ignore_ghostcells, offset_x, offset_y, comm,
                                      block_width, block_height, local_particle_id=local_particle_id)
        self.interior_domain_indices = np.array([-2, -2, 2, 2])
        self.linear_friction = bool(linear_friction)

        self._domain = _native.Domain(
            nx, ny, self.dx, self.dy, self.g, self.r, theta=self.theta,
            desing_eps=desingularization_eps, flux_slope_eps=flux_slope_eps, depth_cutoff=depth_cutoff,
            bc=boundary_conditions.codes(),
            friction_law=_native.GO_FRICTION_LINEAR if linear_friction else _native.GO_FRICTION_QUADRATIC,
            # the kernel's north vector: sinf/cosf of the float angle on the
            # device, as the reference's getNorth (CDKLM16_kernel.cu:68-77)
            north=_native.north_vector(np.float32(a0)) if a0 != 0.0 else (np.float32(0.0), np.float32(1.0)))

        self.bathymetry = Common.Bathymetry(gpu_ctx, self.gpu_stream, nx, ny, ghost_cells_x, ghost_cells_y,
                                            H, boundary_conditions)
        # land tests of the kernel only when the bathymetry holds land
        Hh = np.ma.filled(H, self.bathymetry.mask_value) if np.ma.is_masked(H) else np.asarray(H)
        self._domain.set_land(bool(np.any(np.abs(Hh.astype(np.float32) - self.bathymetry.mask_value) < 1e-3)))
        Hm = self.downloadBathymetry()[1]
        eta0 = np.maximum(eta0, -Hm)          # CDKLM16.py:237-238
        self.gpu_data = Common.SWEDataArakawaA(self.gpu_stream, nx, ny, ghost_cells_x, ghost_cells_y,
                                               eta0, hu0, hv0)
        torch = _native.require_cuda()
        self._dt_dev = torch.zeros(4, dtype=torch.float32, device="cuda")
        self.courant_number = courant_number
        self.num_threads_dt = num_threads_dt
        self.reportGeostrophicEquilibrium = np.int32(reportGeostrophicEquilibrium)
        self.constant_equilibrium_depth = np.max(H)
        self.bc_kernel = Common.BoundaryConditionsArakawaA(gpu_ctx, self.nx, self.ny, ghost_cells_x,
                                                           ghost_cells_y, self.boundary_conditions,
                                                           boundary_conditions_data)
        # open boundaries: the step domain runs the ghost sequence after each stage
        self.bc_kernel.use_domain(self._domain)

        # Coriolis per ghost-inclusive row (CDKLM16.py:310-345), full resolution
        self.coriolis_rows = self._coriolis_rows(eta0, angle, a0)
        self._domain.set_coriolis(self.coriolis_rows)

        # stochastic model error (CDKLM16.py:355-367)
        self.small_scale_perturbation = small_scale_perturbation
        self.small_scale_model_error = None
        self.small_scale_perturbation_interpolation_factor = small_scale_perturbation_interpolation_factor
        if small_scale_perturbation:
            self.small_scale_model_error = OceanStateNoise.OceanStateNoise.fromsim(
                self, soar_q0=small_scale_perturbation_amplitude,
                interpolation_factor=small_scale_perturbation_interpolation_factor, use_lcg=use_lcg,
                xorwow_seed=xorwow_seed, block_width=block_width_model_error,
                block_height=block_height_model_error)
        self.model_time_step = model_time_step
        self.total_time_steps = 0
        if model_time_step is None:
            self.model_time_step = self.dt
        # NetCDF output, the initial state as the first record (CDKLM16.py:375-377)
        if self.write_netcdf:
            self.sim_writer = SimWriter.SimNetCDFWriter(self, super_dir_name=super_dir_name,
                                                        filename=netcdf_filename,
                                                        ignore_ghostcells=self.ignore_ghostcells,
                                                        offset_x=self.offset_x, offset_y=self.offset_y)
        if self.dt <= 0:
            self.updateDt()

    def _coriolis_rows(self, eta0, angle, a0):
        nyh = int(self.ny) + 4
        if self.coriolis_beta != 0.0:
            if angle.size != 1:
                raise RuntimeError("non-constant angle cannot be combined with beta plane model (makes no sense)")
            x = np.linspace((-self.ghost_cells_x + 0.5) * self.dx, (self.nx + self.ghost_cells_x - 0.5) * self.dx,
                            self.nx + 2 * self.ghost_cells_x)
            y = np.linspace((-self.ghost_cells_y + 0.5) * self.dy, (self.ny + self.ghost_cells_y - 0.5) * self.dy,
                            self.ny + 2 * self.ghost_cells_x)
            x, y = np.meshgrid(x, y)
            n = x * np.sin(a0) + y * np.cos(a0)
            coriolis_f = (self.f + self.coriolis_beta * n).astype(np.float32)
        else:
            fa = np.asarray(self.f)
            if fa.size == 1:
                return np.full(nyh, np.float32(fa.reshape(-1)[0]), dtype=np.float32)
            if fa.shape == np.asarray(eta0).shape:
                coriolis_f = fa.astype(np.float32)
            else:
                raise RuntimeError("The shape of f should match up with eta or be scalar.")
        if not np.all(coriolis_f == coriolis_f[:, :1]):
            raise NotImplementedError("a Coriolis field that varies along x is not built")
        return np.ascontiguousarray(coriolis_f[:, 0])

    def cleanUp(self):
        if getattr(self, "sim_writer", None) is not None:
            self.closeNetCDF()
        if getattr(self, "gpu_data", None) is not None:
            self.gpu_data.release()
        if getattr(self, "bathymetry", None) is not None:
            self.bathymetry.release()
        if getattr(self, "small_scale_model_error", None) is not None:
            self.small_scale_model_error.cleanUp()
        self.gpu_ctx = None

    @classmethod
    def fromfilename(cls, gpu_ctx, filename, cont_write_netcdf=True, use_lcg=False, xorwow_seed=None,
                     new_netcdf_filename=None, time0=None):
        """A simulator hot-started from the last record (or the record at
        time0) of a NetCDF file written by SimWriter (CDKLM16.py:411-490):
        the file's parameters, bathymetry, boundary conditions and state.
        As in the reference, the wind is not restored (the file names only
        its source) and the Coriolis parameter read back is the one the
        writer stored, which the constructor shifts again for a beta plane."""
        sim_reader = SimReader.SimNetCDFReader(filename, ignore_ghostcells=False)
        try:
            sim_name = str(sim_reader.get("simulator_short"))
            assert sim_name == cls.__name__, \
                "Trying to initialize a " + cls.__name__ + " simulator with netCDF file based on " + sim_name + \
                " results."
            H = sim_reader.getH()
            if time0 is None:
                eta0, hu0, hv0, time0 = sim_reader.getLastTimeStep()
            else:
                eta0, hu0, hv0, time0 = sim_reader.getStateAtTime(time0)
            if len(H.shape) == 3:
                H = H[0, :, :]
            sim_params = {
                "gpu_ctx": gpu_ctx, "eta0": eta0, "hu0": hu0, "hv0": hv0, "H": H,
                "nx": int(sim_reader.get("nx")), "ny": int(sim_reader.get("ny")),
                "dx": sim_reader.get("dx"), "dy": sim_reader.get("dy"), "dt": sim_reader.get("dt"),
                "g": sim_reader.get("g"), "f": sim_reader.get("coriolis_force"),
                "r": sim_reader.get("bottom_friction_r"), "t": float(time0),
                "theta": sim_reader.get("minmod_theta"), "rk_order": int(sim_reader.get("time_integrator")),
                "coriolis_beta": sim_reader.get("coriolis_beta"), "write_netcdf": cont_write_netcdf,
                "use_lcg": use_lcg, "xorwow_seed": xorwow_seed, "netcdf_filename": new_netcdf_filename,
            }
            wind_type = sim_reader.get("wind_stress_type")
            sim_params["wind_stress"] = WindStress.WindStress()
            if wind_type != "not found":
                raise NotImplementedError("wind_stress_type %s: typed wind parameters are not built" % wind_type)
            sim_params["boundary_conditions"] = sim_reader.getBC()
            if sim_reader.has("small_scale_perturbation"):
                sim_params["small_scale_perturbation"] = sim_reader.get("small_scale_perturbation") == "True"
                if sim_params["small_scale_perturbation"]:
                    sim_params["small_scale_perturbation_amplitude"] = \
                        sim_reader.get("small_scale_perturbation_amplitude")
                    sim_params["small_scale_perturbation_interpolation_factor"] = \
                        int(sim_reader.get("small_scale_perturbation_interpolation_factor"))
            if sim_reader.has("model_time_step"):
                sim_params["model_time_step"] = sim_reader.get("model_time_step")
        finally:
            sim_reader.close()
        return cls(**sim_params)

    # -- stepping -----------------------------------------------------------
    def _launch_steps(self, n, dt, wind_t):
        g = self.gpu_data
        _native.check(_native.load().go_cdklm_step(
            self._domain.handle, _native.stream_handle(self.gpu_stream), int(n), float(dt), float(wind_t),
            _native.ptr(g.h0.tensor), _native.ptr(g.hu0.tensor), _native.ptr(g.hv0.tensor), int(g.h0.pitch),
            _native.ptr(g.h1.tensor), _native.ptr(g.hu1.tensor), _native.ptr(g.hv1.tensor), int(g.h1.pitch),
            _native.ptr(self.bathymetry.Bi.tensor), int(self.bathymetry.Bi.pitch),
            float(self.bathymetry.mask_value)))

    def step(self, t_end=0.0, apply_stochastic_term=True, write_now=True, update_dt=False):
        """Advance by t_end seconds in steps of self.dt; the last step is
        shortened to land on t_end (CDKLM16.py:494-598)."""
        open_bc = self.boundary_conditions.isSponge()
        perturb = self.small_scale_perturbation and apply_stochastic_term
        if self.t == 0:
            self.bc_kernel.update_bc_values(self.gpu_stream, self.t)
            self.bc_kernel.boundaryCondition(self.gpu_stream, self.gpu_data.h0, self.gpu_data.hu0,
                                             self.gpu_data.hv0)
        t_now = 0.0
        time_varying_wind = len(self.wind_stress.t) > 1
        pending_n, pending_dt, pending_w = 0, None, None
        while t_now < t_end:
            if update_dt:
                if pending_n:
                    self._launch_steps(pending_n, pending_dt, pending_w)
                    pending_n = 0
                self.updateDt()
            local_dt = np.float32(min(self.dt, np.float32(t_end - t_now)))
            wind_t = np.float32(self.update_wind_stress())
            if pending_n and (local_dt != pending_dt or wind_t != pending_w or time_varying_wind
                              or self.hasDrifters or open_bc or perturb):
                self._launch_steps(pending_n, pending_dt, pending_w)
                pending_n = 0
            pending_n += 1
            pending_dt, pending_w = local_dt, wind_t
            if self.hasDrifters or time_varying_wind or open_bc or perturb:
                # one launch per step: the drifters move between steps, the
                # wind or the exterior solution of this step's time, the
                # model error perturbs each step's result before its
                # boundary conditions (CDKLM16.py:580-586)
                if open_bc:
                    self.bc_kernel.update_bc_values(self.gpu_stream, self.t)
                self._launch_steps(pending_n, pending_dt, pending_w)
                pending_n = 0
                if perturb:
                    self.small_scale_model_error.perturbSim(self)
                    self.applyBoundaryConditions()
                self.drifterStep(local_dt)
            self.t += np.float64(local_dt)
            t_now += np.float64(local_dt)
            self.num_iterations += 1
        if pending_n:
            self._launch_steps(pending_n, pending_dt, pending_w)
        if self.write_netcdf and write_now:
            self.sim_writer.writeTimestep(self)
        return self.t

    def drifterStep(self, dt):
        """Advances the attached drifters through the new state
        (CDKLM16.py:600-610)."""
        if self.hasDrifters:
            self.drifters.drift(self.gpu_data.h0, self.gpu_data.hu0, self.gpu_data.hv0, self.bathymetry.Bm,
                                self.nx, self.ny, self.t, self.dx, self.dy, dt, np.int32(2), np.int32(2))
            self.drifter_t += dt
            return self.drifter_t

    def callKernel(self, h_in, hu_in, hv_in, h_out, hu_out, hv_out, local_dt, wind_stress_t, rk_step):
        """One sub-step (CDKLM16.py:613-639) through go_cdklm_swe_2D."""
        bc = self.boundary_conditions
        packed = _native.pack_bc(bc.north, bc.east, bc.south, bc.west)
        _native.check(_native.load().go_cdklm_swe_2D(
            self._domain.handle, _native.stream_handle(self.gpu_stream), float(local_dt), int(rk_step),
            _native.ptr(h_in.tensor), int(h_in.pitch), _native.ptr(hu_in.tensor), int(hu_in.pitch),
            _native.ptr(hv_in.tensor), int(hv_in.pitch),
            _native.ptr(h_out.tensor), int(h_out.pitch), _native.ptr(hu_out.tensor), int(hu_out.pitch),
            _native.ptr(hv_out.tensor), int(hv_out.pitch),
            _native.ptr(self.bathymetry.Bi.tensor), int(self.bathymetry.Bi.pitch),
            _native.ptr(self.bathymetry.Bm.tensor), int(self.bathymetry.Bm.pitch),
            float(self.bathymetry.mask_value), float(wind_stress_t), packed))

    def perturbState(self, q0_scale=1):
        """Adds one model-error perturbation (CDKLM16.py:642-644)."""
        if self.small_scale_perturbation:
            self.small_scale_model_error.perturbSim(self, q0_scale=q0_scale)

    def angle_texture_field(self):
        """The grid angle as the reference's 1 x 1 angle texture."""
        return np.array([[self._angle0]], dtype=np.float32)

    def coriolis_texture_field(self):
        """The Coriolis parameter per ghost-inclusive row as a one-column
        texture (rows vary; the kernels read it where f is zero)."""
        rows = np.asarray(self.coriolis_rows, dtype=np.float32)
        if np.all(rows == rows[0]):
            return rows[:1].reshape(1, 1)
        return np.ascontiguousarray(rows.reshape(-1, 1))

    def applyBoundaryConditions(self):
        self.bc_kernel.boundaryCondition(self.gpu_stream, self.gpu_data.h0, self.gpu_data.hu0, self.gpu_data.hv0)

    def dataAssimilationStep(self, observation_time, model_error_final_step=True, write_now=True,
                             courant_number=0.8):
        """CDKLM16.py:650-704."""
        full_model_time_steps = int(round(observation_time - self.t) / self.model_time_step)
        leftover_step_size = observation_time - self.t - full_model_time_steps * self.model_time_step
        if leftover_step_size / self.model_time_step < 0.1 and full_model_time_steps > 1:
            leftover_step_size += self.model_time_step
            full_model_time_steps -= 1
        if leftover_step_size / self.model_time_step < 0.00001:
            leftover_step_size = 0
        assert full_model_time_steps > 0, "There is less than CDKLM16.model_time_step until the observation"
        self.updateDt(courant_number=courant_number)
        for i in range(full_model_time_steps + 1):
            if i == 0 and leftover_step_size == 0:
                continue
            elif i == 0:
                self.step(leftover_step_size, apply_stochastic_term=False, write_now=False)
                self.perturbState(q0_scale=np.sqrt(leftover_step_size / self.model_time_step))
            else:
                self.step(self.model_time_step, apply_stochastic_term=False, write_now=False)
                if (i < full_model_time_steps) or model_error_final_step:
                    self.perturbState()
            self.total_time_steps += 1
            if self.total_time_steps % 5 == 0:
                self.updateDt(courant_number=courant_number)
        if self.write_netcdf and write_now:
            self.sim_writer.writeTimestep(self)
        assert round(observation_time) == round(self.t), \
            'The simulation time is not the same as observation time after dataAssimilationStep!'

    def writeState(self):
        """Appends the current state to the NetCDF file (CDKLM16.py:706-708)."""
        if self.write_netcdf:
            self.sim_writer.writeTimestep(self)

    # -- time step ----------------------------------------------------------
    def maxDtDevice(self):
        """Launch the exact CFL reduction; returns the device scalar tensor."""
        g = self.gpu_data
        _native.check(_native.load().go_max_dt(
            self._domain.handle, _native.stream_handle(self.gpu_stream),
            _native.ptr(g.h0.tensor), _native.ptr(g.hu0.tensor), _native.ptr(g.hv0.tensor), int(g.h0.pitch),
            _native.ptr(self.bathymetry.Bm.tensor), int(self.bathymetry.Bm.pitch),
            float(self.bathymetry.mask_value), _native.ptr(self._dt_dev)))
        return self._dt_dev[0:1]

    def updateDt(self, courant_number=None):
        """dt = courant * exact CFL limit (CDKLM16.py:712-739)."""
        if courant_number is None:
            courant_number = self.courant_number
        d = self.maxDtDevice()
        self.gpu_stream.synchronize()
        dt_host = d.cpu().numpy()
        self._last_max_dt = dt_host.reshape(1, 1)
        self.dt = courant_number * dt_host[0]

    def _getMaxTimestepHost(self, courant_number=0.8):
        """Host CFL reference (CDKLM16.py:741-759)."""
        eta, hu, hv = self.download(interior_domain_only=True)
        Hm = self.downloadBathymetry()[1][2:-2, 2:-2]
        h = eta + Hm
        gravityWaves = np.sqrt(self.g * h)
        u = hu / h
        v = hv / h
        max_dt = 0.25 * min(self.dx / np.max(np.abs(u) + gravityWaves), self.dy / np.max(np.abs(v) + gravityWaves))
        return courant_number * max_dt

    def downloadBathymetry(self, interior_domain_only=False):
        Bi, Bm = self.bathymetry.download(self.gpu_stream)
        if interior_domain_only:
            idx = self.interior_domain_indices
            Bi = Bi[idx[2]:idx[0] + 1, idx[3]:idx[1] + 1]
            Bm = Bm[idx[2]:idx[0], idx[3]:idx[1]]
        return [Bi, Bm]

    def getLandMask(self, interior_domain_only=True):
        if self.gpu_data.h0.mask is None:
            return None
        if interior_domain_only:
            return self.gpu_data.h0.mask[2:-2, 2:-2]
        return self.gpu_data.h0.mask

    def downloadDt(self):
        """The last CFL limit computed by updateDt, as a 1x1 array (the
        reference returns its per-block buffer)."""
        return getattr(self, "_last_max_dt", np.zeros((1, 1), dtype=np.float32))

    def status(self, clear=False):
        """Device status bits (GO_STATUS_NONFINITE when a cell went NaN/Inf)."""
        self.gpu_stream.synchronize()
        return self._domain.status(clear)
