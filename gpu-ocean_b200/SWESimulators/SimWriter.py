"""Simulator output to NetCDF, following the reference's file layout
(gpu_ocean/SWESimulators/SimWriter.py:35-498): the same global attributes,
dimensions (time unlimited, x, y, x_Hi, y_Hi), coordinate variables,
projection, land mask, bathymetry (Hm, Hi) and one eta, hu, hv record per
written time step, so the reference's SimNetCDFReader and
CDKLM16.fromfilename can read the files and restart from them.

The reference writes NetCDF-4 (HDF5, zlib) through netCDF4-python, which is
not available here; this writer produces NetCDF-3 classic files with the
64-bit offset format through scipy.io.netcdf_file (no compression), which
netCDF4-python and every NetCDF reader also open.  Differences: no
compression; the parallel (MPI) layout is not written; with
ignore_ghostcells the interior (two ghost cells cut on each side) is stored,
which is what the x, y dimensions describe (the reference slices one cell,
SimWriter.py:460-466, which does not fit them for CDKLM16).
"""

import datetime
import os
import subprocess

import numpy as np
from scipy.io import netcdf_file


class _NetCDF3File(netcdf_file):
    """scipy's NetCDF-3 writer with its variable order fixed: scipy sorts
    the variables by shape and places a scalar (0-d) variable after the
    record variables, so its value lands inside the second record (seen
    with scipy 1.18 on the time variable).  NetCDF-3 stores all non-record
    variables before the records; this keeps that order, scalars included."""

    def _write_var_array(self):
        if not self.variables:
            return super()._write_var_array()
        self.fp.write(b"\x00\x00\x00\x0b")              # NC_VARIABLE
        self._pack_int(len(self.variables))
        names = sorted(self.variables, key=lambda n: 1 if self.variables[n].isrec else 0)
        for name in names:
            self._write_var_metadata(name)
        self.__dict__["_recsize"] = sum(v._vsize for v in self.variables.values() if v.isrec)
        for name in names:
            self._write_var_data(name)


def _attr(v):
    """An attribute value NetCDF-3 holds: strings, numbers, arrays."""
    if isinstance(v, (bool, np.bool_)):
        return str(bool(v))
    if isinstance(v, (np.floating, float)):
        return np.float32(v) if isinstance(v, np.float32) else np.float64(v)
    if isinstance(v, (np.integer, int)):
        return np.int32(v)
    return v


class SimNetCDFWriter:
    """Writes a simulator's state to a NetCDF file after each call of
    writeTimestep (SimWriter.py:35-443)."""

    def __init__(self, sim, super_dir_name=None, filename=None, num_layers=1, staggered_grid=False,
                 ignore_ghostcells=False, offset_x=0, offset_y=0):
        self.write_parallel = False
        self.gpu_stream = sim.gpu_stream
        self.ignore_ghostcells = ignore_ghostcells
        self.staggered_grid = staggered_grid
        self.num_layers = num_layers
        if staggered_grid or num_layers != 1:
            raise NotImplementedError("only the single-layer, non-staggered (CDKLM16) layout is written")

        now = datetime.datetime.now()
        self.timestamp = now.strftime("%Y_%m_%d-%H_%M_%S")
        self.timestamp_short = now.strftime("%Y_%m_%d")
        try:
            self.git_hash = str.strip(str(subprocess.check_output(["git", "rev-parse", "HEAD"],
                                                                  stderr=subprocess.DEVNULL)))
        except Exception:
            self.git_hash = "git info missing..."
        self.simulator_short = str(sim.__class__.__name__)

        # file name (SimWriter.py:78-100)
        self.super_dir_name = super_dir_name if super_dir_name is not None else os.getcwd()
        self.dir_name = os.path.join(self.super_dir_name, "netcdf_" + self.timestamp_short + "/")
        if not filename:
            self.output_file_name = self.dir_name + self.simulator_short + "_" + self.timestamp + ".nc"
        elif str.find(filename, "/") == -1:
            self.output_file_name = self.dir_name + self.simulator_short + "_" + filename + ".nc"
        else:
            self.output_file_name = filename + ".nc"
            self.dir_name = filename.rsplit("/", 1)[0]
        self.output_file_name = self.output_file_name.replace(".nc.nc", ".nc")
        self.current_directory = os.getcwd()

        # simulator description (SimWriter.py:105-146)
        self.boundary_conditions = str(sim.boundary_conditions)
        self.boundary_conditions_sponge_mr = str({k: int(v) for k, v in
                                                  sim.boundary_conditions.getSponge().items()})
        self.dt = sim.dt
        self.Hi, self.Hm = sim.bathymetry.download(self.gpu_stream)
        self.time_integrator = sim.rk_order
        self.minmod_theta = sim.theta
        self.coriolis_force = sim.f
        self.coriolis_beta = sim.coriolis_beta
        self.y_zero_reference_cell = sim.y_zero_reference_cell - 2
        self.wind_stress = getattr(sim.wind_stress, "source_filename", None)
        self.eddy_viscosity_coefficient = getattr(sim, "A", "NA")
        nx, ny, dx, dy = int(sim.nx), int(sim.ny), sim.dx, sim.dy
        self.dx, self.dy = dx, dy
        gx, gy = int(sim.ghost_cells_x), int(sim.ghost_cells_y)
        self.ghost_cells_east = self.ghost_cells_west = gx
        self.ghost_cells_north = self.ghost_cells_south = gy
        self.bottom_friction_r = sim.r

        if sim.comm:
            self.output_file_name = self.output_file_name.replace(
                ".nc", "_" + str(sim.comm.rank) + "_" + str(sim.local_particle_id) + ".nc")
        os.makedirs(self.dir_name, exist_ok=True)
        self.ncfile = _NetCDF3File(self.output_file_name, "w", version=2)
        nc = self.ncfile
        attrs = {
            "Conventions": "CF-1.4", "git_hash": self.git_hash, "ignore_ghostcells": str(self.ignore_ghostcells),
            "num_layers": self.num_layers, "staggered_grid": str(self.staggered_grid),
            "simulator_short": self.simulator_short, "boundary_conditions": self.boundary_conditions,
            "boundary_conditions_sponge_mr": self.boundary_conditions_sponge_mr,
            "time_integrator": self.time_integrator, "minmod_theta": self.minmod_theta,
            "coriolis_force": self.coriolis_force, "coriolis_beta": self.coriolis_beta,
            "y_zero_reference_cell": self.y_zero_reference_cell,
            "eddy_viscosity_coefficient": self.eddy_viscosity_coefficient, "g": sim.g, "nx": nx, "ny": ny,
            "dx": dx, "dy": dy, "dt": sim.dt, "auto_dt": str(False), "bottom_friction_r": self.bottom_friction_r,
            "ghost_cells_north": gy, "ghost_cells_east": gx, "ghost_cells_south": gy, "ghost_cells_west": gx,
        }
        if self.wind_stress is not None:
            attrs["wind_stress_source"] = self.wind_stress
        if self.simulator_short == "CDKLM16":
            # model error and data assimilation (SimWriter.py:184-199)
            attrs["model_time_step"] = sim.model_time_step
            attrs["small_scale_perturbation"] = str(sim.small_scale_perturbation)
            if sim.small_scale_perturbation:
                attrs["small_scale_perturbation_amplitude"] = sim.small_scale_model_error.soar_q0
                attrs["small_scale_perturbation_interpolation_factor"] = \
                    sim.small_scale_model_error.interpolation_factor
        for k, v in attrs.items():
            setattr(nc, k, _attr(v))

        # dimensions and axes (SimWriter.py:204-331)
        nc.createDimension("time", None)
        xs, ys = (nx, ny) if self.ignore_ghostcells else (nx + 2 * gx, ny + 2 * gy)
        nc.createDimension("x", xs)
        nc.createDimension("y", ys)
        nc.createDimension("x_Hi", nx + 2 * gx + 1)
        nc.createDimension("y_Hi", ny + 2 * gy + 1)
        self.nc_time = nc.createVariable("time", "f", ("time",))
        x = nc.createVariable("x", "f", ("x",))
        y = nc.createVariable("y", "f", ("y",))
        x_Hi = nc.createVariable("x_Hi", "f", ("x_Hi",))
        y_Hi = nc.createVariable("y_Hi", "f", ("y_Hi",))
        for v, name, ax in ((x, "projection_x_coordinate", "X"), (y, "projection_y_coordinate", "Y"),
                            (x_Hi, "projection_x_coordinate", "X"), (y_Hi, "projection_y_coordinate", "Y")):
            v.standard_name = name
            v.axis = ax
            v.units = "meter"
        self.nc_proj = nc.createVariable("projection_stere", "i", ())
        self.nc_proj.grid_mapping_name = "polar_stereographic"
        self.nc_proj.scale_factor_at_projection_origin = 0.9330127018922193
        self.nc_proj.straight_vertical_longitude_from_pole = 70.0
        self.nc_proj.latitude_of_projection_origin = 90.0
        self.nc_proj.earth_radius = 6371000.0
        self.nc_proj.proj4 = "+proj=stere +lat_0=90 +lon_0=70 +lat_ts=60 +units=m +a=6.371e+06 +e=0 +no_defs"
        if not self.ignore_ghostcells:
            x[:] = np.linspace(-gx * dx + dx / 2.0, (nx + gx) * dx - dx / 2.0, nx + 2 * gx)
            y[:] = np.linspace(-gy * dy + dy / 2.0, (ny + gy) * dy - dy / 2.0, ny + 2 * gy)
        else:
            x[:] = np.linspace(offset_x, nx * dx, nx)
            y[:] = np.linspace(offset_y, ny * dy, ny)
        x_Hi[:] = np.linspace(-gx * dx, (nx + gx) * dx, nx + 2 * gx + 1)
        y_Hi[:] = np.linspace(-gy * dy, (ny + gy) * dy, ny + 2 * gy + 1)
        self.nc_time.units = "seconds since 1970-01-01 00:00:00"

        self.nc_land = nc.createVariable("land_binary_mask", "f", ("y", "x"))
        self.nc_land.standard_name = "land_binary_mask"
        self.nc_land.units = "1"
        self.nc_land[:] = 0
        self.nc_Hm = nc.createVariable("Hm", "f", ("y", "x"))
        self.nc_Hi = nc.createVariable("Hi", "f", ("y_Hi", "x_Hi"))
        for v in (self.nc_Hm, self.nc_Hi):
            v.standard_name = "water_surface_reference_datum_altitude"
            v.grid_mapping = "projection_stere"
            v.coordinates = "y x"
            v.units = "meter"
        self.nc_Hm[:] = self._cut(self.Hm)
        self.nc_Hi[:] = self.Hi
        if sim.comm:
            nc.ensemble_member = np.int32(sim.comm.rank)
        self.nc_eta = nc.createVariable("eta", "f", ("time", "y", "x"))
        self.nc_hu = nc.createVariable("hu", "f", ("time", "y", "x"))
        self.nc_hv = nc.createVariable("hv", "f", ("time", "y", "x"))
        for v, name, units, coords in ((self.nc_eta, "water_surface_height_above_reference_datum", "meter", "y x"),
                                       (self.nc_hu, "x_sea_water_velocity", "meter second-1", "y_hu x_hu"),
                                       (self.nc_hv, "y_sea_water_velocity", "meter second-1", "y_hv x_hv")):
            v.standard_name = name
            v.grid_mapping = "projection_stere"
            v.coordinates = coords
            v.units = units
        self.i = 0
        self.writeTimestep(sim)

    def _cut(self, a):
        if not self.ignore_ghostcells:
            return a
        return a[self.ghost_cells_south:a.shape[0] - self.ghost_cells_north,
                 self.ghost_cells_west:a.shape[1] - self.ghost_cells_east]

    def __enter__(self):
        return self

    def __exit__(self, exc_type, exc_value, traceback):
        self.close()

    def close(self):
        if self.ncfile is not None:
            self.ncfile.close()
            self.ncfile = None

    def writeTimestep(self, sim):
        """Appends the simulator's time and state (SimWriter.py:445-475)."""
        eta, hu, hv = sim.download()
        self.write(sim.t, eta, hu, hv)

    def write(self, t, eta, hu, hv, eta2=None, hu2=None, hv2=None):
        """Appends one record (SimWriter.py:478-498, single layer)."""
        self.nc_time[self.i] = t
        self.nc_eta[self.i, :, :] = self._cut(np.asarray(eta, dtype=np.float32))
        self.nc_hu[self.i, :, :] = self._cut(np.asarray(hu, dtype=np.float32))
        self.nc_hv[self.i, :, :] = self._cut(np.asarray(hv, dtype=np.float32))
        self.ncfile.flush()
        self.i += 1
