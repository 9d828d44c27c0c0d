"""Reading simulator output from NetCDF (the reference's
gpu_ocean/SWESimulators/SimReader.py:26-155, without its plotting helpers):
attributes, time steps with or without ghost cells, bathymetry, boundary
conditions, as CDKLM16.fromfilename needs them.

Reads NetCDF-3 files (what SimWriter writes here) through
scipy.io.netcdf_file; a NetCDF-4 file written by the reference can be
converted first (``nccopy -k nc6 in.nc out.nc``).
"""

import numpy as np
from scipy.io import netcdf_file

from . import Common


def _arr(a):
    """A native-byte-order copy (NetCDF data are big-endian)."""
    a = np.asarray(a)
    return np.ascontiguousarray(a, dtype=a.dtype.newbyteorder("="))


def _value(v):
    if isinstance(v, bytes):
        return v.decode()
    if isinstance(v, np.ndarray) and v.size == 1:
        return v.reshape(-1)[0]
    return v


class SimNetCDFReader:

    def __init__(self, filename, ignore_ghostcells=True):
        self.filename = filename
        self.ignore_ghostcells = ignore_ghostcells
        self.ncfile = netcdf_file(filename, "r", mmap=False)
        self.ghostCells = [int(self.get("ghost_cells_north")), int(self.get("ghost_cells_east")),
                           int(self.get("ghost_cells_south")), int(self.get("ghost_cells_west"))]
        self.staggered_grid = str(self.get("staggered_grid")) == "True"
        self.text_font_size = 12

    def close(self):
        self.ncfile.close()

    def get(self, attr):
        """A global attribute, or "not found" (SimReader.py:50-54)."""
        try:
            return _value(self.ncfile._attributes[attr])
        except KeyError:
            return "not found"

    def has(self, fieldname):
        return fieldname in self.ncfile._attributes or fieldname in self.ncfile.variables

    def printVariables(self):
        for var in self.ncfile.variables:
            print(var)

    def printAttributes(self):
        for attr in self.ncfile._attributes:
            print(attr + "\t--> " + str(self.get(attr)))

    def getNumTimeSteps(self):
        return self.ncfile.variables["time"].shape[0]

    def getBC(self):
        return Common.BoundaryConditions.fromstring(self.get("boundary_conditions"))

    def getTimes(self):
        return _arr(self.ncfile.variables["time"][:])

    def getLastTimeStep(self):
        return self.getTimeStep(-1)

    def _crop(self, a):
        if not self.ignore_ghostcells:
            return a
        g = self.ghostCells
        return a[g[2]:-g[0], g[3]:-g[1]]

    def getTimeStep(self, index):
        """eta, hu, hv and the time of record index (SimReader.py:92-113)."""
        v = self.ncfile.variables
        eta = _arr(v["eta"][index, :, :])
        hu = _arr(v["hu"][index, :, :])
        hv = _arr(v["hv"][index, :, :])
        return self._crop(eta), self._crop(hu), self._crop(hv), np.float32(v["time"][index])

    def getH(self):
        if "H" in self.ncfile.variables:
            return _arr(self.ncfile.variables["H"][:, :])
        return _arr(self.ncfile.variables["Hm" if self.staggered_grid else "Hi"][:, :])

    def getHm(self):
        return _arr(self.ncfile.variables["Hm"][:, :])

    def getStateAtTime(self, time):
        """The record whose time equals round(time) (SimReader.py:131-145)."""
        time = np.round(time)
        times = self.ncfile.variables["time"][:]
        for i in range(times.shape[0]):
            if time == times[i]:
                return self.getStateAtTimeStep(i)
        raise RuntimeError("Time " + str(time) + " not in NetCDF file " + self.filename)

    def getStateAtTimeStep(self, index, etaOnly=False):
        v = self.ncfile.variables
        eta = self._crop(_arr(v["eta"][index, :, :]))
        t = v["time"][index]
        if etaOnly:
            return eta, t
        return eta, self._crop(_arr(v["hu"][index, :, :])), self._crop(_arr(v["hv"][index, :, :])), t

    def getEtaAtTimeStep(self, index):
        return self.getStateAtTimeStep(index, etaOnly=True)

    def getAxis(self):
        x = _arr(self.ncfile.variables["x"][:])
        y = _arr(self.ncfile.variables["y"][:])
        if self.ignore_ghostcells:
            x = x[self.ghostCells[2]:-self.ghostCells[0]]
            y = y[self.ghostCells[3]:-self.ghostCells[1]]
        return x, y

    def getEtaXSlice(self, t, y):
        y_index = int(y) + int(self.get("ghost_cells_south"))
        return _arr(self.ncfile.variables["eta"][t, y_index, self.ghostCells[3]:-self.ghostCells[1]])
