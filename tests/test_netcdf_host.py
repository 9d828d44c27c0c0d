"""NetCDF writer and reader on the CPU (SWESimulators.SimWriter,
SimReader) with a stand-in simulator: the reference's file layout
(gpu_ocean/SWESimulators/SimWriter.py:149-443: global attributes,
dimensions, variables), records appended per writeTimestep, the reader's
accessors (SimReader.py:26-155), and BoundaryConditions' string form
(Common.py:899-946), which the files store."""

import types

import numpy as np
import pytest
from scipy.io import netcdf_file

from SWESimulators import SimReader, SimWriter
from SWESimulators.Common import BoundaryConditions

# global attributes SimWriter.py:149-199 writes for a CDKLM16 without
# model error and without a wind source file
REFERENCE_ATTRS = {
    "Conventions", "git_hash", "ignore_ghostcells", "num_layers", "staggered_grid", "simulator_short",
    "boundary_conditions", "boundary_conditions_sponge_mr", "time_integrator", "minmod_theta", "coriolis_force",
    "coriolis_beta", "y_zero_reference_cell", "eddy_viscosity_coefficient", "g", "nx", "ny", "dx", "dy", "dt",
    "auto_dt", "bottom_friction_r", "ghost_cells_north", "ghost_cells_east", "ghost_cells_south",
    "ghost_cells_west", "model_time_step", "small_scale_perturbation"}
REFERENCE_VARS = {"time", "x", "y", "x_Hi", "y_Hi", "projection_stere", "land_binary_mask", "Hm", "Hi", "eta", "hu",
                  "hv"}


class CDKLM16:
    """Stand-in with the attributes SimWriter reads (named CDKLM16 so the
    file says simulator_short = CDKLM16)."""

    def __init__(self, nx=12, ny=9, bc=BoundaryConditions(2, 1, 2, 1)):
        rng = np.random.default_rng(4)
        self.nx, self.ny, self.dx, self.dy = np.int32(nx), np.int32(ny), np.float32(500.0), np.float32(400.0)
        self.dt, self.g, self.f, self.r = np.float32(2.5), np.float32(9.81), np.float32(1.2e-4), np.float32(3e-3)
        self.theta, self.rk_order, self.coriolis_beta = np.float32(1.3), 2, np.float32(0.0)
        self.y_zero_reference_cell = np.float32(2.0)
        self.ghost_cells_x = self.ghost_cells_y = np.int32(2)
        self.boundary_conditions = bc
        self.wind_stress = types.SimpleNamespace(source_filename=None)
        self.A = "NA"
        self.comm = None
        self.model_time_step = np.float32(2.5)
        self.small_scale_perturbation = False
        self.gpu_stream = None
        self.t = 0.0
        Hi = rng.uniform(40, 60, (ny + 5, nx + 5)).astype(np.float32)
        Hm = 0.25 * (Hi[:-1, :-1] + Hi[1:, :-1] + Hi[:-1, 1:] + Hi[1:, 1:])
        self.bathymetry = types.SimpleNamespace(download=lambda s: (Hi, Hm))
        self.state = [rng.standard_normal((ny + 4, nx + 4)).astype(np.float32) for _ in range(3)]

    def download(self):
        return tuple(a.copy() for a in self.state)

    def advance(self, dt):
        self.t += dt
        self.state = [a * np.float32(0.9) + np.float32(0.01) for a in self.state]


def _write(tmp_path, sim, n, **kw):
    w = SimWriter.SimNetCDFWriter(sim, filename=str(tmp_path / "run"), **kw)
    for _ in range(n):
        sim.advance(sim.dt)
        w.writeTimestep(sim)
    w.close()
    return w.output_file_name


def test_layout_matches_reference(tmp_path):
    sim = CDKLM16()
    name = _write(tmp_path, sim, 3)
    assert name == str(tmp_path / "run.nc")
    with netcdf_file(name, "r", mmap=False) as nc:
        assert REFERENCE_ATTRS <= set(nc._attributes)
        assert REFERENCE_VARS <= set(nc.variables)
        assert nc.dimensions["x"] == 16 and nc.dimensions["y"] == 13
        assert nc.dimensions["x_Hi"] == 17 and nc.dimensions["y_Hi"] == 14 and nc.dimensions["time"] is None
        assert nc.variables["eta"].dimensions == ("time", "y", "x")
        assert nc.variables["Hi"].dimensions == ("y_Hi", "x_Hi")
        assert nc.variables["eta"].shape == (4, 13, 16)
        # cell-centre axes with the ghost cells (SimWriter.py:278-284)
        np.testing.assert_allclose(nc.variables["x"][:], (np.arange(16) - 2 + 0.5) * 500.0)
        np.testing.assert_allclose(nc.variables["y_Hi"][:], (np.arange(14) - 2) * 400.0)
        assert nc._attributes["simulator_short"] in (b"CDKLM16", "CDKLM16")


def test_reader_round_trip(tmp_path):
    sim = CDKLM16()
    states = [sim.download()]
    w = SimWriter.SimNetCDFWriter(sim, filename=str(tmp_path / "rt"))
    for _ in range(4):
        sim.advance(sim.dt)
        states.append(sim.download())
        w.writeTimestep(sim)
    w.close()
    r = SimReader.SimNetCDFReader(str(tmp_path / "rt.nc"), ignore_ghostcells=False)
    assert r.getNumTimeSteps() == 5
    np.testing.assert_allclose(r.getTimes(), np.arange(5) * 2.5)
    for k in range(5):
        eta, hu, hv, t = r.getTimeStep(k)
        assert np.array_equal(eta, states[k][0]) and np.array_equal(hu, states[k][1])
        assert np.array_equal(hv, states[k][2]) and t == np.float32(2.5 * k)
    eta, hu, hv, t = r.getLastTimeStep()
    assert np.array_equal(hv, states[-1][2]) and t == np.float32(10.0)
    eta, hu, hv, t = r.getStateAtTime(5.2)
    assert np.array_equal(eta, states[2][0])
    with pytest.raises(RuntimeError):
        r.getStateAtTime(3.0)
    assert np.array_equal(r.getH(), sim.bathymetry.download(None)[0])
    assert r.get("nx") == 12 and r.get("dt") == np.float32(2.5) and r.get("absent") == "not found"
    assert r.has("Hm") and r.has("coriolis_force") and not r.has("H")
    bc = r.getBC()
    assert bc.codes() == (2, 1, 2, 1)
    r.close()
    r = SimReader.SimNetCDFReader(str(tmp_path / "rt.nc"), ignore_ghostcells=True)
    eta, hu, hv, t = r.getTimeStep(1)
    assert np.array_equal(eta, states[1][0][2:-2, 2:-2])
    r.close()


def test_interior_only_file(tmp_path):
    sim = CDKLM16()
    name = _write(tmp_path, sim, 2, ignore_ghostcells=True)
    with netcdf_file(name, "r", mmap=False) as nc:
        assert nc.variables["eta"].shape == (3, 9, 12)
        assert np.array_equal(nc.variables["hu"][2], sim.download()[1][2:-2, 2:-2])


@pytest.mark.parametrize("codes, sponge", [((1, 1, 1, 1), {"north": 0, "south": 0, "east": 0, "west": 0}),
                                           ((2, 2, 2, 2), {"north": 0, "south": 0, "east": 0, "west": 0}),
                                           ((3, 1, 4, 2), {"north": 10, "east": 0, "south": 7, "west": 0})])
def test_boundary_conditions_string_round_trip(codes, sponge):
    if codes[1] != codes[3] and 2 in (codes[1], codes[3]):
        codes = (codes[0], 2, codes[2], 2)
    b = BoundaryConditions(*codes, spongeCells=sponge)
    s = str(b)
    assert "np.int32" not in s
    c = BoundaryConditions.fromstring(s)
    assert c.codes() == b.codes() and {k: int(v) for k, v in c.getSponge().items()} == sponge
    # the older list form of the sponge widths (north, east, south, west)
    legacy = BoundaryConditions.fromstring("north: Wall, east: Periodic, south: Wall, west: Periodic, "
                                           "spongeCells: [1, 2, 3, 4]")
    assert legacy.codes() == (1, 2, 1, 2) and legacy.getSponge()["south"] == 3


def test_reader_returns_native_byte_order(tmp_path):
    sim = CDKLM16()
    name = _write(tmp_path, sim, 1)
    r = SimReader.SimNetCDFReader(name, ignore_ghostcells=False)
    eta, hu, hv, t = r.getLastTimeStep()
    for a in (eta, hu, hv, r.getH(), r.getTimes(), r.getHm()):
        assert a.dtype.isnative and a.flags.c_contiguous
    r.close()
