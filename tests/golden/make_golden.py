"""Generate ``cdklm16_timestep50.npz`` from the reference's own test data.

Run in a container where metno/gpu-ocean is mounted at REF (the default is
the read-only mount used while building this repository):

    python tests/golden/make_golden.py [REF]

What it stores (all float32, exact):

* the 12 CDKLM16 golden cases of ``gpu_ocean/tests/schemes/CDKLM16_test.py``
  (lines 154-421): the expected eta/hu/hv after ``sim.step(50.0)`` read from
  ``gpu_ocean/tests/timestep50/CDKLM16_*.dat`` (74 x 54 text files written
  from float32 device arrays, so the float32 cast is exact -- checked below);
* the initial conditions of each case, produced by importing the
  reference's ``gpu_ocean/tests/testUtils.py`` (addCentralBump,
  addCornerBump, addUpperCornerBump, makeBottomTopography) with the test's
  setUp() parameters (nx=50, ny=70, dx=dy=200, flat Hi=60).

Nothing at test time reads the reference tree; the tests only read the npz.
"""

import os
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GOCEAN_REFERENCE")
if not REF:
    raise SystemExit("name the gpu-ocean source tree: make_golden.py <tree> or GOCEAN_REFERENCE=<tree>")
TESTS = os.path.join(REF, "gpu_ocean", "tests")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cdklm16_timestep50.npz")

sys.path.insert(0, TESTS)
import testUtils  # noqa: E402  (the reference's own helper module)

NX, NY = 50, 70
DX = DY = 200.0
HALO = np.array([2, 2, 2, 2])

# (case name, bc (north, east, south, west), bump, f, beta, bathymetry, golden file key)
# CDKLM16_test.py:154-421; periodic "central" cases reuse the wall golden file.
CASES = [
    ("wall_central", (1, 1, 1, 1), "central", 0.0, 0.0, False, ("wallBC", "central", "")),
    ("wall_corner", (1, 1, 1, 1), "corner", 0.0, 0.0, False, ("wallBC", "corner", "")),
    ("wall_upperCorner", (1, 1, 1, 1), "upperCorner", 0.0, 0.0, False, ("wallBC", "upperCorner", "")),
    ("periodic_central", (2, 2, 2, 2), "central", 0.0, 0.0, False, ("wallBC", "central", "")),
    ("periodic_corner", (2, 2, 2, 2), "corner", 0.0, 0.0, False, ("periodic", "corner", "")),
    ("periodic_upperCorner", (2, 2, 2, 2), "upperCorner", 0.0, 0.0, False, ("periodic", "upperCorner", "")),
    ("periodicNS_central", (2, 1, 2, 1), "central", 0.0, 0.0, False, ("wallBC", "central", "")),
    ("periodicNS_corner", (2, 1, 2, 1), "corner", 0.0, 0.0, False, ("periodicNS", "corner", "")),
    ("periodicNS_upperCorner", (2, 1, 2, 1), "upperCorner", 0.0, 0.0, False, ("periodicNS", "upperCorner", "")),
    ("periodicEW_central", (1, 2, 1, 2), "central", 0.0, 0.0, False, ("wallBC", "central", "")),
    ("periodicEW_corner", (1, 2, 1, 2), "corner", 0.0, 0.0, False, ("periodicEW", "corner", "")),
    ("periodicEW_upperCorner", (1, 2, 1, 2), "upperCorner", 0.0, 0.0, False, ("periodicEW", "upperCorner", "")),
    ("coriolis_central", (1, 1, 1, 1), "central", 0.01, 0.0, False, ("coriolis", "central", "")),
    ("betamodel_central", (1, 1, 1, 1), "central", 0.01 - 2 * 1e-6 * DY, 1e-6, False, ("betamodel", "central", "")),
    ("bathymetry_central", (1, 1, 1, 1), "central", 0.0, 0.0, True, ("wallBC", "central", "bathymetry_")),
]

BUMPS = {
    "central": testUtils.addCentralBump,
    "corner": testUtils.addCornerBump,
    "upperCorner": testUtils.addUpperCornerBump,
}


def load_dat(bc, init, bathy):
    prefix = os.path.join(TESTS, "timestep50", "CDKLM16_" + bc + "_" + init + "_" + bathy)
    out = []
    for field in ("eta", "u", "v"):
        a = np.loadtxt(prefix + field + ".dat")
        a32 = a.astype(np.float32)
        assert np.array_equal(a32.astype(np.float64), a), prefix + field + " is not float32-exact"
        out.append(a32)
    return out


def main():
    data = {}
    names = []
    for name, bc, bump, f, beta, bathy, key in CASES:
        shape = (NY + 4, NX + 4)
        eta0 = np.zeros(shape, dtype=np.float32)
        Hi = np.ones((shape[0] + 1, shape[1] + 1), dtype=np.float32) * 60
        BUMPS[bump](eta0, NX, NY, DX, DY, HALO)
        if bathy:
            testUtils.makeBottomTopography(Hi, NX, NY, DX, DY, HALO)
        eta, u, v = load_dat(*key)
        data[name + "/eta0"] = eta0
        data[name + "/Hi"] = Hi.astype(np.float32)
        data[name + "/bc"] = np.array(bc, dtype=np.int32)
        data[name + "/f_beta"] = np.array([f, beta], dtype=np.float64)
        data[name + "/eta"] = eta
        data[name + "/hu"] = u
        data[name + "/hv"] = v
        names.append(name)
    data["cases"] = np.array(names)
    data["setup"] = np.array([NX, NY, DX, DY, 0.9, 9.81, 50.0])  # nx, ny, dx, dy, dt, g, T
    np.savez_compressed(OUT, **data)
    print("wrote", OUT, os.path.getsize(OUT), "bytes,", len(names), "cases")


if __name__ == "__main__":
    main()
