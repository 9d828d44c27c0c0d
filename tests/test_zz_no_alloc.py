"""go_cdklm_step_static: the step that allocates nothing.

The file name puts it last in collection order, so it runs after every other
test has used the library (many domains created and destroyed); it also
passes when run alone.  Its state must match go_cdklm_step bit for bit on
two calls in a row, the second with a different Coriolis table and wind,
which shows that each call rewrites the static table.  A third and fourth
call show that the status word is cleared at the start of each call.
"""

import ctypes
import os

import numpy as np
import pytest

from SWESimulators import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MAX_ROWS = 16388    # ny + 4 limit of the static Coriolis table


def _lib():
    if not os.path.exists(_native.LIB_PATH):
        import subprocess
        import sys
        subprocess.run([sys.executable, os.path.join(ROOT, "gpu-ocean_b200", "build.py")], check=True)
    return _native.load()


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _call(lib, desc, stream, f_rows, wind, n_steps, dt, h0, h1, Hi, land, status=None):
    """h0, h1: (eta, hu, hv) device tensors; Hi: device tensor of corners."""
    P = _native.ptr
    return lib.go_cdklm_step_static(
        ctypes.byref(desc), stream, _fptr(f_rows), int(f_rows.size), float(wind[0]), float(wind[1]),
        int(n_steps), float(dt), P(h0[0]), P(h0[1]), P(h0[2]), h0[0].stride(0) * 4,
        P(h1[0]), P(h1[1]), P(h1[2]), h1[0].stride(0) * 4, P(Hi), Hi.stride(0) * 4, float(land),
        ctypes.byref(status) if status is not None else None)


def test_rejects_ny_over_static_limit():
    """Rejected on the host, before any CUDA call (runs without a GPU)."""
    lib = _lib()
    desc = _native.GoDomainDesc()
    desc.nx, desc.ny = 64, MAX_ROWS - 3
    desc.dx = desc.dy = 100.0
    desc.g, desc.theta = 9.81, 1.3
    desc.desing_eps = desc.flux_slope_eps = 0.1
    desc.depth_cutoff = 1e-5
    desc.rk_order = 2
    desc.bc_north = desc.bc_east = desc.bc_south = desc.bc_west = 1
    desc.north_y = 1.0
    fake = [ctypes.c_void_p(256 * (i + 1)) for i in range(7)]   # never dereferenced

    def call(f_rows):
        return lib.go_cdklm_step_static(ctypes.byref(desc), None, _fptr(f_rows), int(f_rows.size), 0.0, 0.0, 1,
                                        1.0, fake[0], fake[1], fake[2], 4 * 68, fake[3], fake[4], fake[5],
                                        4 * 68, fake[6], 4 * 69, 1e20, None)

    assert call(np.zeros(1, np.float32)) == _native.GO_ERR_INVALID
    assert b"static scratch" in lib.go_last_error()
    desc.ny = 48                     # within the limit, but a table of the wrong length
    assert call(np.zeros(7, np.float32)) == _native.GO_ERR_INVALID
    assert b"Coriolis table" in lib.go_last_error()


@pytest.mark.gpu
def test_two_calls_match_go_cdklm_step_bitwise():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA GPU")
    from SWESimulators import CDKLM16, Common, SyntheticCases as SC

    lib = _lib()
    ctx = Common.CUDAContext()
    c = SC.grf(192, dx=1000.0, seed_bathy=51000, seed_bumps=51500, steps=1)
    sim = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
    stream = torch.cuda.Stream()
    sh = _native.stream_handle(stream)
    g = sim.gpu_data
    ref0 = (g.h0.tensor, g.hu0.tensor, g.hv0.tensor)
    ref1 = (g.h1.tensor, g.hu1.tensor, g.hv1.tensor)
    torch.cuda.synchronize()
    st0 = tuple(t.clone() for t in ref0)
    st1 = tuple(t.clone() for t in ref1)
    Hi = sim.bathymetry.Bi.tensor
    land = float(sim.bathymetry.mask_value)
    desc = sim._domain.desc
    dt = np.float32(c.dt)
    status = ctypes.c_uint32(0xFFFF)

    def compare():
        torch.cuda.synchronize()
        for a, b in zip(ref0 + ref1, st0 + st1):
            assert torch.equal(a, b)

    # setup call: looks up the scratch address, no launches
    assert _call(lib, desc, sh, np.asarray(sim.coriolis_rows, np.float32), (0, 0), 0, dt, st0, st1, Hi,
                 land) == _native.GO_OK, lib.go_last_error()

    # call 1: the case's beta-plane table (ny+4 rows) and its wind
    rows = np.ascontiguousarray(np.asarray(sim.coriolis_rows, np.float32))
    wind = (np.float32(c.wind[0]), np.float32(c.wind[1]))
    sim._domain.set_coriolis(rows)
    sim._domain.set_wind_uniform(wind[0], wind[0], wind[1], wind[1])
    sim._launch_steps(7, dt, 0.0)
    rc = _call(lib, desc, sh, rows, wind, 7, dt, st0, st1, Hi, land, status)
    assert rc == _native.GO_OK, lib.go_last_error()
    assert status.value == 0
    compare()

    # call 2: an f-plane (one value) and another wind, continuing the state
    fplane = np.array([1.3e-4], np.float32)
    wind2 = (np.float32(-2.0e-5), np.float32(3.5e-5))
    sim._domain.set_coriolis(fplane)
    sim._domain.set_wind_uniform(wind2[0], wind2[0], wind2[1], wind2[1])
    sim._launch_steps(5, dt, 0.0)
    status.value = 0xFFFF
    rc = _call(lib, desc, sh, fplane, wind2, 5, dt, st0, st1, Hi, land, status)
    assert rc == _native.GO_OK, lib.go_last_error()
    assert status.value == 0
    compare()

    # calls 3 and 4: a non-finite cell raises the status word; the next
    # call starts from a cleared word and free device memory is unchanged
    bad0 = tuple(t.clone() for t in st0)
    bad1 = tuple(t.clone() for t in st1)
    bad0[1][60:64, 60:64] = float("nan")
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    assert _call(lib, desc, sh, fplane, wind2, 1, dt, bad0, bad1, Hi, land, status) == _native.GO_OK
    assert status.value & _native.GO_STATUS_NONFINITE
    assert _call(lib, desc, sh, rows, wind, 2, dt, st0, st1, Hi, land, status) == _native.GO_OK
    assert status.value == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
