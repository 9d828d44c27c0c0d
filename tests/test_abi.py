"""The C ABI library: builds, loads, exports every entry point declared in
include/gocean.h, and rejects invalid arguments before touching a GPU."""

import ctypes
import os
import re

import pytest

from SWESimulators import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gocean.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(go_[a-z0-9_A-Z]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_native.LIB_PATH):
        import subprocess
        import sys
        subprocess.run([sys.executable, os.path.join(ROOT, "gpu-ocean_b200", "build.py")], check=True)
    return _native.load()


def test_header_declares_the_bound_functions():
    names = declared_functions()
    assert set(names) == set(_native.SIGNATURES), (set(names) ^ set(_native.SIGNATURES))


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_checked_index_library_exports_every_declared_symbol(lib):
    """lib/libgocean_debug.so (the stage kernels built with
    -DGO_DEBUG_BOUNDS) is a drop-in for lib/libgocean.so."""
    path = os.path.join(ROOT, "gpu-ocean_b200", "lib", "libgocean_debug.so")
    if not os.path.exists(path):
        import subprocess
        import sys
        subprocess.run([sys.executable, os.path.join(ROOT, "gpu-ocean_b200", "build.py")], check=True)
    dbg = ctypes.CDLL(path)
    for name in declared_functions():
        assert hasattr(dbg, name), name


def test_version_and_empty_error(lib):
    assert b"sm_100a" in lib.go_version()
    assert isinstance(lib.go_last_error(), bytes)


def _desc(**kw):
    d = _native.GoDomainDesc()
    d.nx, d.ny = 64, 48
    d.dx = d.dy = 100.0
    d.g = 9.81
    d.theta = 1.3
    d.desing_eps = d.flux_slope_eps = 0.1
    d.depth_cutoff = 1e-5
    d.rk_order = 2
    d.bc_north = d.bc_east = d.bc_south = d.bc_west = 1
    d.north_y = 1.0
    for k, v in kw.items():
        setattr(d, k, v)
    return d


@pytest.mark.parametrize("kw, code", [
    (dict(nx=2), _native.GO_OK - 1),
    (dict(dx=0.0), -1),
    (dict(r=-1.0), -1),
    (dict(rk_order=3), -3),
    (dict(bc_north=5), -3),          # no boundary kind 5
    (dict(bc_north=2), -1),          # periodic on one side only
    (dict(friction_law=7), -1),
])
def test_invalid_domains_rejected(lib, kw, code):
    h = ctypes.c_void_p()
    rc = lib.go_domain_create(ctypes.byref(_desc(**kw)), ctypes.byref(h))
    assert rc == code
    assert h.value is None
    assert len(lib.go_last_error()) > 0


def test_null_arguments_rejected(lib):
    assert lib.go_domain_create(None, None) == -1
    assert lib.go_domain_destroy(None) == 0
    assert lib.go_cdklm_step(None, None, 1, 1.0, 0.0, None, None, None, 4, None, None, None, 4, None, 4, 1e20) == -1
    assert lib.go_max_dt(None, None, None, None, None, 4, None, 4, 1e20, None) == -1


def test_pack_bc_matches_reference_layout():
    # CDKLM16.py:620-624: north<<24 | south<<16 | east<<8 | west
    assert _native.pack_bc(1, 2, 3, 4) == (1 << 24) | (3 << 16) | (2 << 8) | 4
