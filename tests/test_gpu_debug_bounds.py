"""The checked-index build (lib/libgocean_debug.so, GO_DEBUG_BOUNDS): on
small and ragged grids, every boundary combination, every launch shape and
a mixed batch, no global access or shared ring read of the stage kernels
falls outside its array (no GO_STATUS_BOUNDS), and the results are the bits
of the normal build."""

import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from SWESimulators import _native  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
DEBUG_LIB = os.path.join(os.path.dirname(HERE), "gpu-ocean_b200", "lib", "libgocean_debug.so")


def _run(tmp_path, debug):
    out = str(tmp_path / ("debug.npz" if debug else "plain.npz"))
    env = dict(os.environ)
    env["GOCEAN_DEBUG_BOUNDS"] = "1" if debug else "0"
    subprocess.run([sys.executable, os.path.join(HERE, "bounds_cases.py"), out], check=True, env=env,
                   timeout=600)
    return np.load(out)


def test_checked_indices_stay_in_bounds_and_change_nothing(tmp_path):
    if not os.path.exists(DEBUG_LIB):
        pytest.skip("lib/libgocean_debug.so not built")
    dbg = _run(tmp_path, True)
    plain = _run(tmp_path, False)
    assert sorted(dbg.files) == sorted(plain.files)
    for key in dbg.files:
        if key.endswith("_status"):
            assert int(dbg[key]) & _native.GO_STATUS_BOUNDS == 0, key
            assert int(dbg[key]) == int(plain[key]), key
        else:
            assert np.array_equal(dbg[key], plain[key]), key
