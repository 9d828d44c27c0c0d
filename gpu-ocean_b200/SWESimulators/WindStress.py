"""Wind stress forcing, gpu_ocean/SWESimulators/WindStress.py:34-65.

``X`` and ``Y`` are lists of 2-D float32 arrays of kinematic wind stress
(N/m^2 divided by the water density), one per time in ``t``.  1x1 arrays
are uniform wind.
"""

import numpy as np


class WindStress:

    def __init__(self, source_filename=None, t=None, X=None, Y=None):
        self.source_filename = source_filename
        self.t = [0]
        self.X = [np.zeros((1, 1), dtype=np.float32, order='C')]
        self.Y = [np.zeros((1, 1), dtype=np.float32, order='C')]
        self.numWindSteps = 1
        if t is not None:
            assert X is not None, "missing wind forcing X"
            assert Y is not None, "missing wind forcing Y"
            assert len(t) == len(X), str(len(t)) + " vs " + str(len(X))
            assert len(t) == len(Y), str(len(t)) + " vs " + str(len(Y))
            self.numWindSteps = len(t)
            for i in range(len(X)):
                assert X[i].dtype == 'float32', "Wind data needs to be of type np.float32"
                assert Y[i].dtype == 'float32', "Wind data needs to be of type np.float32"
            self.t = t
            self.X = X
            self.Y = Y

    def is_uniform(self):
        return all(np.asarray(a).size == 1 for a in self.X) and all(np.asarray(a).size == 1 for a in self.Y)


def sample_at_cells(field, nx, ny, stream=None):
    """The wind array sampled at each interior cell of an nx x ny grid the
    way the reference's kernel reads its wind texture (common.cu:616-650
    called with ti+0.5, tj+0.5 and NX, NY at CDKLM16_kernel.cu:827-828):
    a bilinear, clamped, normalised texture lookup at
    ((i+2+0.5)/nx, (j+2+0.5)/ny), done on the GPU by go_sample_wind so the
    texture unit's fixed-point filter weights are the reference's.
    Returns a (ny, nx) float32 device tensor."""
    from . import _native
    torch = _native.require_cuda()
    a = np.ascontiguousarray(np.asarray(field, dtype=np.float32))
    if a.ndim != 2:
        raise ValueError("a wind stress field is a 2-D array")
    out = torch.empty((int(ny), int(nx)), dtype=torch.float32, device="cuda")
    _native.check(_native.load().go_sample_wind(
        _native.stream_handle(stream), a.ctypes.data_as(_native.ctypes.c_void_p), int(a.shape[1]),
        int(a.shape[0]), int(nx), int(ny), _native.ptr(out), int(nx) * 4))
    return out
