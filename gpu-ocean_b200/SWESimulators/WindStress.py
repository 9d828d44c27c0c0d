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


def sample_at_cells(field, nx, ny):
    """Sample a wind array the way the reference's normalized, bilinear,
    clamped texture lookup does at each interior cell
    (common.cu:616-650 called with ti+0.5, tj+0.5 and NX, NY at
    CDKLM16_kernel.cu:827-828): s = (i+2+0.5)/nx, t = (j+2+0.5)/ny for
    interior indices i, j.  Weights are exact here; the texture unit
    quantises them to 1/256.  Returns an (ny, nx) float32 array."""
    a = np.asarray(field, dtype=np.float64)
    H, W = a.shape
    s = (np.arange(nx) + 2.5) / float(nx)
    t = (np.arange(ny) + 2.5) / float(ny)
    x = s * W - 0.5
    y = t * H - 0.5
    x0 = np.floor(x).astype(np.int64)
    y0 = np.floor(y).astype(np.int64)
    ax = x - x0
    ay = y - y0
    xi0 = np.clip(x0, 0, W - 1)
    xi1 = np.clip(x0 + 1, 0, W - 1)
    yi0 = np.clip(y0, 0, H - 1)
    yi1 = np.clip(y0 + 1, 0, H - 1)
    v00 = a[np.ix_(yi0, xi0)]
    v01 = a[np.ix_(yi0, xi1)]
    v10 = a[np.ix_(yi1, xi0)]
    v11 = a[np.ix_(yi1, xi1)]
    AX = ax[None, :]
    AY = ay[:, None]
    out = (1 - AY) * ((1 - AX) * v00 + AX * v01) + AY * ((1 - AX) * v10 + AX * v11)
    return out.astype(np.float32)
