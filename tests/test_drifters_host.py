"""Host-side drifter bookkeeping (SWESimulators.BaseDrifterCollection) on
the CPU, against the known answers of the reference's drifter test suite
(gpu_ocean/tests/dataAssimilation/BaseDrifterTest.py:50-380): default
layout, distances, innovations and the collection mean under every
combination of periodic boundaries, a changed domain size, resampling.

The collection here stores its positions in a NumPy array (a test double of
the device collection); GPU tests run the same answers through
GPUDrifterCollection."""

import numpy as np
import pytest

from SWESimulators.BaseDrifterCollection import BaseDrifterCollection
from SWESimulators.Common import BoundaryConditions


class HostDrifters(BaseDrifterCollection):
    def __init__(self, n, **kw):
        super().__init__(n, **kw)
        self._pos = np.zeros((n + 1, 2))
        self.uniformly_distribute_drifters()

    def getDrifterPositions(self):
        return self._pos[:-1].copy()

    def getObservationPosition(self):
        return self._pos[-1].copy()

    def setDrifterPositions(self, p):
        self._pos[:-1] = np.asarray(p).reshape(-1, 2)

    def setObservationPosition(self, o):
        self._pos[-1] = np.asarray(o).reshape(2)

    def enforceBoundaryConditions(self):
        for k in range(self._pos.shape[0]):
            self._pos[k] = self._enforceBoundaryConditionsOnPosition(*self._pos[k])


SMALL = np.array([[0.9, 0.9], [0.9, 0.1], [0.1, 0.9]])
OBS = np.array([0.1, 0.1])


def small_set():
    d = HostDrifters(3, observation_variance=0.25, boundaryConditions=BoundaryConditions(2, 2, 2, 2))
    d.setDrifterPositions(SMALL)
    d.setObservationPosition(OBS)
    return d


def test_default_layout():
    d = HostDrifters(6)
    expect = [[1 / 6, 1 / 4], [3 / 6, 1 / 4], [5 / 6, 1 / 4], [1 / 6, 3 / 4], [3 / 6, 3 / 4], [5 / 6, 3 / 4]]
    np.testing.assert_allclose(d.getDrifterPositions(), expect, atol=1e-6)
    assert d.getObservationPosition().tolist() == [0, 0]
    bc = d.getBoundaryConditions()           # (BoundaryConditions.get() raises in the reference too)
    assert (bc.north, bc.east, bc.south, bc.west) == (1, 1, 1, 1)
    assert (d.getDomainSizeX(), d.getDomainSizeY()) == (1.0, 1.0)


@pytest.mark.parametrize("bc, distances, innovations", [
    ((2, 2, 2, 2), [np.sqrt(0.08), 0.2, 0.2], [[0.2, 0.2], [0.2, 0.0], [0.0, 0.2]]),
    ((1, 1, 1, 1), [np.sqrt(1.28), 0.8, 0.8], [[-0.8, -0.8], [-0.8, 0.0], [0.0, -0.8]]),
    ((1, 2, 1, 2), [np.sqrt(0.68), 0.2, 0.8], [[0.2, -0.8], [0.2, 0.0], [0.0, -0.8]]),
    ((2, 1, 2, 1), [np.sqrt(0.68), 0.8, 0.2], [[-0.8, 0.2], [-0.8, 0.0], [0.0, 0.2]]),
])
def test_distances_and_innovations(bc, distances, innovations):
    d = small_set()
    d.setBoundaryConditions(BoundaryConditions(*bc))
    np.testing.assert_allclose(d.getDistances(), distances, atol=1e-6)
    np.testing.assert_allclose(d.getInnovations(), innovations, atol=1e-6)


def test_collection_mean():
    d = small_set()
    np.testing.assert_allclose(d.getCollectionMean(), [1 - 0.1 / 3, 1 - 0.1 / 3], atol=1e-6)
    d.setBoundaryConditions(BoundaryConditions(1, 1, 1, 1))
    np.testing.assert_allclose(d.getCollectionMean(), [1.9 / 3, 1.9 / 3], atol=1e-6)
    d.setBoundaryConditions(BoundaryConditions(2, 1, 2, 1))
    np.testing.assert_allclose(d.getCollectionMean(), [1.9 / 3, 1 - 0.1 / 3], atol=1e-6)


def test_domain_size_changes_periodic_distances():
    d = small_set()
    d.setDomainSize(10.3, 5.4)
    np.testing.assert_allclose(d.getDistances(), [np.sqrt(1.28), 0.8, 0.8], atol=1e-6)


def test_weights_and_resample():
    d = small_set()
    g = d.getGaussianWeight()
    c = d.getCauchyWeight()
    assert abs(g.sum() - 1) < 1e-12 and abs(c.sum() - 1) < 1e-12
    assert np.argmax(g) == 1 or np.isclose(g[1], g.max())
    d.resample([1, 1, 2], 0.0)
    np.testing.assert_allclose(d.getDrifterPositions(), SMALL[[1, 1, 2]])
    with pytest.raises(RuntimeError):
        d.resample([0, 1], 0.0)


def test_initialize_uniform_inside_domain():
    d = HostDrifters(1000, domain_size_x=10.3, domain_size_y=5.4)
    np.random.seed(3)
    d.initializeUniform()
    p = d.getDrifterPositions()
    assert p[:, 0].min() >= 0 and p[:, 0].max() <= 10.3
    assert p[:, 1].min() >= 0 and p[:, 1].max() <= 5.4


def test_drifter_cells_for_the_misfit():
    # Observations.drifter_cells: floor(x / dx) in float32 as the observation
    # kernel reads its cell, clamped to the interior at the east/north edge
    from SWESimulators.Adjoint import Observations
    dx, dy, nx, ny = 500.0, 400.0, 10, 8
    pos = np.array([[0.0, 0.0], [3 * dx, 2 * dy], [3 * dx - 1e-3, 2 * dy - 1e-3], [nx * dx, ny * dy],
                    [4.5 * dx, 7.99 * dy]])
    cells = Observations.drifter_cells(pos, nx, ny, dx, dy)
    assert cells.tolist() == [[0, 0], [3, 2], [2, 1], [nx - 1, ny - 1], [4, 7]]
    assert Observations.drifter_cells(pos.reshape(1, 5, 2), nx, ny, dx, dy).shape == (1, 5, 2)
