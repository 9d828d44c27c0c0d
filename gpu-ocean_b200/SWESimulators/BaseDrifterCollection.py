"""Drifter collections: the host-side bookkeeping shared by every drifter
set (gpu_ocean/SWESimulators/BaseDrifterCollection.py:31-425).

A collection holds numDrifters positions plus one observation position
(index numDrifters), in metres from the south-west corner of the interior
domain.  Subclasses store the positions (GPUDrifterCollection keeps them on
the device) and implement get/set and the periodic wrap; the distance,
innovation, weight, mean and resampling arithmetic lives here and runs on
the host in float64, as the reference's does.
"""

import numpy as np

from .Common import BoundaryConditions


class BaseDrifterCollection(object):

    def __init__(self, numDrifters, observation_variance=0.1, boundaryConditions=None,
                 domain_size_x=1.0, domain_size_y=1.0):
        self.numDrifters = int(numDrifters)
        self.obs_index = self.numDrifters
        self.observation_variance = observation_variance
        self.domain_size_x = domain_size_x
        self.domain_size_y = domain_size_y
        self.boundaryConditions = boundaryConditions if boundaryConditions is not None else BoundaryConditions()

    # -- storage, implemented by the subclasses ------------------------------
    def getDrifterPositions(self):
        raise NotImplementedError

    def getObservationPosition(self):
        raise NotImplementedError

    def setDrifterPositions(self, newDrifterPositions):
        raise NotImplementedError

    def setObservationPosition(self, newObservationPosition):
        raise NotImplementedError

    def enforceBoundaryConditions(self):
        raise NotImplementedError

    def copy(self):
        raise NotImplementedError

    def cleanUp(self):
        pass

    def __del__(self):
        try:
            self.cleanUp()
        except Exception:
            pass

    # -- plain attributes ----------------------------------------------------
    def getNumDrifters(self):
        return self.numDrifters

    def getObservationVariance(self):
        return self.observation_variance

    def getBoundaryConditions(self):
        return self.boundaryConditions

    def getDomainSizeX(self):
        return self.domain_size_x

    def getDomainSizeY(self):
        return self.domain_size_y

    def setBoundaryConditions(self, boundaryConditions):
        self.boundaryConditions = boundaryConditions

    def setDomainSize(self, size_x, size_y):
        self.domain_size_x = size_x
        self.domain_size_y = size_y

    # -- initial positions ---------------------------------------------------
    def uniformly_distribute_drifters(self, initialization_cov_drifters=None):
        """Drifters at the cell centres of a near-square grid of
        round(sqrt(n)) rows of ceil(n / rows) cells over the domain, filled
        row by row from the south-west, each then drawn from a normal
        distribution around its centre with the given 2x2 covariance (a
        scalar is a multiple of the identity; none keeps the centres)
        (BaseDrifterCollection.py:147-184)."""
        n = self.getNumDrifters()
        rows = int(np.round(np.sqrt(n)))
        cols = int(np.ceil(1.0 * n / rows))
        ids = np.arange(n)
        positions = np.empty((n, 2))
        positions[:, 0] = (ids % cols + 0.5) * self.domain_size_x / cols
        positions[:, 1] = (ids // cols + 0.5) * self.domain_size_y / rows
        cov = initialization_cov_drifters
        if cov is None:
            cov = np.zeros((2, 2))
        elif np.isscalar(cov):
            cov = np.eye(2) * cov
        cov = np.asarray(cov)
        if cov.shape != (2, 2):
            raise ValueError("initialization_cov_drifters has the wrong shape: " + str(cov))
        if np.any(cov != 0):
            for d in range(n):
                positions[d, :] = np.random.multivariate_normal(positions[d, :], cov)
        self.setDrifterPositions(positions)

    def initializeUniform(self):
        """Drifters uniformly at random over the domain; the observation
        uniformly in its central half (BaseDrifterCollection.py:347-363)."""
        positions = np.random.rand(self.getNumDrifters() + 1, 2)
        positions[-1, :] = positions[-1, :] * 0.5 + 0.25
        positions[:, 0] *= self.domain_size_x
        positions[:, 1] *= self.domain_size_y
        self.setDrifterPositions(positions[:-1, :])
        self.setObservationPosition(positions[-1, :])

    # -- distances to the observation ---------------------------------------
    def _getClosestPositions(self, obs=None):
        """Each drifter's position, or on a periodic axis its image (shifted
        by -L, 0 or +L, the first of the nearest) closest to the observation
        (BaseDrifterCollection.py:186-219)."""
        bc = self.boundaryConditions
        ns, ew = bc.isPeriodicNorthSouth(), bc.isPeriodicEastWest()
        positions = np.array(self.getDrifterPositions(), dtype=np.float64, copy=True)
        if not (ns or ew):
            return positions
        ox, oy = self.getObservationPosition() if obs is None else (obs[0], obs[1])
        for axis, periodic, size, o in ((0, ew, self.getDomainSizeX(), ox), (1, ns, self.getDomainSizeY(), oy)):
            if not periodic:
                continue
            images = positions[:, axis][:, None] + np.array([-size, 0.0, size])[None, :]
            pick = np.argmin(np.abs(images - o), axis=1)
            positions[:, axis] = images[np.arange(images.shape[0]), pick]
        return positions

    def getInnovations(self, obs=None):
        """d = observation - drifter (closest periodic image), n x 2
        (BaseDrifterCollection.py:238-256)."""
        if obs is None:
            obs = self.getObservationPosition()
            closest = self._getClosestPositions()
        else:
            closest = self._getClosestPositions(obs)
        closest[:, 0] = obs[0] - closest[:, 0]
        closest[:, 1] = obs[1] - closest[:, 1]
        return closest

    def getDistances(self, obs=None):
        """Euclidean length of each innovation (BaseDrifterCollection.py:221-236)."""
        d = self.getInnovations(obs)
        return np.sqrt(d[:, 0] ** 2 + d[:, 1] ** 2)

    def getGaussianWeight(self, distances=None, normalize=True):
        """Normal density of the distances with the observation variance
        (BaseDrifterCollection.py:258-272)."""
        if distances is None:
            distances = self.getDistances()
        var = self.getObservationVariance()
        w = (1.0 / np.sqrt(2 * np.pi * var)) * np.exp(-(distances ** 2 / (2 * var)))
        return w / np.sum(w) if normalize else w

    def getCauchyWeight(self, distances=None, normalize=True):
        """Cauchy density of the distances with scale sqrt(variance)
        (BaseDrifterCollection.py:274-288)."""
        if distances is None:
            distances = self.getDistances()
        var = self.getObservationVariance()
        w = 1.0 / (np.pi * np.sqrt(var) * (1 + (distances ** 2 / var)))
        return w / np.sum(w) if normalize else w

    def _enforceBoundaryConditionsOnPosition(self, x, y):
        """A coordinate mapped into the domain by one period (as
        BaseDrifterCollection.py:290-304 does it, including its use of the
        x extent for a negative y)."""
        if x < 0:
            x = self.domain_size_x + x
        if y < 0:
            y = self.domain_size_x + y
        if x > self.domain_size_x:
            x = x - self.domain_size_x
        if y > self.domain_size_y:
            y = y - self.domain_size_y
        return x, y

    def getCollectionMean(self, obs=None):
        """Mean of the closest periodic images, mapped into the domain
        (BaseDrifterCollection.py:306-318)."""
        closest = self._getClosestPositions(obs=obs)
        mx, my = np.mean(closest, axis=0)
        mx, my = self._enforceBoundaryConditionsOnPosition(mx, my)
        return np.array([mx, my])

    def resample(self, newSampleIndices, reinitialization_variance):
        """Drifters replaced by those at newSampleIndices; the first copy of
        each index keeps its position, later copies are drawn around it with
        the given variance; then the periodic wrap
        (BaseDrifterCollection.py:320-345)."""
        old = np.array(self.getDrifterPositions(), dtype=np.float64, copy=True)
        idx = np.asarray(newSampleIndices)
        if self.getNumDrifters() != len(idx):
            raise RuntimeError("ERROR: The size of the new ensemble differs from the old size!\n"
                               "(old size, new size): " + str((self.getNumDrifters(), len(idx))))
        new = np.zeros((len(idx), 2))
        if reinitialization_variance == 0:
            new[:, :] = old[idx, :]
        else:
            seen = np.zeros(self.getNumDrifters(), dtype=bool)
            var = np.eye(2) * reinitialization_variance
            for k, i in enumerate(idx):
                if seen[i]:
                    new[k, :] = np.random.multivariate_normal(old[i, :], var)
                else:
                    new[k, :] = old[i, :]
                    seen[i] = True
        self.setDrifterPositions(new)
        self.enforceBoundaryConditions()

    def plotDistanceInfo(self, title=None):
        raise NotImplementedError("plotting needs matplotlib, which is not available")
