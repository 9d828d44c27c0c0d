"""Drifters on the GPU (SWESimulators.GPUDrifterCollection, go_drift_*,
go_observe_flow).

* The known answers of the reference's drifter suite
  (gpu_ocean/tests/dataAssimilation/BaseDrifterTest.py) through the device
  collection: default layout, set/get, distances, copy.
* Trajectories: drifters attached to a simulator against the reference's own
  passiveDrifterKernel (oracle/_ref, built with nvcc defaults as the
  reference builds it) driven by the same states, with and without wind
  drift, walls and periodic sides: positions bit for bit.
* The periodic wrap and the flow observation against the reference's
  kernels, bit for bit.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from SWESimulators import CDKLM16, Common, SyntheticCases as SC  # noqa: E402
from SWESimulators.GPUDrifterCollection import GPUDrifterCollection  # noqa: E402
from SWESimulators.WindStress import WindStress  # noqa: E402
from oracle import build_ref, ref_kernel  # noqa: E402

CFG = build_ref.CONFIGS["small_beta"]       # any reference library holds the drifter kernels


@pytest.fixture(scope="module")
def ctx():
    return Common.CUDAContext()


def _ref_available():
    if not ref_kernel.available(CFG):
        pytest.skip("reference kernel library not built")


def test_default_and_small_set(ctx):
    d = GPUDrifterCollection(ctx, 6)
    expect = [[1 / 6, 1 / 4], [3 / 6, 1 / 4], [5 / 6, 1 / 4], [1 / 6, 3 / 4], [3 / 6, 3 / 4], [5 / 6, 3 / 4]]
    np.testing.assert_allclose(d.getDrifterPositions(), expect, atol=1e-6)
    assert d.getObservationPosition().tolist() == [0, 0]
    assert d.getObservationVariance() == 0.01

    s = GPUDrifterCollection(ctx, 3, observation_variance=0.25, boundaryConditions=Common.BoundaryConditions(2, 2, 2, 2))
    s.setDrifterPositions(np.array([[0.9, 0.9], [0.9, 0.1], [0.1, 0.9]]))
    s.setObservationPosition(np.array([0.1, 0.1]))
    np.testing.assert_allclose(s.getDistances(), [np.sqrt(0.08), 0.2, 0.2], atol=1e-6)
    s.setObservationPosition(np.array([0.523, 0.999]))
    np.testing.assert_allclose(s.getDrifterPositions(), [[0.9, 0.9], [0.9, 0.1], [0.1, 0.9]], atol=1e-6)
    np.testing.assert_allclose(s.getObservationPosition(), [0.523, 0.999], atol=1e-6)
    s.setDomainSize(10.3, 5.4)
    c = s.copy()
    moved = s.getDrifterPositions()
    moved[1] = [0.5, 0.5]
    s.setDrifterPositions(moved)
    np.testing.assert_allclose(c.getDrifterPositions()[1], [0.9, 0.1], atol=1e-6)
    assert (c.getDomainSizeX(), c.getDomainSizeY()) == (10.3, 5.4)


def _case(n, bc):
    c = SC.grf(n, dx=500.0, bc=bc, steps=60)
    return c


@pytest.mark.parametrize("bc, wind_factor", [((1, 2, 1, 2), 0.0), ((2, 2, 2, 2), 0.0), ((2, 2, 2, 2), 0.02)])
def test_trajectories_vs_reference_kernel(ctx, bc, wind_factor):
    """300 drifters attached to a 96 x 80 simulation, 60 steps; after each
    step the reference's kernel drifts its own copy through the same state."""
    _ref_available()
    c = SC.grf(96, ny=80, dx=500.0, bc=bc, steps=60)
    kw = c.kwargs()
    rng = np.random.default_rng(5)
    wind = None
    if wind_factor:
        Xw, Yw = (rng.uniform(-5.0, 5.0, (7, 6)).astype(np.float32) for _ in range(2))
        wind = WindStress(t=[0], X=[Xw], Y=[Yw])
    sim = CDKLM16.CDKLM16(ctx, dt=c.dt, **kw)
    Lx, Ly = c.nx * c.dx, c.ny * c.dy
    drifters = GPUDrifterCollection(ctx, 300, boundaryConditions=Common.BoundaryConditions(*bc),
                                    domain_size_x=Lx, domain_size_y=Ly, wind=wind, wind_drift_factor=wind_factor)
    start = np.stack([rng.uniform(0.15, 0.85, 300) * Lx, rng.uniform(0.15, 0.85, 300) * Ly], axis=1)
    obs = np.array([0.5 * Lx, 0.5 * Ly])
    drifters.setDrifterPositions(start)
    drifters.setObservationPosition(obs)
    sim.attachDrifters(drifters)
    ref = ref_kernel.RefDrifters(CFG, drifters.getDrifterPositions(), drifters.getObservationPosition(),
                                 wind_fields=(Xw, Xw, Yw, Yw) if wind_factor else None)
    g = sim.gpu_data
    Bm = sim.bathymetry.Bm
    for _ in range(c.steps):
        t_before = sim.t
        sim.step(c.dt)
        sim.gpu_stream.synchronize()
        # the wind weight GPUDrifterCollection.update_wind gives for one wind time
        wind_t = max(0.0, min(1.0, (t_before - 0.0) / 1.0e-10))
        ref.drift((g.h0.tensor, int(g.h0.pitch)), (g.hu0.tensor, int(g.hu0.pitch)), (g.hv0.tensor, int(g.hv0.pitch)),
                  (Bm.tensor, int(Bm.pitch)), c.nx, c.ny, c.dx, c.dy, np.float32(c.dt), bc[0] == 2, bc[1] == 2,
                  wind_t=np.float32(wind_t), wind_drift_factor=np.float32(wind_factor))
    theirs = ref.positions()
    mine = np.concatenate([drifters.getDrifterPositions(), drifters.getObservationPosition()[None, :]])
    moved = np.abs(mine - np.concatenate([start, obs[None, :]])).max()
    print("bc", bc, "wind", wind_factor, "max displacement %.1f m" % moved,
          "max |mine - reference| %.3g" % np.abs(mine - theirs).max())
    assert moved > 1.0
    assert np.array_equal(mine, theirs)


def test_wrap_and_observation_vs_reference_kernel(ctx):
    _ref_available()
    c = SC.grf(96, ny=80, dx=500.0, bc=(2, 2, 2, 2), steps=5)
    sim = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
    for _ in range(c.steps):
        sim.step(c.dt)
    Lx, Ly = c.nx * c.dx, c.ny * c.dy
    rng = np.random.default_rng(9)
    pos = np.stack([rng.uniform(-0.3, 1.3, 200) * Lx, rng.uniform(-0.3, 1.3, 200) * Ly], axis=1)
    d = GPUDrifterCollection(ctx, 200, boundaryConditions=Common.BoundaryConditions(2, 2, 2, 2),
                             domain_size_x=Lx, domain_size_y=Ly)
    d.setDrifterPositions(pos)
    d.setObservationPosition([1.2 * Lx, -0.1 * Ly])
    ref = ref_kernel.RefDrifters(CFG, d.getDrifterPositions(), d.getObservationPosition())
    d.enforceBoundaryConditions()
    ref.enforce_bc(Lx, Ly, True, True)
    mine = np.concatenate([d.getDrifterPositions(), d.getObservationPosition()[None, :]])
    assert np.array_equal(mine, ref.positions())
    assert mine[:, 0].min() >= 0 and mine[:, 0].max() <= Lx and mine[:, 1].min() >= 0 and mine[:, 1].max() <= Ly
    g = sim.gpu_data
    o_mine = d.observeUnderlyingFlow(g.hu0, g.hv0, c.nx, c.ny, c.dx, c.dy)
    o_ref = ref.observe((g.h0.tensor, int(g.h0.pitch)), (g.hu0.tensor, int(g.hu0.pitch)),
                        (g.hv0.tensor, int(g.hv0.pitch)), c.nx, c.ny, c.dx, c.dy)
    assert o_mine.shape == (200, 2)
    assert np.array_equal(o_mine, o_ref)
    assert np.abs(o_mine).max() > 0
