"""Model error on a GPU (go_grf_perturb, go_batch_grf_perturb): the field
matches the NumPy twin, keeps periodic ghosts consistent, and the batched
pass adds exactly what the member-by-member pass adds."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from SWESimulators import BatchedEnsemble, CDKLM16, Common, ModelError, SyntheticCases as SC  # noqa: E402
from oracle import model_error_oracle as M  # noqa: E402


@pytest.fixture(scope="module")
def ctx():
    return Common.CUDAContext()


def flat_sim(ctx, nx, ny, bc=(1, 2, 1, 2)):
    c = SC.grf(nx, ny=ny, dx=1000.0, bc=bc, steps=1)
    z = np.zeros_like(c.eta0)
    kw = c.kwargs()
    kw.update(eta0=z, hu0=z.copy(), hv0=z.copy())
    return CDKLM16.CDKLM16(ctx, dt=c.dt, **kw)


@pytest.mark.parametrize("nx, ny, bc", [(192, 160, (1, 2, 1, 2)), (130, 96, (2, 2, 2, 2)), (1100, 40, (1, 1, 1, 1))])
def test_field_matches_numpy_twin(ctx, nx, ny, bc):
    sim = flat_sim(ctx, nx, ny, bc)
    ModelError.perturb(sim, 20245, 5, 9, std=0.05, corr_cells=15.0)
    eta = sim.download()[0]
    ref = 0.05 * M.field(nx, ny, 20245, 5, 9, 15.0, periodic_y=(bc[0] == 2))
    err = np.abs(eta[2:ny + 2, 2:nx + 2] - ref).max()
    print("GRF %dx%d: max |gpu - twin| = %.2e (std 0.05)" % (nx, ny, err))
    assert err < 0.05 * 2e-5
    # periodic ghost images follow the interior
    if bc[1] == 2:
        assert np.array_equal(eta[2:ny + 2, 0:2], eta[2:ny + 2, nx:nx + 2])
        assert np.array_equal(eta[2:ny + 2, nx + 2:nx + 4], eta[2:ny + 2, 2:4])
    if bc[0] == 2:
        assert np.array_equal(eta[0:2, 2:nx + 2], eta[ny:ny + 2, 2:nx + 2])


def test_batched_equals_member_by_member(ctx):
    sizes = [(128, 96), (200, 128), (96, 96)]
    single = [flat_sim(ctx, nx, ny) for nx, ny in sizes]
    for m, s in enumerate(single):
        ModelError.model_error(s, m, 4)
    batched = [flat_sim(ctx, nx, ny) for nx, ny in sizes]
    b = BatchedEnsemble.BatchedCDKLM16(batched)
    b.model_error(4)
    b.model_error(5)
    for m, s in enumerate(single):
        ModelError.model_error(s, m, 5)
    torch.cuda.synchronize()
    for a, c in zip(single, batched):
        assert np.array_equal(a.download()[0], c.download()[0])


def test_perturbed_ensemble_steps(ctx):
    """A perturbed member still steps bit-identically in the batch."""
    sims = [flat_sim(ctx, 128, 128) for _ in range(2)]
    alone = [flat_sim(ctx, 128, 128) for _ in range(2)]
    for m in range(2):
        ModelError.initial_perturbation(sims[m], m)
        ModelError.initial_perturbation(alone[m], m)
    b = BatchedEnsemble.BatchedCDKLM16(sims)
    b.advance(5)
    b.model_error(1)
    b.advance(5)
    for m, s in enumerate(alone):
        for _ in range(5):
            s.step(s.dt)
        ModelError.model_error(s, m, 1)
        for _ in range(5):
            s.step(s.dt)
    torch.cuda.synchronize()
    for a, c in zip(sims, alone):
        assert np.array_equal(np.stack(a.download()), np.stack(c.download()))


def test_event_loop_batched_equals_plain_loop(ctx):
    """run_events (batched, graph replays) == the member-by-member loop with
    the same model error and common-dt updates."""
    def members():
        sims = [flat_sim(ctx, 96, 80) for _ in range(3)]
        for m, s in enumerate(sims):
            ModelError.initial_perturbation(s, m)
        return sims
    a = members()
    b = BatchedEnsemble.BatchedCDKLM16(a, graph_steps=4)
    b.update_dt(0.7)
    steps = b.run_events(1, 3, interval=60.0)
    p = members()
    dts = []
    for s in p:
        s.updateDt(courant_number=1.0)
        dts.append(s.dt)
    dt = np.float32(0.7 * float(min(dts)))       # as update_dt: product in FP64, then rounded
    for e in range(1, 4):
        for m, s in enumerate(p):
            s.dt = dt
            s.step(60.0)
            ModelError.model_error(s, m, e)
        lims = []
        for s in p:
            s.updateDt(courant_number=1.0)
            lims.append(s.dt)
        dt = np.float32(0.7 * float(min(lims)))
    torch.cuda.synchronize()
    assert steps == p[0].num_iterations
    for x, y in zip(a, p):
        assert np.array_equal(np.stack(x.download()), np.stack(y.download()))
        assert x.t == y.t


@pytest.mark.parametrize("launch,interval", [(None, 60.0), ((8, 12, 0), 45.5), ((5, 16, 0), 3.0)])
def test_device_event_loop_equals_host_loop(ctx, launch, interval):
    """go_batch_run_events (one graph launch, nested WHILE nodes) == the
    host-driven event loop: states, model times, step counts and the
    common dt, bit for bit; the graph is reused across calls.  An interval
    shorter than dt makes every event one short step."""
    def members():
        sims = [flat_sim(ctx, 96, 80) for _ in range(6)]
        for m, s in enumerate(sims):
            ModelError.initial_perturbation(s, m)
        return sims
    runs = []
    for device in (True, False):
        sims = members()
        b = BatchedEnsemble.BatchedCDKLM16(sims, graph_steps=4, launch=launch)
        b.update_dt(0.7)
        steps = b.run_events(1, 2, interval=interval, device_loop=device)
        steps += b.run_events(3, 3, interval=interval, device_loop=device)
        torch.cuda.synchronize()
        runs.append((steps, sims, float(np.float32(sims[0].dt))))
    (sd, dev, dtd), (sh, host, dth) = runs
    assert sd == sh and dtd == dth
    if interval < 10.0:   # dt is above 10 s on this grid: every event is one short step
        assert sd == 5
    for x, y in zip(dev, host):
        assert np.array_equal(np.stack(x.download()), np.stack(y.download()))
        assert x.t == y.t and x.num_iterations == y.num_iterations
