"""Additive model error: seeded Gaussian random fields added to eta.

The batched-ensemble workload perturbs each member's surface elevation
once at t = 0 and every 60 s of model time by a correlated Gaussian field
(std 0.05 m, correlation 15 cells).  The field comes from Philox4x32-10
counter-based normals keyed by (key0, key1) with the event number as
counter, Box-Muller, and a separable Gaussian filter
(include/gocean.h go_grf_perturb), so the single-simulator path below and
``BatchedCDKLM16.perturb`` add identical fields: member m of a batch uses
key (key0, m).

The reference's model error (gpu_ocean/SWESimulators/OceanStateNoise.py,
called from OceanNoiseEnsemble.py:506-531 after every member step) draws
its field by another method; this generator is the one the workload
names, not a port of it.
"""

from . import _native

INITIAL_SEED = 30000        # member m's initial perturbation: key (30000 + m, 0), event 0
MODEL_ERROR_SEED = 20245    # model error at event e >= 1: key (20245, m)

# one scratch buffer per device, shared by every perturbation; the event
# recorded after its last use orders the next user (perturbations of
# different members run on the members' own streams)
_scratch = {}


def _scratch_for(n_floats, stream):
    """The device's scratch (at least n_floats), with `stream` ordered after
    its previous user."""
    torch = _native.require_cuda()
    dev = torch.cuda.current_device()
    buf, last = _scratch.get(dev, (None, None))
    if buf is None or buf.numel() < n_floats:
        if last is not None:
            last.synchronize()
        buf = torch.empty(int(n_floats), dtype=torch.float32, device="cuda")
        last = None
    if last is not None:
        stream.wait_event(last)
    _scratch[dev] = (buf, last)
    return buf


def _scratch_used(stream):
    torch = _native.require_cuda()
    dev = torch.cuda.current_device()
    buf, _ = _scratch[dev]
    ev = torch.cuda.Event()
    ev.record(stream)
    _scratch[dev] = (buf, ev)


def perturb(sim, key0, key1, event, std=0.05, corr_cells=15.0):
    """sim.gpu_data.h0 (eta) += std * field(key0, key1, event) on the
    simulator's stream; periodic ghost images are kept consistent."""
    lib = _native.load()
    n = lib.go_grf_scratch_floats(int(sim.nx), int(sim.ny), float(corr_cells))
    if n == 0:
        raise ValueError("invalid grid or correlation length")
    sim.gpu_stream.wait_stream(_native.require_cuda().cuda.current_stream())
    buf = _scratch_for(n, sim.gpu_stream)
    eta = sim.gpu_data.h0
    _native.check(lib.go_grf_perturb(sim._domain.handle, _native.stream_handle(sim.gpu_stream),
                                     _native.ptr(eta.tensor), int(eta.pitch), int(key0) & 0xFFFFFFFF,
                                     int(key1) & 0xFFFFFFFF, int(event) & 0xFFFFFFFF, float(std),
                                     float(corr_cells), _native.ptr(buf), int(buf.numel())))
    _scratch_used(sim.gpu_stream)


def initial_perturbation(sim, member, std=0.05, corr_cells=15.0):
    """Member m's initial eta perturbation (key (30000 + m, 0), event 0)."""
    perturb(sim, INITIAL_SEED + int(member), 0, 0, std, corr_cells)


def model_error(sim, member, event, std=0.05, corr_cells=15.0):
    """Model error of member m at event e >= 1 (key (20245, m))."""
    perturb(sim, MODEL_ERROR_SEED, int(member), int(event), std, corr_cells)
