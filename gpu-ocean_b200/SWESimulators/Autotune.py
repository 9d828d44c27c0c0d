"""Autotuner for the CDKLM16 step launches.

Chooses, by timing with CUDA events on the actual workload:
  * for one domain: the launch shape (threads per block and blocks per SM,
    include/gocean.h go_domain_set_launch) and the rows per block strip;
  * for a batch: the same plus the persistent grid size and the number of
    steps per captured CUDA graph.
The state is saved before and restored after the trials, so tuning does not
advance the simulation.  Results are cached in a JSON file keyed by the GPU
name, grid size(s), member count and kernel variant
(GOCEAN_TUNE_CACHE, default ~/.cache/gocean_b200/tune.json).
"""

import json
import os

import numpy as np

from . import _native

DOMAIN_CANDIDATES = [(4, 2), (4, 4), (4, 8), (4, 16), (4, 24), (4, 32), (5, 8), (5, 16), (5, 24), (5, 32),
                     (6, 4), (6, 8), (6, 16), (6, 24), (6, 32), (7, 16), (7, 24), (2, 4), (2, 8), (2, 16),
                     (1, 16), (3, 16), (0, 16), (8, 12), (8, 24), (8, 36), (8, 48)]
BATCH_CANDIDATES = [(4, 16, 0), (4, 32, 0), (5, 16, 0), (5, 24, 0), (5, 32, 0), (6, 16, 0), (6, 24, 0), (6, 32, 0),
                    (7, 32, 0), (2, 32, 0), (1, 16, 0), (5, 32, 148 * 5), (8, 24, 0), (8, 32, 0), (8, 48, 0)]
GRAPH_LENGTHS = [10, 50]


def cache_path():
    return os.environ.get("GOCEAN_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "gocean_b200", "tune.json"))


def _load_cache():
    try:
        with open(cache_path()) as fh:
            return json.load(fh)
    except Exception:
        return {}


def _store_cache(key, value):
    data = _load_cache()
    data[key] = value
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(data, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def _variant(sim):
    return "r%g-lf%d-ws%d" % (float(sim.r), int(getattr(sim, "linear_friction", False)),
                             int(not sim.wind_stress.is_uniform()))


def _device_name():
    torch = _native.require_cuda()
    return torch.cuda.get_device_name(torch.cuda.current_device())


def _snapshot(sims):
    return [[a.tensor.clone() for a in (s.gpu_data.h0, s.gpu_data.hu0, s.gpu_data.hv0,
                                         s.gpu_data.h1, s.gpu_data.hu1, s.gpu_data.hv1)] for s in sims]


def _restore(sims, snap):
    for s, saved in zip(sims, snap):
        for a, t in zip((s.gpu_data.h0, s.gpu_data.hu0, s.gpu_data.hv0,
                         s.gpu_data.h1, s.gpu_data.hu1, s.gpu_data.hv1), saved):
            a.tensor.copy_(t)


def _time(fn, stream, repeats=3):
    torch = _native.require_cuda()
    best = None
    for _ in range(repeats):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        fn()
        e.record(stream)
        e.synchronize()
        t = s.elapsed_time(e)
        best = t if best is None else min(best, t)
    return best


def tune_domain(sim, candidates=None, steps=20, use_cache=True):
    """Best (shape, rows_per_block) for one CDKLM16 simulator; applies it."""
    key = "domain|%s|%dx%d|%s" % (_device_name(), int(sim.nx), int(sim.ny), _variant(sim))
    if use_cache:
        hit = _load_cache().get(key)
        if hit:
            sim._domain.set_launch(*hit["launch"])
            return tuple(hit["launch"]), hit
    torch = _native.require_cuda()
    candidates = candidates or DOMAIN_CANDIDATES
    snap = _snapshot([sim])
    dt = np.float32(sim.dt)
    times = {}
    for shape, rows in candidates:
        sim._domain.set_launch(shape, rows)
        sim._launch_steps(2, dt, 0.0)
        times[(shape, rows)] = _time(lambda: sim._launch_steps(steps, dt, 0.0), sim.gpu_stream)
    torch.cuda.synchronize()
    _restore([sim], snap)
    best = min(times, key=times.get)
    sim._domain.set_launch(*best)
    result = {"launch": list(best), "ms_per_step": times[best] / steps,
              "trials": {"%d/%d" % k: v / steps for k, v in times.items()}}
    _store_cache(key, result)
    return best, result


def tune_batch(batched, candidates=None, graph_lengths=None, steps=20, use_cache=True):
    """Best (shape, rows, blocks) and graph length for a BatchedCDKLM16;
    applies both."""
    sims = batched.sims
    sizes = sorted({(int(s.nx), int(s.ny)) for s in sims})
    key = "batch|%s|n%d|%s|%s" % (_device_name(), len(sims), ";".join("%dx%d" % s for s in sizes[:8]),
                                  _variant(sims[0]))
    if use_cache:
        hit = _load_cache().get(key)
        if hit:
            batched.batch.set_launch(*hit["launch"])
            batched.graph_steps = 0
            if hit.get("graph_steps"):
                batched.capture(hit["graph_steps"])
            return hit
    torch = _native.require_cuda()
    candidates = candidates or BATCH_CANDIDATES
    graph_lengths = graph_lengths or GRAPH_LENGTHS
    snap = _snapshot(sims)
    batched._sync_members()
    times = {}
    for c in candidates:
        batched.batch.set_launch(*c)
        batched.batch.step(1, batched.stream)
        times[c] = _time(lambda: batched.batch.step(steps, batched.stream), batched.stream)
    best = min(times, key=times.get)
    batched.batch.set_launch(*best)
    gtimes = {0: times[best] / steps}
    for g in graph_lengths:
        batched.batch.capture(g, batched.stream)
        batched.batch.replay(batched.stream)
        gtimes[g] = _time(lambda: batched.batch.replay(batched.stream), batched.stream) / g
    torch.cuda.synchronize()
    _restore(sims, snap)
    gbest = min(gtimes, key=gtimes.get)
    batched.graph_steps = 0
    if gbest:
        batched.capture(gbest)
    result = {"launch": list(best), "graph_steps": gbest, "ms_per_step": gtimes[gbest],
              "trials": {"/".join(str(x) for x in k): v / steps for k, v in times.items()},
              "graph_trials": {str(k): v for k, v in gtimes.items()}}
    _store_cache(key, result)
    return result


ADJOINT_BATCH_CANDIDATES = [(128, 32), (128, 16), (64, 32), (64, 16)]


def tune_adjoint_batch(problem, candidates=None, steps=3):
    """Best (block columns, rows per strip) for a BatchedMisfitProblem's
    adjoint step, timed on its current buffers; the adjoint state is saved
    and restored around the trials.  Applies and returns the choice."""
    torch = _native.require_cuda()
    lib = _native.load()
    candidates = candidates or ADJOINT_BATCH_CANDIDATES
    lam, lw = problem.lam.t.clone(), problem.lam_wind.clone()
    times = {}
    for bw, rows in candidates:
        _native.check(lib.go_adjoint_batch_set_launch(problem.adj, int(bw), int(rows)))
        _native.check(lib.go_adjoint_batch_step(problem.adj, problem.sh))
        times[(bw, rows)] = _time(lambda: [_native.check(lib.go_adjoint_batch_step(problem.adj, problem.sh))
                                           for _ in range(steps)], problem.stream) / steps
    best = min(times, key=times.get)
    _native.check(lib.go_adjoint_batch_set_launch(problem.adj, int(best[0]), int(best[1])))
    torch.cuda.synchronize()
    problem.lam.t.copy_(lam)
    problem.lam_wind.copy_(lw)
    return {"launch": list(best), "ms_per_adjoint_step": times[best],
            "trials": {"%d/%d" % k: v for k, v in times.items()}}

