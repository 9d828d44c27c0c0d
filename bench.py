"""CDKLM16 throughput benchmark (Gcell-steps/s and fraction of HBM peak).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload grf4096|bump256|ensemble100|adjoint512] [--no-secondary]

A "step" is one Heun RK2 time step of the whole grid (two sub-step
launches).  The default workload is the headline single-grid case:
4096 x 4096 cells, dx = dy = 500 m, walls north/south, periodic east/west,
beta plane, Gaussian-random-field bathymetry, 8 Gaussian bumps, uniform
wind, quadratic friction r = 3e-3, synthetic seeded data.  The state
(403 MB for the two buffers) is larger than the 126 MB L2, so no flush is
needed between steps.

On one GPU the grf4096 line also carries "secondary": the batched
ensemble (100 x 512^2 with model-error events, batched vs the
member-by-member loop) and the adjoint (gradient of a 500-step
observation misfit at 512^2 vs the plain forward); --workload ensemble100
or adjoint512 prints those alone.

Prints one JSON line (rank 0).  With N > 1 (torchrun, one rank per GPU)
every rank advances its own replica of the grid: a single grid does not
shard, so the multi-GPU number is N independent replicas (weak scaling).

--impl reference runs the reference's own CDKLM16 kernel (oracle/_ref,
rebuilt for sm_100a from gpu_ocean/SWESimulators/gpu_kernels) with the
reference's launch sequence, on rank 0 only.
"""

import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, os.path.join(ROOT, "gpu-ocean_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

METRIC = "CDKLM16 Gcell-steps/s + % HBM peak; batched ensemble & adjoint vs plain, 1 B200"
UNIT = "Gcell-steps/s"
ALG_BYTES_PER_CELL_STEP = 68.0   # stage 0: 16 read + 12 write; stage 1: 28 read + 12 write


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.nvml = []          # (sm MHz, max sm MHz, reason names) sampled through NVML
        self._h = None

    def _handle(self):
        # NVML handle of the CUDA device (by PCI address; NVML numbers the
        # GPUs of the machine, CUDA those visible to the process)
        if self._h is None:
            import pynvml
            import torch
            pynvml.nvmlInit()
            p = torch.cuda.get_device_properties(self.gpu)
            try:
                bus = "%08X:%02X:%02X.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
                self._h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                self._h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
        return self._h

    def poll(self, event, period_s=0.0005):
        """Samples the clocks through NVML until `event` completes: the
        caller has queued the timed work, so the samples fall inside the
        timed region however short it is."""
        try:
            import pynvml
            h = self._handle()
            bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
            while True:
                done = event.query()
                sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
                r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.nvml.append((float(sm), float(smax), [n for n, b in bits.items() if r & b]))
                if done:
                    break
                time.sleep(period_s)
        except Exception:
            pass

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        for a, b, r in self.nvml:
            sm.append(a)
            smax.append(b)
            reasons.update(r)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


def max_over_ranks(x, world):
    import torch
    if world == 1:
        return x
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_case(name):
    from SWESimulators import SyntheticCases as SC
    return SC.grf4096() if name == "grf4096" else SC.bump256()


def _oracle_rate(n, budget_s, dx=500.0, max_steps=200, seed_bumps=20242, one_stage=False):
    """Gcell-steps/s of the FP64 NumPy restatement on one core for the
    headline physics on an n x n grid: RK2 steps until budget_s has passed
    (at least one), after one untimed step; one_stage times a single RK
    stage and counts it as half a step."""
    from oracle import cdklm16_oracle as O
    from SWESimulators import SyntheticCases as SC
    c = SC.grf(n, dx=dx, steps=1, seed_bumps=seed_bumps)
    sim = O.OracleSim(c.eta0, c.hu0, c.hv0, c.Hi, c.nx, c.ny, c.dx, c.dy, c.dt, c.g, c.f, c.r,
                      coriolis_beta=c.beta, bc=c.bc, wind=c.wind)
    if one_stage:
        t0 = time.perf_counter()
        sim._stage(sim.h0, sim.h1, float(np.float32(c.dt)), 0)
        el = time.perf_counter() - t0
        return c.nx * c.ny * 0.5 / el / 1e9, 0.5, el
    if n <= 1024:
        sim.rk2_step(np.float32(c.dt))    # warm-up
    steps = 0
    t0 = time.perf_counter()
    while True:
        sim.rk2_step(np.float32(c.dt))
        steps += 1
        el = time.perf_counter() - t0
        if el > budget_s or steps >= max_steps:
            break
    return c.nx * c.ny * steps / el / 1e9, steps, el


def _member_proc(args):
    n, budget, m = args
    os.environ["OMP_NUM_THREADS"] = "1"
    return _oracle_rate(n, budget, dx=1000.0, seed_bumps=30000 + m)


def cpu_baseline(workload):
    """FP64 NumPy restatement of the reference kernel (the reference itself has
    no CPU path) on the host cores, on bounded samples of the same physics:
    one core at 512^2 (the reported value), 256^2 and 4096^2 (one RK2 step);
    and the ensemble form, one process per core with one 512^2 member each,
    throughput summed."""
    if workload != "grf4096":
        from oracle import cdklm16_oracle as O
        from SWESimulators import SyntheticCases as SC
        c = SC.bump256()
        sim = O.OracleSim(c.eta0, c.hu0, c.hv0, c.Hi, c.nx, c.ny, c.dx, c.dy, c.dt, c.g, c.f, c.r,
                          coriolis_beta=c.beta, bc=c.bc, wind=c.wind)
        n, t0 = 0, time.perf_counter()
        while True:
            sim.rk2_step(np.float32(c.dt))
            n += 1
            el = time.perf_counter() - t0
            if el > 12.0 or n >= 200:
                break
        return {"value": c.nx * c.ny * n / el / 1e9, "unit": UNIT, "cores": 1, "kind": "port",
                "sample": "FP64 NumPy restatement, bump256, %d RK2 steps, %.1f s, 1 core" % (n, el)}
    cores = os.cpu_count() or 1
    v512, s512, e512 = _oracle_rate(512, 10.0)
    v256, s256, e256 = _oracle_rate(256, 4.0)
    v4k, s4k, e4k = _oracle_rate(4096, 0.0, one_stage=True)
    ens = None
    try:
        import multiprocessing as mproc
        with mproc.get_context("spawn").Pool(cores) as pool:
            t0 = time.perf_counter()
            res = pool.map(_member_proc, [(512, 6.0, m) for m in range(cores)])
            wall = time.perf_counter() - t0
        ens = {"value": float(sum(r[0] for r in res)), "unit": UNIT, "processes": cores,
               "sample": "%d processes, one 512^2 member each (initial state of member m), %d-%d RK2 steps each; "
                         "wall %.1f s" % (cores, min(r[1] for r in res), max(r[1] for r in res), wall)}
    except Exception as e:          # a pool failure must not lose the headline line
        ens = {"error": "%s: %s" % (type(e).__name__, e)}
    return {"value": v512, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "FP64 NumPy restatement, grf4096 physics at 512x512, %d RK2 steps, %.1f s, 1 core, "
                      "host %s (%d cores), OMP_NUM_THREADS=%s"
                      % (s512, e512, os.uname().machine, cores, os.environ.get("OMP_NUM_THREADS", "unset")),
            "by_grid_1core": {"256x256": v256, "512x512": v512, "4096x4096": v4k,
                              "samples": "256^2: %d steps %.1f s; 512^2: %d steps %.1f s; 4096^2: %g step (one stage) %.1f s"
                                         % (s256, e256, s512, e512, s4k, e4k)},
            "ensemble_all_cores": ens}


def load_traffic(cells):
    path = os.path.join(ROOT, "profiles", "cdklm16_stage_traffic.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["dram_bytes_per_cell_per_launch"]) * cells
    except Exception:
        return None


def run_ours(args, world, rank, local):
    import torch
    from SWESimulators import CDKLM16, Common

    c = make_case(args.workload)
    cells = c.nx * c.ny
    ctx = Common.CUDAContext(local)
    sim = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
    if args.rows or args.shape:
        sim._domain.set_launch(args.shape, args.rows)
    if args.arith >= 0:
        sim._domain.set_arith(args.arith)
    stream = sim.gpu_stream
    sim.step(c.dt)                     # first call applies the t == 0 boundary refresh
    for _ in range(args.warmup):
        sim._launch_steps(1, np.float32(c.dt), 0.0)
    barrier(world)
    sampler = ClockSampler(local)
    sampler.start()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    sim._launch_steps(args.steps, np.float32(c.dt), 0.0)
    end.record(stream)
    sampler.poll(end)
    end.synchronize()
    barrier(world)
    clocks = sampler.stop()
    t_ms = max_over_ranks(start.elapsed_time(end), world)
    status = sim.status()

    # end to end through the public API with host buffers
    host = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (c.eta0, c.hu0, c.hv0)]
    sim2 = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
    sim2.step(c.dt)
    warm = sim2.download()             # warm-up download: the page-locked host buffers get cached
    del warm
    torch.cuda.synchronize()
    barrier(world)
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    e_start.record(sim2.gpu_stream)
    sim2.upload(host[0], host[1], host[2])
    for _ in range(args.steps):
        sim2.step(c.dt)
    out = sim2.download()
    e_end.record(sim2.gpu_stream)
    e_end.synchronize()
    barrier(world)
    e_ms = max_over_ranks(e_start.elapsed_time(e_end), world)
    h2d = sum(int(a.numel()) * 4 for a in host)          # upload fills h0; h1 is a device-side copy
    d2h = sum(int(a.size) * 4 for a in out)
    return dict(c=c, cells=cells, t_ms=t_ms, e_ms=e_ms, clocks=clocks, status=status, h2d=h2d, d2h=d2h,
                launches=2 * args.steps * sim._domain.stage_launches(), stage_launches=sim._domain.stage_launches())


def _timed(fn):
    """(result, ms) of fn() between two device syncs, CUDA events."""
    import torch
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record()
    out = fn()
    torch.cuda.synchronize()
    b.record()
    b.synchronize()
    return out, a.elapsed_time(b)


def run_ensemble(ctx, n_members=100, n=512, target_steps=3000, graph_steps=50, plain_steps=600):
    """Batched ensemble (100 members of 512^2, config-2 physics at dx = 1 km,
    shared bathymetry seed 20243): per event every member advances 60 s at
    the common dt, gets model error, and the common dt = 0.7 CFL is
    recomputed.  The batch runs about 3000 steps in one launch of the
    device event-loop graph (one launch per RK stage over all members
    inside it); the member-by-member loop of the reference's ensembles runs
    the first events (about 600 steps) from the same initial states, and
    its states are compared with a batched run of those events."""
    import torch
    from SWESimulators import BatchedEnsemble, CDKLM16, ModelError, SyntheticCases as SC

    c = SC.grf(n, dx=1000.0, seed_bathy=20243, steps=1)

    def members():
        sims = []
        for m in range(n_members):
            s = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
            ModelError.initial_perturbation(s, m)
            sims.append(s)
        torch.cuda.synchronize()
        return sims

    # batched: the whole run is one launch of the event-loop graph
    sims = members()
    batch = BatchedEnsemble.BatchedCDKLM16(sims, graph_steps=graph_steps)
    batch.update_dt(0.7)
    warm = batch.run_events(1, 1)                         # warm-up event (graph capture, scratch)
    per_event = max(warm, 1)
    n_events = max(1, int(round(target_steps / per_event)))
    steps_b, t_b = _timed(lambda: batch.run_events(2, n_events))
    del batch, sims
    # the same members again, batched over the first events only, for the
    # comparison with the member-by-member loop
    n_plain = max(1, int(round(plain_steps / per_event)))
    sims = members()
    batch = BatchedEnsemble.BatchedCDKLM16(sims, graph_steps=graph_steps)
    batch.update_dt(0.7)
    batch.run_events(1, 1 + n_plain)
    snap = [np.stack(s.download()) for s in sims]
    del batch, sims
    # plain member-by-member loop over the first events
    plain = members()
    lims = []
    for s in plain:
        s.updateDt(courant_number=1.0)
        lims.append(s.dt)
    dt = np.float32(0.7 * float(min(lims)))

    def plain_events(e0, ne):
        nonlocal dt
        steps = 0
        for e in range(e0, e0 + ne):
            n0 = plain[0].num_iterations
            for m, s in enumerate(plain):
                s.dt = dt
                s.step(60.0)
                ModelError.model_error(s, m, e)
            steps += plain[0].num_iterations - n0
            lim = []
            for s in plain:
                s.updateDt(courant_number=1.0)
                lim.append(s.dt)
            dt = np.float32(0.7 * float(min(lim)))
        return steps

    plain_events(1, 1)
    steps_p, t_p = _timed(lambda: plain_events(2, n_plain))
    same = all(np.array_equal(a, np.stack(y.download())) for a, y in zip(snap, plain))
    cells = n_members * n * n
    vb = cells * steps_b / (t_b * 1e-3) / 1e9
    vp = cells * steps_p / (t_p * 1e-3) / 1e9
    return {"workload": "ensemble100", "members": n_members, "grid": "%dx%d" % (n, n),
            "events": n_events, "graph_launches": 1, "steps": steps_b, "batched_gcell_steps_s": vb,
            "plain_loop_gcell_steps_s": vp, "plain_loop_steps": steps_p, "speedup": vb / vp,
            "batched_ms": t_b, "plain_ms": t_p, "identical_states": bool(same), "graph_steps": graph_steps,
            "note": "per event: 60 s of steps at the common dt, model error (Philox GRF, std 0.05 m, corr 15 "
                    "cells), dt = 0.7 CFL min over members; the timed batched run is one launch of the "
                    "device event-loop graph (go_batch_run_events); the member-by-member loop and a second "
                    "batched run from the same perturbed states are compared after their common events"}


def run_mixed(ctx, n_domains=64, steps=3000, graph_steps=50, plain_steps=300):
    """Mixed batch: 64 independent domains with nx, ny drawn uniformly from
    {128, 256, ..., 1024} (default_rng(20244)), config-2 physics at dx = 1 km,
    each with its own GRF bathymetry (seed 40000 + k) and bumps, stepped at
    its own CFL time step.  The batch runs 3000 steps; the member-by-member
    loop (CDKLM16.step of each domain in turn) runs 300, and both states are
    compared after those."""
    import torch
    from SWESimulators import BatchedEnsemble, CDKLM16, SyntheticCases as SC

    rng = np.random.default_rng(20244)
    sizes = rng.choice(np.arange(128, 1025, 128), size=(n_domains, 2))

    def domains():
        sims = []
        for k, (nx, ny) in enumerate(sizes):
            c = SC.grf(int(nx), ny=int(ny), dx=1000.0, seed_bathy=40000 + k, seed_bumps=41000 + k, steps=1)
            sims.append(CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs()))
        torch.cuda.synchronize()
        return sims

    sims = domains()
    batch = BatchedEnsemble.BatchedCDKLM16(sims, graph_steps=graph_steps)
    batch.advance(graph_steps)                              # warm-up (graph, TMA maps)
    _, t1 = _timed(lambda: batch.advance(plain_steps))
    snap = [np.stack(s.download()) for s in sims]
    _, t2 = _timed(lambda: batch.advance(steps - plain_steps))
    plain = domains()
    for s in plain:
        for _ in range(graph_steps):
            s.step(s.dt)

    def plain_loop(k):
        for _ in range(k):
            for s in plain:
                s.step(s.dt)

    plain_loop(0)
    _, tp = _timed(lambda: plain_loop(plain_steps))
    same = all(np.array_equal(a, np.stack(y.download())) for a, y in zip(snap, plain))
    cells = int(np.sum(sizes[:, 0] * sizes[:, 1]))
    vb = cells * steps / ((t1 + t2) * 1e-3) / 1e9
    vp = cells * plain_steps / (tp * 1e-3) / 1e9
    return {"workload": "mixed64", "domains": n_domains, "cells_per_step": cells,
            "sizes": "nx, ny in {128, ..., 1024}, default_rng(20244)", "steps": steps,
            "batched_gcell_steps_s": vb, "plain_loop_gcell_steps_s": vp, "plain_loop_steps": plain_steps,
            "speedup": vb / vp, "batched_ms": t1 + t2, "plain_ms": tp, "identical_states": bool(same),
            "graph_steps": graph_steps}


def run_drifters(ctx, n_drifters=100000, steps=100):
    """Drifters on the headline 4096^2 case: the drift launch alone
    (drifter-steps/s, one thread per drifter plus the observation row) and
    CDKLM16.step(dt) with and without the drifters attached."""
    import torch
    from SWESimulators import CDKLM16, Common
    from SWESimulators.GPUDrifterCollection import GPUDrifterCollection

    c = make_case("grf4096")
    sim = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
    sim.step(c.dt)
    stream = sim.gpu_stream

    def timed(fn):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b)

    timed(lambda: [sim.step(c.dt) for _ in range(5)])
    plain_ms = timed(lambda: [sim.step(c.dt) for _ in range(steps)])
    Lx, Ly = c.nx * c.dx, c.ny * c.dy
    d = GPUDrifterCollection(ctx, n_drifters, boundaryConditions=Common.BoundaryConditions(*c.bc),
                             domain_size_x=Lx, domain_size_y=Ly, gpu_stream=stream)
    rng = np.random.default_rng(7)
    d.setDrifterPositions(np.stack([rng.uniform(0.05, 0.95, n_drifters) * Lx,
                                    rng.uniform(0.05, 0.95, n_drifters) * Ly], axis=1))
    d.setObservationPosition([0.5 * Lx, 0.5 * Ly])
    g = sim.gpu_data

    def drift_only():
        for _ in range(steps):
            d.drift(g.h0, g.hu0, g.hv0, sim.bathymetry.Bm, c.nx, c.ny, sim.t, c.dx, c.dy, np.float32(c.dt), 2, 2)

    timed(drift_only)
    drift_ms = timed(drift_only)
    sim.attachDrifters(d)
    timed(lambda: [sim.step(c.dt) for _ in range(5)])
    with_ms = timed(lambda: [sim.step(c.dt) for _ in range(steps)])
    return {"workload": "drifters", "grid": "4096x4096", "drifters": n_drifters, "steps": steps,
            "drift_us_per_launch": 1e3 * drift_ms / steps,
            "drifter_steps_per_s": n_drifters * steps / (drift_ms * 1e-3),
            "step_ms_plain": plain_ms / steps, "step_ms_with_drifters": with_ms / steps,
            "overhead": with_ms / plain_ms - 1.0,
            "note": "CUDA events on the simulator's stream; drifters uniform over the interior; the step loop "
                    "launches each step separately once drifters are attached (as CDKLM16.step does)"}


def run_open_bc(ctx, steps=100, sponge=10):
    """Open boundaries on the headline 4096^2 physics: flow relaxation over
    10-cell sponges on all four sides towards a time-interpolated exterior
    solution, against the same grid with walls, CDKLM16.step(dt) per step."""
    import torch
    from SWESimulators import CDKLM16, Common

    c = make_case("grf4096")
    rng = np.random.default_rng(11)

    def side(n):
        lev = [[(rng.uniform(-0.2, 0.2) * np.ones((1, n))).astype(np.float32) for _ in range(3)] for _ in range(2)]
        return Common.SingleBoundaryConditionData(h=[lev[0][0], lev[1][0]], hu=[lev[0][1], lev[1][1]],
                                                  hv=[lev[0][2], lev[1][2]])

    def timed(sim):
        stream = sim.gpu_stream
        sim.step(c.dt)
        for _ in range(5):
            sim.step(c.dt)
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            sim.step(c.dt)
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / steps

    kw = c.kwargs()
    kw["boundary_conditions"] = Common.BoundaryConditions(1, 1, 1, 1)
    walls_ms = timed(CDKLM16.CDKLM16(ctx, dt=c.dt, **kw))
    kw["boundary_conditions"] = Common.BoundaryConditions(3, 3, 3, 3, spongeCells={
        "north": sponge, "east": sponge, "south": sponge, "west": sponge})
    kw["boundary_conditions_data"] = Common.BoundaryConditionsData(
        t=[0.0, 1000.0 * c.dt], north=side(c.nx + 4), south=side(c.nx + 4), east=side(c.ny + 4), west=side(c.ny + 4))
    open_ms = timed(CDKLM16.CDKLM16(ctx, dt=c.dt, **kw))
    return {"workload": "open_bc", "grid": "4096x4096", "sponge_cells": sponge, "steps": steps,
            "step_ms_walls": walls_ms, "step_ms_open": open_ms, "overhead": open_ms / walls_ms - 1.0,
            "note": "CUDA events on the simulator's stream; open: relaxation kernels after each RK stage, "
                    "exterior solution interpolated in time, one step per launch"}


def run_model_error(ctx, steps=50, reps=20, n=4096):
    """Stochastic model error on the headline 4096^2 case: CDKLM16.step(dt)
    with small_scale_perturbation (LCG draws, SOAR, geostrophic balance
    after every step) against the plain step, and the perturbation alone
    (draws, SOAR, balance) with its HBM roofline.  Algorithmic bytes per
    cell: draws 12 (seed read and write 16 per pair of cells, 4 written),
    SOAR 8 (xi read, coarse written), balance 32 (coarse, Hi, eta, hu, hv
    read; eta, hu, hv written)."""
    import torch
    from SWESimulators import CDKLM16, Common
    from SWESimulators.OceanStateNoise import OceanStateNoise

    c = make_case("grf4096")
    if n != c.nx:
        from SWESimulators import SyntheticCases as SC
        c = SC.grf(n, dx=c.dx, steps=1)
    peak, _ = measured_peak()

    def timed(stream, fn, n):
        fn()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(n):
            fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / n

    plain = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
    plain_ms = timed(plain.gpu_stream, lambda: plain.step(c.dt), steps)
    del plain
    sim = CDKLM16.CDKLM16(ctx, dt=c.dt, small_scale_perturbation=True, small_scale_perturbation_amplitude=1e-4,
                          use_lcg=True, **c.kwargs())
    with_ms = timed(sim.gpu_stream, lambda: sim.step(c.dt), steps)
    noise = sim.small_scale_model_error
    s = sim.gpu_stream
    draw_ms = timed(s, noise.generateNormalDistribution, reps)
    soar_bal_ms = timed(s, lambda: noise.perturbSim(sim, update_random_field=False), reps)
    all_ms = timed(s, lambda: noise.perturbSim(sim), reps)
    cells = c.nx * c.ny
    traffic = 52.0 * cells
    out = {"workload": "model_error", "grid": "%dx%d" % (c.nx, c.ny), "generator": "lcg", "interpolation_factor": 1,
           "steps": steps, "step_ms_plain": plain_ms, "step_ms_with_model_error": with_ms,
           "cells": cells, "overhead": with_ms / plain_ms - 1.0, "perturb_ms": all_ms, "draws_ms": draw_ms,
           "soar_balance_ms": soar_bal_ms,
           "roofline": {"bound": "hbm", "achieved": traffic / (all_ms * 1e-3) / 1e9, "unit": "GB/s",
                        "bytes_per_cell": 52, "peak": peak,
                        "frac": traffic / (all_ms * 1e-3) / 1e9 / peak},
           "note": "CUDA events on the simulator's stream; perturb = draws + SOAR + balance (3 launches); "
                   "peak = measured copy bandwidth"}
    del sim, noise
    # XORWOW draws (the reference's default generator)
    x = OceanStateNoise(ctx, s, c.nx, c.ny, c.dx, c.dy, Common.BoundaryConditions(*c.bc), False, use_lcg=False,
                        xorwow_seed=1)
    out["xorwow_draws_ms"] = timed(s, x.generateNormalDistribution, reps)
    del x
    out["ensemble"] = run_model_error_ensemble(ctx)
    return out


def run_model_error_ensemble(ctx, members=32, n=512, steps=20):
    """The reference's ensemble with model error (OceanNoiseEnsemble.step:
    every member steps and is perturbed after every step): 32 members of
    512^2, LCG, member by member (CDKLM16.step per member, 5 launches a
    step each) against BatchedCDKLM16.step (2 step launches and 3 model-error
    launches a step for all members, plus the members' boundary updates).
    Wall time around synchronised loops, per step."""
    import time
    import torch
    from SWESimulators import CDKLM16, SyntheticCases as SC
    from SWESimulators.BatchedEnsemble import BatchedCDKLM16

    c = SC.grf(n, dx=1000.0, bc=(2, 2, 2, 2), steps=1)
    sims = [CDKLM16.CDKLM16(ctx, dt=c.dt, small_scale_perturbation=True, small_scale_perturbation_amplitude=1e-4,
                            use_lcg=True, **c.kwargs()) for _ in range(members)]

    def wall(fn):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3 / steps

    loop_ms = wall(lambda: [s.step(steps * c.dt) for s in sims])
    ens = BatchedCDKLM16(sims)
    batched_ms = wall(lambda: ens.step(steps * c.dt))
    cells = members * n * n
    return {"members": members, "grid": "%dx%d" % (n, n), "steps": steps, "loop_ms_per_step": loop_ms,
            "batched_ms_per_step": batched_ms, "speedup": loop_ms / batched_ms,
            "batched_gcell_steps_s": cells / (batched_ms * 1e-3) / 1e9,
            "loop_gcell_steps_s": cells / (loop_ms * 1e-3) / 1e9,
            "note": "wall clock around synchronised loops; model error after every step"}


def run_adjoint(ctx, n=512, n_steps=500, k=50, kind=0, rows=0):
    """Gradient of the observation misfit (64 cells, steps 50..500, truth
    bumps seed 50001, background 50002) w.r.t. the initial state and the
    wind field, against the plain forward run of the same 500 steps."""
    import torch
    from SWESimulators import Adjoint, CDKLM16, SyntheticCases as SC, _native

    c = SC.grf(n, dx=1000.0, seed_bumps=50002, steps=1)
    ct = SC.grf(n, dx=1000.0, seed_bumps=50001, steps=1)
    sim = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
    truth = CDKLM16.CDKLM16(ctx, dt=c.dt, **ct.kwargs())
    rng = np.random.default_rng(50003)
    flat = rng.choice((n - 4) * (n - 4), size=64, replace=False)
    ij = np.stack([2 + flat % (n - 4), 2 + flat // (n - 4)], axis=1)
    steps = list(range(50, n_steps + 1, 50))
    states = {}
    for s in range(1, n_steps + 1):
        truth.step(c.dt)
        if s in steps:
            states[s] = truth.download(interior_domain_only=True)
    obs = Adjoint.Observations(ij, steps, Adjoint.Observations.sample(states, ij))
    x0 = [torch.as_tensor(np.ascontiguousarray(a), device="cuda") for a in sim.download(interior_domain_only=True)]
    X = torch.full((n, n), float(c.wind[0]), device="cuda")
    Y = torch.full((n, n), float(c.wind[1]), device="cuda")
    out = {"workload": "adjoint512", "grid": "%dx%d" % (n, n), "steps": n_steps, "observations": "64 cells x 10"}
    for kk, tag in ((k, "k%d" % k), (n_steps, "store_all")):
        prob = Adjoint.MisfitProblem(sim, n_steps, obs, dt=c.dt, checkpoint_every=kk)
        _native.check(_native.load().go_domain_set_adjoint_launch(prob.domain.handle, int(kind), int(rows)))
        prob.gradient(*x0, X, Y)                      # warm-up
        best_g, best_p = None, None
        for _ in range(3):
            prob._load(*x0, X, Y)
            prob.stream.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(prob.stream)
            prob._plain_steps(n_steps)
            b.record(prob.stream)
            b.synchronize()
            tp = a.elapsed_time(b)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            J, *g = prob.gradient(*x0, X, Y)
            torch.cuda.synchronize()
            tg = 1e3 * (time.perf_counter() - t0)
            best_g = tg if best_g is None else min(best_g, tg)
            best_p = tp if best_p is None else min(best_p, tp)
        out["plain_forward_ms"] = best_p
        out["forward_adjoint_ms_" + tag] = best_g
        out["ratio_" + tag] = best_g / best_p
        out["J"] = J
        del prob
        torch.cuda.empty_cache()
    out["note"] = ("forward+adjoint = forward with checkpoints + misfit, reverse sweep (segment recompute for k=%d; "
                   "none when the whole trajectory is stored); wall clock on the host, plain forward by CUDA events"
                   % k)
    return out


def run_adjoint_batch(ctx, M=32, n=1024, n_steps=1000, obs_every=50, memory_fraction=0.8):
    """Batched adjoint: M members of n^2 (config-2 physics at dx = 1 km,
    initial eta perturbed by the members' GRFs), the misfit of 64 truth
    observations every obs_every steps for every member, gradients w.r.t.
    each member's initial state and wind field, binomial checkpointing over
    whole-ensemble snapshots in memory_fraction of the free HBM.  Reported
    beside the member-by-member forward loop over the same steps."""
    import torch
    from SWESimulators import Adjoint, Autotune, CDKLM16, ModelError, SyntheticCases as SC

    c = SC.grf(n, dx=1000.0, seed_bathy=20243, steps=1)
    ct = SC.grf(n, dx=1000.0, seed_bathy=20243, seed_bumps=50001, steps=1)
    sims = []
    for m in range(M):
        s = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
        ModelError.initial_perturbation(s, m)
        sims.append(s)
    truth = CDKLM16.CDKLM16(ctx, dt=c.dt, **ct.kwargs())
    rng = np.random.default_rng(50003)
    flat = rng.choice((n - 4) * (n - 4), size=64, replace=False)
    ij = np.stack([2 + flat % (n - 4), 2 + flat // (n - 4)], axis=1)
    steps = list(range(obs_every, n_steps + 1, obs_every))
    states = {}
    for k in range(1, n_steps + 1):
        truth.step(c.dt)
        if k in steps:
            states[k] = truth.download(interior_domain_only=True)
    obs = Adjoint.Observations(ij, steps, Adjoint.Observations.sample(states, ij))
    torch.cuda.synchronize()
    xs = torch.stack([torch.stack([torch.as_tensor(np.ascontiguousarray(a), device="cuda")
                                   for a in s.download(interior_domain_only=True)]) for s in sims])
    winds = torch.stack([torch.full((2, n, n), float(c.wind[0]), device="cuda")] * M)
    # member-by-member forward loop over the same steps (the reference's ensemble stepping)
    plain = [CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs()) for _ in range(M)]
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for s in plain:
        s.step(n_steps * np.float64(np.float32(c.dt)) - 1e-6 * float(c.dt))
    torch.cuda.synchronize()
    t1.record()
    t1.synchronize()
    plain_ms = t0.elapsed_time(t1)
    plain_steps = plain[0].num_iterations
    del plain
    torch.cuda.empty_cache()
    bp = Adjoint.BatchedMisfitProblem(sims, n_steps, obs, dt=c.dt, memory_fraction=memory_fraction)
    tune = Autotune.tune_adjoint_batch(bp)
    torch.cuda.synchronize()
    t_start = time.perf_counter()
    J, g, gw = bp.gradient(xs, winds)
    torch.cuda.synchronize()
    grad_ms = 1e3 * (time.perf_counter() - t_start)
    cells = M * n * n
    out = {"workload": "adjoint_batch", "members": M, "grid": "%dx%d" % (n, n), "steps": n_steps,
           "observations": "64 cells x %d" % len(steps), "snapshots": bp.revolve.s,
           "snapshot_gb": bp.snapshot_bytes / 1e9, "forward_steps_in_schedule": bp.revolve.forward_steps(),
           "forward_adjoint_ms": grad_ms, "plain_loop_forward_ms": plain_ms, "plain_loop_steps": plain_steps,
           "ratio_vs_plain_loop": grad_ms / plain_ms * plain_steps / n_steps,
           "forward_adjoint_gcell_steps_s": cells * n_steps / (grad_ms * 1e-3) / 1e9,
           "adjoint_launch": tune, "J_mean": float(np.mean(J)),
           "note": "wall clock around BatchedMisfitProblem.gradient (host-driven schedule); plain loop by "
                   "CUDA events around CDKLM16.step over the same number of steps, member by member"}
    bp.close()
    del bp, sims
    torch.cuda.empty_cache()
    return out


def run_adjoint_stages(ctx, n, reps=20, kind=0, rows=0):
    """Device time of one forward RK2 step (go_traj_step) and of each
    adjoint stage (go_adjoint_stage, fold included) on an n x n grid of the
    headline physics after 3 steps; used for the stage-level comparison and
    as the ncu target."""
    import ctypes
    import torch
    from SWESimulators import Adjoint, CDKLM16, SyntheticCases as SC, _native

    lib = _native.load()
    c = SC.grf(n, dx=1000.0, steps=1)
    sim = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
    for _ in range(3):
        sim.step(c.dt)
    torch.cuda.synchronize()
    prob = Adjoint.MisfitProblem(sim, 1, Adjoint.Observations(np.zeros((0, 2)), [], np.zeros((0, 0, 3))))
    _native.check(lib.go_domain_set_adjoint_launch(prob.domain.handle, int(kind), int(rows)))
    prob.wind[0, :, :n].fill_(float(c.wind[0]))
    prob.wind[1, :, :n].fill_(float(c.wind[1]))
    slab = Adjoint.StateSlab(3, n, n)
    g = sim.gpu_data
    for f, a in enumerate((g.h0, g.hu0, g.hv0)):
        slab.full(0)[f].copy_(a.view)
    lam = Adjoint.StateSlab(3, n, n)
    lam.interior(0).normal_(generator=torch.Generator(device="cuda").manual_seed(5))
    lw = torch.zeros_like(prob.lam_wind)
    torch.cuda.synchronize()
    dt = float(np.float32(c.dt))
    P = _native.ptr
    prob._traj_step(slab, 0, slab, 1, slab, 2)

    def fwd():
        prob._traj_step(slab, 0, slab, 1, slab, 2)

    def adj(k):
        q_in, q_out, l_out, l_in = (1, 2, 0, 1) if k == 1 else (0, 1, 1, 0)
        _native.check(lib.go_adjoint_stage(prob.domain.handle, prob.sh, k, dt, slab.gs(q_in), slab.gs(q_out),
                                           lam.gs(l_out), lam.gs(l_in), lam.gs(2), P(lw[0]), P(lw[1]),
                                           prob.wpitch, P(prob.Hi), prob.Hi_pitch))

    def timed(fn):
        for _ in range(3):
            fn()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(prob.stream)
        for _ in range(reps):
            fn()
        b.record(prob.stream)
        b.synchronize()
        return a.elapsed_time(b) / reps * 1e3

    tf = timed(fwd)
    t1 = timed(lambda: adj(1))
    t0 = timed(lambda: adj(0))
    return {"workload": "adjoint_stage", "grid": "%dx%d" % (n, n), "adjoint_launch": [int(kind), int(rows)],
            "forward_step_us": tf, "adjoint_stage1_us": t1,
            "adjoint_stage0_us": t0, "adjoint_step_over_forward_step": (t0 + t1) / tf, "reps": reps}


def run_reference(args):
    import torch
    from oracle import build_ref, ref_kernel
    from oracle import cdklm16_oracle as O

    cfg_name = "grf4096" if args.workload == "grf4096" else "bump256"
    cfg = build_ref.CONFIGS[cfg_name]
    if not ref_kernel.available(cfg):
        return None, "reference kernel library %s not built" % os.path.basename(build_ref.lib_name(cfg))
    c = make_case(args.workload)
    Hi = O.fix_bi_ghost_corners(c.Hi, c.nx, c.ny, c.bc)
    ref = ref_kernel.RefKernelSim(cfg, c.eta0, c.hu0, c.hv0, Hi, c.dt, c.f, c.beta, c.bc, wind=c.wind)
    ref.step(c.dt)
    for _ in range(args.warmup):
        ref.run_steps(1, np.float32(c.dt))
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    s.record(ref.stream)
    ref.run_steps(args.steps, np.float32(c.dt))
    e.record(ref.stream)
    sampler.poll(e)
    e.synchronize()
    clocks = sampler.stop()
    return dict(c=c, cells=c.nx * c.ny, t_ms=s.elapsed_time(e), clocks=clocks), None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["grf4096", "bump256", "ensemble100", "mixed64", "adjoint512", "adjoint_stage",
                                           "drifters", "open_bc", "adjoint_batch", "model_error"],
                    default="grf4096")
    ap.add_argument("--grid", type=int, default=None,
                    help="grid size of the adjoint_stage (default 2048) and model_error (default 4096) workloads")
    ap.add_argument("--adj-kind", type=int, default=0, help="adjoint launch form (include/gocean.h GO_ADJ_*)")
    ap.add_argument("--adj-rows", type=int, default=0, help="rows per strip of the marching adjoint (0: automatic)")
    ap.add_argument("--rows", type=int, default=0, help="rows per block strip (0: library default)")
    ap.add_argument("--shape", type=int, default=0, help="launch shape 0..8 (include/gocean.h GO_SHAPE_*); with --rows 0 as well, the library default")
    ap.add_argument("--arith", type=int, default=-1,
                    help="quotients: 0 '/' as the reference source, 1 reciprocals (library default)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the batched-ensemble and adjoint measurements added to the grf4096 line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world, rank, local = dist_setup(args.gpus)
    peak, peak_kind = measured_peak()
    config = {"workload": args.workload, "grid": "4096x4096" if args.workload == "grf4096" else "256x256",
              "l2": "state larger than L2 (403 MB), no flush" if args.workload == "grf4096" else
              "state fits L2 (1.6 MB)", "replicas": world}

    if args.impl == "reference":
        if rank != 0:
            return
        r, why = run_reference(args)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return
        value = r["cells"] * args.steps / (r["t_ms"] * 1e-3) / 1e9
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["t_ms"] / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
                "impl": "reference", "clocks": r["clocks"],
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "gpu_ocean cdklm_swe_2D + periodic BC kernels, rebuilt for sm_100a (texture objects), "
                        "reference launch sequence"}
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.workload)
        print(json.dumps(line))
        return

    if args.workload in ("ensemble100", "mixed64", "adjoint512", "adjoint_stage", "adjoint_batch", "drifters",
                         "open_bc", "model_error"):
        if rank != 0:
            return
        from SWESimulators import Common
        ctx = Common.CUDAContext(local)
        sampler = ClockSampler(local)
        sampler.start()
        if args.workload == "ensemble100":
            r = run_ensemble(ctx)
        elif args.workload == "mixed64":
            r = run_mixed(ctx)
        elif args.workload == "adjoint512":
            r = run_adjoint(ctx, kind=args.adj_kind, rows=args.adj_rows)
        elif args.workload == "adjoint_batch":
            r = run_adjoint_batch(ctx)
        elif args.workload == "drifters":
            r = run_drifters(ctx)
        elif args.workload == "open_bc":
            r = run_open_bc(ctx)
        elif args.workload == "model_error":
            r = run_model_error(ctx, n=args.grid or 4096)
        else:
            r = run_adjoint_stages(ctx, args.grid or 2048, reps=args.steps if args.steps < 2000 else 20,
                                   kind=args.adj_kind, rows=args.adj_rows)
        clocks = sampler.stop()
        if args.workload == "adjoint_stage":
            cells = (args.grid or 2048) ** 2
            us = r["adjoint_stage0_us"] + r["adjoint_stage1_us"]
            print(json.dumps({"metric": METRIC, "value": cells / (us * 1e-6) / 1e9, "unit": UNIT, "n_gpus": 1,
                              "steps": r["reps"], "warmup": 3, "ms_per_step": us * 1e-3,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                              "data": "synthetic", "config": {"workload": "adjoint_stage", "grid": r["grid"]},
                              "result": r, "clocks": clocks}))
            return
        if args.workload in ("ensemble100", "mixed64"):
            value, ms = r["batched_gcell_steps_s"], r["batched_ms"] / max(r["steps"], 1)
        elif args.workload == "adjoint_batch":
            value, ms = r["forward_adjoint_gcell_steps_s"], r["forward_adjoint_ms"] / r["steps"]
        elif args.workload == "drifters":
            value, ms = 4096 * 4096 / (r["step_ms_with_drifters"] * 1e-3) / 1e9, r["step_ms_with_drifters"]
        elif args.workload == "open_bc":
            value, ms = 4096 * 4096 / (r["step_ms_open"] * 1e-3) / 1e9, r["step_ms_open"]
        elif args.workload == "model_error":
            value = r["cells"] / (r["step_ms_with_model_error"] * 1e-3) / 1e9
            ms = r["step_ms_with_model_error"]
        else:
            cells_steps = 512 * 512 * r["steps"]
            value, ms = cells_steps / (r["forward_adjoint_ms_k50"] * 1e-3) / 1e9, r["forward_adjoint_ms_k50"] / r["steps"]
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": r["steps"], "warmup": 1,
                "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic", "config": {"workload": args.workload}, "result": r,
                "clocks": clocks}
        print(json.dumps(line))
        return

    r = run_ours(args, world, rank, local)
    if rank != 0:
        return
    cells = r["cells"]
    value = world * cells * args.steps / (r["t_ms"] * 1e-3) / 1e9
    e2e = world * cells * args.steps / (r["e_ms"] * 1e-3) / 1e9
    # per RK stage: the stage's launches (boundary frame, region, ghost
    # columns for the column-pair shape; one kernel otherwise) move the
    # stage's algorithmic bytes together
    stage_s = (r["t_ms"] * 1e-3) / (2 * args.steps)
    achieved = (ALG_BYTES_PER_CELL_STEP / 2.0) * cells / stage_s / 1e9
    traffic = load_traffic(cells)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["t_ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "basis": "68 B/cell-step algorithmic, per RK stage 34 B/cell over the stage's %d "
                                  "launch(es), timed together" % r["stage_launches"]},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": r["h2d"] / args.steps,
                    "d2h_bytes_per_step": r["d2h"] / args.steps,
                    "note": "upload state from pinned host, %d x CDKLM16.step(dt), download; bytes amortised"
                            % args.steps},
            "gpu_launches": r["launches"], "clocks": r["clocks"], "status_word": r["status"]}
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.workload)
    if world == 1 and not args.no_secondary and args.workload == "grf4096":
        from SWESimulators import Common
        ctx = Common.CUDAContext(local)
        secondary = {}
        for name, fn in (("ensemble100", run_ensemble), ("mixed64", run_mixed), ("adjoint512", run_adjoint),
                         ("adjoint_batch", run_adjoint_batch), ("drifters", run_drifters),
                         ("open_bc", run_open_bc), ("model_error", run_model_error)):
            try:
                secondary[name] = fn(ctx)
            except Exception as e:      # a secondary failure must not lose the headline line
                secondary[name] = {"error": "%s: %s" % (type(e).__name__, e)}
        line["secondary"] = secondary
    print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
