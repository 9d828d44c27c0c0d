"""CDKLM16 throughput benchmark (Gcell-steps/s and fraction of HBM peak).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload grf4096|bump256]

A "step" is one Heun RK2 time step of the whole grid (two sub-step
launches).  The default workload is the headline single-grid case:
4096 x 4096 cells, dx = dy = 500 m, walls north/south, periodic east/west,
beta plane, Gaussian-random-field bathymetry, 8 Gaussian bumps, uniform
wind, quadratic friction r = 3e-3, synthetic seeded data.  The state
(403 MB for the two buffers) is larger than the 126 MB L2, so no flush is
needed between steps.

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

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
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


def cpu_baseline(workload):
    """FP64 NumPy restatement of the reference kernel on one host core, on a
    bounded sample of the same physics (the reference itself has no CPU
    path)."""
    from oracle import cdklm16_oracle as O
    from SWESimulators import SyntheticCases as SC
    c = SC.grf(512, dx=500.0, steps=1) if workload == "grf4096" else SC.bump256()
    sim = O.OracleSim(c.eta0, c.hu0, c.hv0, c.Hi, c.nx, c.ny, c.dx, c.dy, c.dt, c.g, c.f, c.r,
                      coriolis_beta=c.beta, bc=c.bc, wind=c.wind)
    sim.rk2_step(np.float32(c.dt))    # warm-up
    n = 0
    t0 = time.perf_counter()
    while True:
        sim.rk2_step(np.float32(c.dt))
        n += 1
        el = time.perf_counter() - t0
        if el > 12.0 or n >= 200:
            break
    value = c.nx * c.ny * n / el / 1e9
    return {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "FP64 NumPy restatement, %s physics at %dx%d, %d RK2 steps, %.1f s, 1 core, host %s (%d cores)"
            % (workload, c.nx, c.ny, n, el, os.uname().machine, os.cpu_count() or 0)}


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
    end.synchronize()
    barrier(world)
    clocks = sampler.stop()
    t_ms = max_over_ranks(start.elapsed_time(end), world)
    status = sim.status()

    # end to end through the public API with host buffers
    host = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (c.eta0, c.hu0, c.hv0)]
    sim2 = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
    sim2.step(c.dt)
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
    h2d = sum(int(a.numel()) * 4 for a in host) * 2      # upload fills h0 and h1
    d2h = sum(int(a.size) * 4 for a in out)
    return dict(c=c, cells=cells, t_ms=t_ms, e_ms=e_ms, clocks=clocks, status=status, h2d=h2d, d2h=d2h,
                launches=2 * args.steps)


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
    e.synchronize()
    clocks = sampler.stop()
    return dict(c=c, cells=c.nx * c.ny, t_ms=s.elapsed_time(e), clocks=clocks), None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["grf4096", "bump256"], default="grf4096")
    ap.add_argument("--rows", type=int, default=0, help="rows per block strip (0: library default)")
    ap.add_argument("--shape", type=int, default=0, help="launch shape 0..4 (include/gocean.h)")
    ap.add_argument("--arith", type=int, default=-1,
                    help="quotients: 0 '/' as the reference source, 1 reciprocals (library default)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
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

    r = run_ours(args, world, rank, local)
    if rank != 0:
        return
    cells = r["cells"]
    value = world * cells * args.steps / (r["t_ms"] * 1e-3) / 1e9
    e2e = world * cells * args.steps / (r["e_ms"] * 1e-3) / 1e9
    launch_s = (r["t_ms"] * 1e-3) / r["launches"]
    achieved = (ALG_BYTES_PER_CELL_STEP / 2.0) * cells / launch_s / 1e9
    traffic = load_traffic(cells)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["t_ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "basis": "68 B/cell-step algorithmic, per stage launch 34 B/cell"},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": r["h2d"] / args.steps,
                    "d2h_bytes_per_step": r["d2h"] / args.steps,
                    "note": "upload state from pinned host, %d x CDKLM16.step(dt), download; bytes amortised"
                            % args.steps},
            "gpu_launches": r["launches"], "clocks": r["clocks"], "status_word": r["status"]}
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.workload)
    print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
