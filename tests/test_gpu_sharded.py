"""ShardedEnsemble (SWESimulators/Distributed.py) end to end: two gloo ranks
that share the one GPU each step their round-robin half of a 6-member
ensemble with one batched launch per RK stage, agree on the common time
step (MIN all-reduce) at every model-error event, and exchange member
states for a resampling, as MPIOceanModelEnsemble.py:166-258, 424 does
with mpi4py.  The union of both ranks' members must equal the same
schedule run by one rank over all members, bit for bit.

The two ranks' kernels never wait on one another: each rank runs its own
batch; the collectives travel through host memory over gloo."""

import os
import socket
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "gpu-ocean_b200")

N_MEMBERS = 6
PAIRS = [(0, 3), (1, 2), (4, 4), (5, 0)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _run_schedule(ens):
    """update_dt, two events, a resampling, one more event; the states."""
    dt0 = float(ens.update_dt(0.7))
    steps = ens.run_events(1, 2, interval=60.0)
    ens.resample(PAIRS)
    steps += ens.run_events(3, 1, interval=60.0)
    torch.cuda.synchronize()
    nx4 = ens.sims[0].nx + 4 if ens.sims else 0   # the arrays' rows are padded beyond the nx + 4 cells
    return dt0, steps, {m: [t.cpu().numpy()[:, :nx4].copy() for t in ts] for m, ts in ens.states().items()}


def _maker():
    from SWESimulators import CDKLM16, Common, ModelError, SyntheticCases as SC
    ctx = Common.CUDAContext(0)
    c = SC.grf(64, dx=1000.0, seed_bathy=20243, steps=1)

    def make(m):
        s = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
        ModelError.initial_perturbation(s, m)
        return s
    return make


def _worker(rank, world, port, q):
    import datetime
    if PKG not in sys.path:
        sys.path.insert(0, PKG)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from SWESimulators import Distributed as D
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        ens = D.ShardedEnsemble(_maker(), N_MEMBERS)
        q.put((rank,) + _run_schedule(ens))
        del ens
    except Exception as e:   # reported to the parent, which fails the test
        q.put((rank, "error", repr(e), None))
    finally:
        dist.destroy_process_group()


def test_sharded_ensemble_equals_one_rank():
    import torch.multiprocessing as mp
    from SWESimulators import Distributed as D
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = {}
    try:
        for _ in range(2):
            r = q.get(timeout=600)
            results[r[0]] = r[1:]
    finally:
        for p in procs:
            p.join(timeout=120)
            if p.is_alive():
                p.terminate()
    for r in (0, 1):
        assert results[r][0] != "error", results[r]
    # one rank over all members, same schedule
    ens1 = D.ShardedEnsemble(_maker(), N_MEMBERS)
    assert ens1.world == 1 and ens1.members == list(range(N_MEMBERS))
    dt1, steps1, states1 = _run_schedule(ens1)
    for r in (0, 1):
        dt, steps, states = results[r]
        assert dt == dt1 and steps == steps1
        assert sorted(states) == D.local_members(N_MEMBERS, 2, r)
        for m, arrs in states.items():
            for f, (a, b) in enumerate(zip(arrs, states1[m])):
                where = np.argwhere(a != b)
                assert where.size == 0, (r, m, f, where[:6].tolist(), a[tuple(where[0])], b[tuple(where[0])])
    # the resampling really moved states: member 3 started from member 0's
    assert not np.array_equal(states1[3][0], states1[1][0])
