"""Ensemble sharding across ranks (SWESimulators.Distributed) on the CPU:
two gloo ranks on 127.0.0.1 run the same collectives the GPU path runs over
NCCL (member ownership, all-gather of per-member scalars, global MIN of the
time step, resampling exchanges of member states)."""

import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "gpu-ocean_b200")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime
    if PKG not in sys.path:
        sys.path.insert(0, PKG)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    from SWESimulators import Distributed as D
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n = 7
        mine = D.local_members(n, world, rank)
        gathered = D.gather_member_scalars(n, [10.0 * m + 0.5 for m in mine])
        gmin = D.global_min(100.0 - rank)
        states = {m: [torch.full((3, 4), float(m)), torch.full((2,), float(-m))] for m in mine}
        pairs = [(0, 1), (2, 2), (3, 0), (5, 6), (6, 4)]
        D.exchange_members(n, pairs, states)
        q.put((rank, mine, gathered.tolist(), gmin,
               {m: [float(t.flatten()[0]) for t in states[m]] for m in mine}))
    finally:
        dist.destroy_process_group()


def test_member_ownership_is_a_partition():
    from SWESimulators import Distributed as D
    for n, world in ((7, 2), (100, 8), (3, 4)):
        parts = [D.local_members(n, world, r) for r in range(world)]
        flat = sorted(m for p in parts for m in p)
        assert flat == list(range(n))
        assert all(D.owner(m, world) == r for r, p in enumerate(parts) for m in p)


def test_collectives_on_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        results = sorted(q.get(timeout=120) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [r[1] for r in results] == [[0, 2, 4, 6], [1, 3, 5]]
    for _, _, gathered, gmin, _ in results:
        assert gathered == [10.0 * m + 0.5 for m in range(7)]
        assert gmin == 99.0
    after = {}
    for _, _, _, _, st in results:
        after.update(st)
    # simultaneous semantics: every destination takes its source's state from before the exchange
    expect = {0: 3, 1: 0, 2: 2, 3: 3, 4: 6, 5: 5, 6: 5}
    for m, src in expect.items():
        assert after[m] == [float(src), float(-src)]
