"""Ensemble members across GPUs.

One process per GPU (torch.distributed; NCCL on GPUs).  Members and
independent domains shard with no per-step communication: member m lives
on rank m % world and every rank advances its own members with one batched
launch per RK stage.  The only collectives are the ones an ensemble's
data-assimilation analysis needs, which the reference does with mpi4py
(gpu_ocean/SWESimulators/MPIOceanModelEnsemble.py:194-258, 424):

* the common time step: MIN over all members' CFL limits (all_reduce);
* per-member scalars (weights, innovations, misfits): all_gather, ordered
  by global member index;
* resampling: member states copied between ranks (send/recv of the three
  ghost-inclusive arrays).

The helpers take tensors of any device, so the CPU tests run them over the
gloo backend and the GPU path over NCCL.
"""

import numpy as np

from . import _native


def owner(member, world):
    """Rank that holds global member `member`."""
    return int(member) % int(world)


def local_members(n_members, world, rank):
    """Global indices of the members rank `rank` holds (round robin)."""
    return [m for m in range(int(n_members)) if owner(m, world) == int(rank)]


def _dist():
    import torch.distributed as dist
    return dist


def global_min(value, device="cpu", group=None):
    """MIN of a float over all ranks."""
    import torch
    dist = _dist()
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    return float(t.item())


def gather_member_scalars(n_members, local_values, device="cpu", group=None):
    """All ranks' per-member scalars as one array indexed by global member.
    local_values: this rank's values in the order of local_members()."""
    import torch
    dist = _dist()
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    mine = local_members(n_members, world, rank)
    vals = np.asarray(local_values, dtype=np.float64).reshape(-1)
    if vals.size != len(mine):
        raise ValueError("rank %d holds %d members, got %d values" % (rank, len(mine), vals.size))
    per = (int(n_members) + world - 1) // world
    buf = torch.zeros(per, dtype=torch.float64, device=device)
    buf[:vals.size] = torch.as_tensor(vals, device=device)
    if world == 1:
        parts = [buf]
    else:
        parts = [torch.zeros_like(buf) for _ in range(world)]
        dist.all_gather(parts, buf, group=group)
    out = np.zeros(int(n_members))
    for r, p in enumerate(parts):
        host = p.cpu().numpy()
        for k, m in enumerate(local_members(n_members, world, r)):
            out[m] = host[k]
    return out


def exchange_members(n_members, pairs, states, group=None):
    """Resampling: for each (src, dst) pair of global member indices, member
    dst's state becomes member src's.  states: {global member: list of
    tensors} for this rank's members (updated in place).  Pairs whose ends
    are on one rank are copied locally; the others are sent and received
    (every rank walks the pairs in the same order, so the matching
    send/recv calls pair up)."""
    dist = _dist()
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    pending = {}
    for src, dst in pairs:
        rs, rd = owner(src, world), owner(dst, world)
        if rs == rd == rank:
            pending[dst] = [t.clone() for t in states[src]]
    for src, dst in pairs:
        rs, rd = owner(src, world), owner(dst, world)
        if rs == rd:
            continue
        if rank == rs:
            for t in states[src]:
                dist.send(t.contiguous(), dst=rd, group=group)
        elif rank == rd:
            recv = [t.clone() for t in states[dst]]
            for t in recv:
                dist.recv(t, src=rs, group=group)
            pending[dst] = recv
    for dst, tensors in pending.items():
        for t, new in zip(states[dst], tensors):
            t.copy_(new)


class ShardedEnsemble:
    """This rank's members of an ensemble, stepped by one BatchedCDKLM16,
    with the common time step agreed over all ranks."""

    def __init__(self, make_member, n_members, graph_steps=0, group=None):
        from . import BatchedEnsemble
        torch = _native.require_cuda()
        dist = _dist()
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.n_members = int(n_members)
        self.members = local_members(self.n_members, self.world, self.rank)
        self.sims = [make_member(m) for m in self.members]
        self.device = torch.device("cuda", torch.cuda.current_device())
        # collectives run on the device over NCCL; gloo (CPU tests, several
        # ranks on one GPU) takes host tensors
        gloo = dist.is_initialized() and dist.get_backend(group) == "gloo"
        self.comm_device = torch.device("cpu") if gloo else self.device
        self.batch = BatchedEnsemble.BatchedCDKLM16(self.sims, graph_steps=graph_steps) if self.sims else None

    def update_dt(self, courant=0.7):
        local = float(np.min(self.batch.max_dt())) if self.batch else float("inf")
        dt = np.float32(courant * global_min(local, self.comm_device, self.group))
        if self.batch:
            self.batch.set_dt([dt] * len(self.sims))
        return dt

    def states(self):
        """{global member: [eta, hu, hv]} of this rank's members (the
        ghost-inclusive device arrays of Q^n)."""
        return {m: [s.gpu_data.h0.tensor, s.gpu_data.hu0.tensor, s.gpu_data.hv0.tensor]
                for m, s in zip(self.members, self.sims)}

    def resample(self, pairs):
        """Resampling after an analysis (MPIOceanModelEnsemble.py:244-258,
        281-287): for each (src, dst) pair of global members, member dst
        takes member src's state.  Over gloo the states travel through host
        copies."""
        import torch
        for s in self.sims:
            s.gpu_stream.synchronize()
        if self.batch:
            self.batch.stream.synchronize()
        dev = self.states()
        if self.comm_device.type == "cpu":
            host = {m: [t.cpu() for t in ts] for m, ts in dev.items()}
            exchange_members(self.n_members, pairs, host, self.group)
            for m, ts in dev.items():
                for t, h in zip(ts, host[m]):
                    t.copy_(h)
        else:
            exchange_members(self.n_members, pairs, dev, self.group)
        torch.cuda.synchronize()

    def run_events(self, first_event, n_events, interval=60.0, std=0.05, corr_cells=15.0, courant=0.7):
        """BatchedCDKLM16.run_events with the member keys of the global
        ensemble and the time step agreed over all ranks."""
        steps = 0
        for e in range(int(first_event), int(first_event) + int(n_events)):
            if self.batch:
                n0 = self.sims[0].num_iterations
                self.batch.step(interval)
                steps += self.sims[0].num_iterations - n0
                self._model_error(e, std, corr_cells)
            self.update_dt(courant)
        return steps

    def _model_error(self, event, std, corr_cells):
        from . import ModelError
        for m, s in zip(self.members, self.sims):
            s.gpu_stream.wait_stream(self.batch.stream)
            ModelError.model_error(s, m, event, std, corr_cells)
        for s in self.sims:
            self.batch.stream.wait_stream(s.gpu_stream)

    def gather(self, local_values):
        return gather_member_scalars(self.n_members, local_values, self.comm_device, self.group)
