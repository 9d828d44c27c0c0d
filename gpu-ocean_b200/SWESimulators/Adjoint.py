"""Adjoint of the CDKLM16 time step.

No counterpart in the reference: gpu-ocean has no adjoint.  This module
returns gradients of an observation misfit

    J = sum over observation times and points of
        w_eta (eta - eta_obs)^2 + w_vel ((hu - hu_obs)^2 + (hv - hv_obs)^2)

with respect to the initial state (eta0, hu0, hv0) and a wind-stress field
(X, Y) per interior cell, constant in time.  The forward model is the
B200 CDKLM16 step (go_cdklm_step / go_traj_step, bit-identical to the
reference kernel); the reverse sweep runs the hand-written adjoint of each
RK stage (go_adjoint_step).  Memory is held by checkpointing: every
``checkpoint_every`` steps the state is kept, and each segment is
recomputed from its checkpoint before its reverse sweep (the last segment
is kept from the forward pass).  ``Revolve`` gives binomial schedules for
runs whose full trajectory does not fit.

``CDKLM16Misfit`` (J as a differentiable function of the initial state and
the wind) and ``CDKLM16Step`` (one RK2 step) wrap the problem in
``torch.autograd.Function`` objects.

Scope: north-up grids with wall and periodic boundaries; land and cells
shallower than the desingularisation depth are differentiated through the
branch the forward takes (land and dry cells are constants, desingularised
cells use u = hu / D(h)).
"""

import ctypes

import numpy as np

from . import _native


def _has_land(sim):
    """Whether any bathymetry corner of the simulator is land (the forward
    then runs its land-aware kernels, as CDKLM16 does)."""
    Bi = sim.downloadBathymetry()[0]
    return bool(np.any(np.abs(Bi.astype(np.float32) - np.float32(sim.bathymetry.mask_value)) < 1e-3))


def _round_up(n, m):
    return (n + m - 1) // m * m


class StateSlab:
    """n device states, each three (ny+4) x P float32 planes (eta, hu, hv)
    with P = nx+4 rounded up to 32 floats."""

    def __init__(self, n, nx, ny):
        torch = _native.require_cuda()
        self.n, self.nx, self.ny = int(n), int(nx), int(ny)
        self.P = _round_up(self.nx + 4, 32)
        self.t = torch.zeros((self.n, 3, self.ny + 4, self.P), dtype=torch.float32, device="cuda")
        self._gs = [self._make(i) for i in range(self.n)]

    def _make(self, i):
        s = _native.GoState()
        s.eta = int(self.t[i, 0].data_ptr())
        s.hu = int(self.t[i, 1].data_ptr())
        s.hv = int(self.t[i, 2].data_ptr())
        s.pitch = self.P * 4
        return s

    def gs(self, i):
        return ctypes.byref(self._gs[i])

    def interior(self, i):
        return self.t[i, :, 2:self.ny + 2, 2:self.nx + 2]

    def full(self, i):
        return self.t[i, :, :, :self.nx + 4]


def _copy_state(dst, i, src, k):
    dst.t[i].copy_(src.t[k])


class Observations:
    """Observed cells and values.  ij: (n, 2) interior (i, j) indices, the
    same cells at every observation time, or (len(steps), n, 2) cells per
    time (observations that move, such as drifters); steps: the step
    numbers (1..n_steps) after which J sums the misfit; values:
    (len(steps), n, 3) observed (eta, hu, hv)."""

    def __init__(self, ij, steps, values, w_eta=100.0, w_vel=1.0):
        torch = _native.require_cuda()
        ij = np.asarray(ij, dtype=np.int32)
        self.per_step = ij.ndim == 3
        ij = np.ascontiguousarray(ij.reshape(len(steps), -1, 2) if self.per_step else ij.reshape(-1, 2))
        self.n = ij.shape[-2]
        values = np.asarray(values, dtype=np.float32).reshape(len(steps), self.n, 3)
        self.steps = [int(s) for s in steps]
        if sorted(set(self.steps)) != self.steps:
            raise ValueError("observation steps must be increasing and distinct")
        self.ij_host = ij
        self.ij = torch.as_tensor(ij, device="cuda")
        self.values = torch.as_tensor(np.ascontiguousarray(values), device="cuda")
        self.index = {s: k for k, s in enumerate(self.steps)}
        self.w_eta = float(w_eta)
        self.w_vel = float(w_vel)

    def cells(self, k):
        """Device (n, 2) cells of observation time k."""
        return self.ij[k] if self.per_step else self.ij

    @classmethod
    def drifter_cells(cls, positions, nx, ny, dx, dy):
        """Interior cells under drifter positions (..., 2) in metres from the
        south-west interior corner: floor(x / dx), floor(y / dy) in float32,
        the cell the reference's observation kernel reads
        (observationKernels.cu:53-64, go_observe_flow), clamped to the
        interior (a drifter exactly on the east or north edge)."""
        p = np.asarray(positions, dtype=np.float32)
        i = np.floor(p[..., 0] / np.float32(dx)).astype(np.int64)
        j = np.floor(p[..., 1] / np.float32(dy)).astype(np.int64)
        return np.stack([np.clip(i, 0, nx - 1), np.clip(j, 0, ny - 1)], axis=-1).astype(np.int32)

    @classmethod
    def from_drifters(cls, positions, steps, currents, nx, ny, dx, dy, w_vel=1.0):
        """A misfit of drifter-observed currents: at each observation step
        s_k the (hu, hv) a drifter at positions[k] would observe
        (GPUDrifterCollection.observeUnderlyingFlow, observationKernels.cu:
        29-81) against currents[k], weight w_vel, eta unobserved.  The
        positions are given (the observed trajectories); the dependence of
        the positions on the flow is not differentiated."""
        pos = np.asarray(positions, dtype=np.float32).reshape(len(steps), -1, 2)
        cur = np.asarray(currents, dtype=np.float32).reshape(len(steps), -1, 2)
        values = np.zeros(cur.shape[:2] + (3,), dtype=np.float32)
        values[..., 1:] = cur
        return cls(cls.drifter_cells(pos, nx, ny, dx, dy), steps, values, w_eta=0.0, w_vel=w_vel)

    @staticmethod
    def sample(states_by_step, ij):
        """(len(steps), n, 3) values of host states {step: (eta, hu, hv)
        interior arrays} at the cells ij -- for building synthetic
        observations from a truth run."""
        ij = np.asarray(ij, dtype=np.int64).reshape(-1, 2)
        out = []
        for s in sorted(states_by_step):
            e, u, v = states_by_step[s]
            out.append(np.stack([e[ij[:, 1], ij[:, 0]], u[ij[:, 1], ij[:, 0]], v[ij[:, 1], ij[:, 0]]], axis=1))
        return np.asarray(out, dtype=np.float32)


class MisfitProblem:
    """J(eta0, hu0, hv0, X, Y) over n_steps RK2 steps of size dt on the grid,
    bathymetry, Coriolis, friction and boundaries of ``sim`` (a CDKLM16)."""

    def __init__(self, sim, n_steps, obs, dt=None, checkpoint_every=50):
        torch = _native.require_cuda()
        d = sim._domain.desc
        if abs(float(d.north_x)) > 0.0 or float(d.north_y) != 1.0:
            raise NotImplementedError("the adjoint is built for north-up grids only")
        if max(d.bc_north, d.bc_east, d.bc_south, d.bc_west) > 2:
            raise NotImplementedError("the adjoint is built for wall and periodic boundaries only")
        has_land = _has_land(sim)
        self.sim = sim
        self.nx, self.ny = int(sim.nx), int(sim.ny)
        self.n_steps = int(n_steps)
        self.dt = np.float32(sim.dt if dt is None else dt)
        self.obs = obs
        for s in obs.steps:
            if s < 0 or s > self.n_steps:
                raise ValueError("observation step %d outside 0..%d" % (s, self.n_steps))
        ij = obs.ij_host
        if ij.size and (ij[..., 0].min() < 0 or ij[..., 0].max() >= self.nx or ij[..., 1].min() < 0
                        or ij[..., 1].max() >= self.ny):
            raise ValueError("observation cells must be interior cells (0 <= i < nx, 0 <= j < ny)")
        self.k = max(1, min(int(checkpoint_every), self.n_steps))
        self.domain = _native.Domain(self.nx, self.ny, d.dx, d.dy, d.g, d.r, theta=d.theta,
                                     desing_eps=d.desing_eps, flux_slope_eps=d.flux_slope_eps,
                                     depth_cutoff=d.depth_cutoff,
                                     bc=(d.bc_north, d.bc_east, d.bc_south, d.bc_west),
                                     friction_law=d.friction_law, north=(d.north_x, d.north_y))
        self.domain.set_coriolis(sim.coriolis_rows)
        self.domain.set_land(has_land)
        self.Hi = sim.bathymetry.Bi.tensor
        self.Hi_pitch = int(sim.bathymetry.Bi.pitch)
        self.land = float(sim.bathymetry.mask_value)
        self.stream = torch.cuda.Stream()
        self.sh = _native.stream_handle(self.stream)
        self._rstream = torch.cuda.Stream()        # segment recompute, beside the reverse sweep
        self._rsh = _native.stream_handle(self._rstream)
        self._qn2 = self._qs2 = None               # second trajectory buffer (allocated on first use)
        Pw = _round_up(self.nx, 32)
        self.wind = torch.zeros((2, self.ny, Pw), dtype=torch.float32, device="cuda")
        self.lam_wind = torch.zeros((2, self.ny, Pw), dtype=torch.float32, device="cuda")
        self.wpitch = Pw * 4
        wx, wy = self.wind[0], self.wind[1]
        self.domain.set_wind_field(wx, wx, wy, wy)
        n_seg = (self.n_steps + self.k - 1) // self.k
        self.ckpt = StateSlab(max(n_seg, 1), self.nx, self.ny)
        self.qn = StateSlab(self.k + 1, self.nx, self.ny)
        self.qs = StateSlab(self.k, self.nx, self.ny)
        self.work = StateSlab(2, self.nx, self.ny)
        self.lam = StateSlab(3, self.nx, self.ny)      # lambda, scratch Q*, scratch Q^n
        self.J_dev = torch.zeros(1, dtype=torch.float64, device="cuda")
        self._ready = False
        self.recomputed_steps = 0

    # -- helpers -------------------------------------------------------------
    def _lib(self):
        return _native.load()

    def _segments(self):
        return [(a, min(a + self.k, self.n_steps)) for a in range(0, self.n_steps, self.k)]

    def _misfit(self, slab, i, step):
        if step not in self.obs.index:
            return
        o = self.obs
        k = o.index[step]
        _native.check(self._lib().go_obs_misfit(self.sh, slab.gs(i), self.nx, self.ny, o.n, _native.ptr(o.cells(k)),
                                                _native.ptr(o.values[k]), o.w_eta, o.w_vel,
                                                _native.ptr(self.J_dev)))

    def _obs_adjoint(self, slab, i, step):
        if step not in self.obs.index:
            return
        o = self.obs
        k = o.index[step]
        _native.check(self._lib().go_obs_adjoint(self.sh, slab.gs(i), self.lam.gs(0), self.nx, self.ny, o.n,
                                                 _native.ptr(o.cells(k)), _native.ptr(o.values[k]), o.w_eta, o.w_vel))

    def _traj_step(self, a_slab, ai, s_slab, si, b_slab, bi, sh=None):
        sh = self.sh if sh is None else sh
        _native.check(self._lib().go_traj_step(self.domain.handle, sh, float(self.dt), 0.0, a_slab.gs(ai),
                                               s_slab.gs(si), b_slab.gs(bi), _native.ptr(self.Hi),
                                               self.Hi_pitch, self.land))

    def _plain_steps(self, n):
        w = self.work
        g0, g1 = w._gs[0], w._gs[1]
        _native.check(self._lib().go_cdklm_step(
            self.domain.handle, self.sh, int(n), float(self.dt), 0.0,
            ctypes.c_void_p(g0.eta), ctypes.c_void_p(g0.hu), ctypes.c_void_p(g0.hv), g0.pitch,
            ctypes.c_void_p(g1.eta), ctypes.c_void_p(g1.hu), ctypes.c_void_p(g1.hv), g1.pitch,
            _native.ptr(self.Hi), self.Hi_pitch, self.land))

    def _load(self, eta0, hu0, hv0, wind_x, wind_y):
        torch = _native.require_cuda()
        w = self.work
        with torch.cuda.stream(self.stream):
            w.t[0].zero_()
            for f, a in enumerate((eta0, hu0, hv0)):
                w.interior(0)[f].copy_(torch.as_tensor(a, dtype=torch.float32, device="cuda").reshape(self.ny, self.nx))
            for f, a in enumerate((wind_x, wind_y)):
                self.wind[f, :, :self.nx].copy_(torch.as_tensor(a, dtype=torch.float32, device="cuda")
                                                .reshape(self.ny, self.nx))
        g = w._gs[0]
        _native.check(self._lib().go_boundary_condition(self.domain.handle, self.sh, ctypes.c_void_p(g.eta),
                                                        ctypes.c_void_p(g.hu), ctypes.c_void_p(g.hv), g.pitch))

    # -- forward ---------------------------------------------------------------
    def forward(self, eta0, hu0, hv0, wind_x, wind_y):
        """J for the given initial interior state and wind field (device
        tensors or host arrays of ny x nx).  Keeps the checkpoints and the
        last segment's trajectory for ``backward``."""
        torch = _native.require_cuda()
        self.stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(self.stream):
            self._load(eta0, hu0, hv0, wind_x, wind_y)
            self.J_dev.zero_()
            self._misfit(self.work, 0, 0)
            segs = self._segments()
            for s, (a, b) in enumerate(segs):
                _copy_state(self.ckpt, s, self.work, 0)
                if s == len(segs) - 1:
                    # the last segment's trajectory is kept for the reverse sweep
                    _copy_state(self.qn, 0, self.work, 0)
                    for t in range(b - a):
                        self._traj_step(self.qn, t, self.qs, t, self.qn, t + 1)
                        self._misfit(self.qn, t + 1, a + t + 1)
                    _copy_state(self.work, 0, self.qn, b - a)
                else:
                    n = a
                    for event in sorted({x for x in self.obs.steps if a < x <= b} | {b}):
                        self._plain_steps(event - n)
                        n = event
                        self._misfit(self.work, 0, n)
        self._ready = True
        self.stream.synchronize()
        return float(self.J_dev.item())

    def final_state(self):
        """Interior (eta, hu, hv) after the last forward run (device views)."""
        return self.work.interior(0)

    # -- reverse ---------------------------------------------------------------
    def backward(self):
        """Gradients (d eta0, d hu0, d hv0, d X, d Y) of J from the last
        ``forward``; device tensors of ny x nx."""
        if not self._ready:
            raise RuntimeError("backward() needs a forward() first")
        torch = _native.require_cuda()
        lib = self._lib()
        lam = self.lam
        lw = self.lam_wind
        self.stream.synchronize()
        self.domain.status(clear=True)
        segs = self._segments()
        last = len(segs) - 1
        # Segment s reads its trajectory from buffer (last - s) % 2; the last
        # segment's is buffer 0, kept by the forward pass.  The forward
        # recompute of segment s-1 runs on a second stream into the other
        # buffer while the adjoint sweeps segment s, so the recompute fills
        # the SMs the adjoint leaves idle; events order each buffer's reuse.
        if last > 0 and self._qn2 is None:
            self._qn2 = StateSlab(self.k + 1, self.nx, self.ny)
            self._qs2 = StateSlab(self.k, self.nx, self.ny)
        bufs = [(self.qn, self.qs), (self._qn2, self._qs2)]
        ready, freed = {}, {}

        def recompute(s):
            a, b = segs[s]
            i = (last - s) % 2
            qn, qs = bufs[i]
            if i in freed:
                self._rstream.wait_event(freed[i])
            with torch.cuda.stream(self._rstream):
                _copy_state(qn, 0, self.ckpt, s)
                for t in range(b - a):
                    self._traj_step(qn, t, qs, t, qn, t + 1, sh=self._rsh)
            ready[s] = torch.cuda.Event()
            ready[s].record(self._rstream)
            self.recomputed_steps += b - a

        with torch.cuda.stream(self.stream):
            lam.t.zero_()
            lw.zero_()
            if last > 0:
                recompute(last - 1)
            for s in range(last, -1, -1):
                a, b = segs[s]
                i = (last - s) % 2
                qn, qs = bufs[i]
                if s != last:
                    self.stream.wait_event(ready[s])
                    if s > 0:
                        recompute(s - 1)
                for n in range(b - 1, a - 1, -1):
                    t = n - a
                    self._obs_adjoint(qn, t + 1, n + 1)
                    _native.check(lib.go_adjoint_step(
                        self.domain.handle, self.sh, float(self.dt), qn.gs(t), qs.gs(t),
                        qn.gs(t + 1), lam.gs(0), lam.gs(0), lam.gs(1), lam.gs(2), _native.ptr(lw[0]),
                        _native.ptr(lw[1]), self.wpitch, _native.ptr(self.Hi), self.Hi_pitch))
                freed[i] = torch.cuda.Event()
                freed[i].record(self.stream)
            if 0 in self.obs.index:
                _copy_state(self.qn, 0, self.ckpt, 0)
                self._obs_adjoint(self.qn, 0, 0)
        self._rstream.synchronize()
        self.stream.synchronize()
        g = lam.interior(0).clone()
        return g[0], g[1], g[2], lw[0, :, :self.nx].clone(), lw[1, :, :self.nx].clone()

    def gradient(self, eta0, hu0, hv0, wind_x, wind_y):
        J = self.forward(eta0, hu0, hv0, wind_x, wind_y)
        return (J,) + tuple(self.backward())


class Revolve:
    """Binomial checkpointing: the schedule that reverses n_steps model steps
    with `snapshots` stored states (slot 0 holds step 0) and the fewest
    forward steps (Griewank 1992; Griewank & Walther 2000, "Algorithm 799:
    revolve").  The split points come from the recursion

        F(c, t) = min_m  m + F(c - 1, t - m) + F(c, m),   F(c, 1) = 0,
        F(0, t) = t (t - 1) / 2,

    F(c, t) = forward steps to reverse t steps from a stored start with c free
    slots; every reversed step also takes one forward step of its own (the
    stage states of the adjoint), which F does not count.

    `actions` lists ("advance", a, b), ("takeshot", slot, step),
    ("restore", slot, step) and ("reverse", n): at "reverse", the current
    state is Q^n; the step n -> n+1 is taken once more and reversed."""

    _tables = {}

    def __init__(self, n_steps, snapshots):
        n, s = int(n_steps), int(snapshots)
        if n < 1 or s < 1:
            raise ValueError("need n_steps >= 1 and snapshots >= 1")
        self.n = n
        self.s = min(s, n)
        self.F, self.split = self._table(n, self.s - 1)
        self.actions = self._schedule()

    @classmethod
    def _table(cls, t_max, c_max):
        key = (t_max, c_max)
        if key not in cls._tables:
            t = np.arange(t_max + 1, dtype=np.int64)
            F = np.zeros((c_max + 1, t_max + 1), dtype=np.int64)
            split = np.ones((c_max + 1, t_max + 1), dtype=np.int64)
            F[0] = t * (t - 1) // 2
            for c in range(1, c_max + 1):
                lim = min(c + 1, t_max)
                F[c, :lim + 1] = np.maximum(t[:lim + 1] - 1, 0)      # enough slots: one step at a time
                for tt in range(lim + 1, t_max + 1):
                    m = np.arange(1, tt)
                    cost = m + F[c - 1, tt - m] + F[c, 1:tt]
                    k = int(np.argmin(cost))
                    F[c, tt] = cost[k]
                    split[c, tt] = m[k]
            cls._tables[key] = (F, split)
        return cls._tables[key]

    def forward_steps(self):
        """Forward steps of the schedule: advances plus one per reversed step."""
        return int(self.F[self.s - 1, self.n]) + self.n

    def _schedule(self):
        acts = [("takeshot", 0, 0)]
        cur = 0
        stack = [(0, self.n, 0, tuple(range(1, self.s)))]
        while stack:
            a, b, slot_a, free = stack.pop()
            if b - a == 1 or not free:
                for n in range(b - 1, a - 1, -1):
                    if cur != a:
                        acts.append(("restore", slot_a, a))
                        cur = a
                    if n > a:
                        acts.append(("advance", a, n))
                    acts.append(("reverse", n))
                    cur = n + 1
                continue
            m = a + int(self.split[len(free), b - a])
            if cur != a:
                acts.append(("restore", slot_a, a))
                cur = a
            acts.append(("advance", a, m))
            acts.append(("takeshot", free[0], m))
            cur = m
            stack.append((a, m, slot_a, free))          # after the right part, with the slot freed
            stack.append((m, b, free[0], free[1:]))
        return acts


class MemberSlab:
    """M members' states in one (M, 3, ny+4, P) float32 tensor, so that a
    whole ensemble state is copied in one call."""

    def __init__(self, M, nx, ny, tensor=None):
        torch = _native.require_cuda()
        self.M, self.nx, self.ny = int(M), int(nx), int(ny)
        self.P = _round_up(self.nx + 4, 32)
        self.t = tensor if tensor is not None else torch.zeros((self.M, 3, self.ny + 4, self.P),
                                                               dtype=torch.float32, device="cuda")
        self._gs = []
        for m in range(self.M):
            g = _native.GoState()
            g.eta = int(self.t[m, 0].data_ptr())
            g.hu = int(self.t[m, 1].data_ptr())
            g.hv = int(self.t[m, 2].data_ptr())
            g.pitch = self.P * 4
            self._gs.append(g)

    def gs(self, m):
        return ctypes.byref(self._gs[m])

    def interior(self):
        return self.t[:, :, 2:self.ny + 2, 2:self.nx + 2]


class BatchedMisfitProblem:
    """The misfit problem for an ensemble: M members of one grid size, each
    with its own initial state and wind field and the same observations;
    J_m and its gradient for every member.  The forward steps all members in
    one launch per RK stage (go_batch_*), the reverse sweep runs the batched
    adjoint (go_adjoint_batch_step), and memory is held by binomial
    checkpointing (Revolve) over whole-ensemble snapshots."""

    def __init__(self, sims, n_steps, obs, dt=None, snapshots=None, memory_fraction=0.8):
        torch = _native.require_cuda()
        lib = _native.load()
        self.sims = list(sims)
        self.M = len(self.sims)
        s0 = self.sims[0]
        self.nx, self.ny = int(s0.nx), int(s0.ny)
        for s in self.sims:
            if (int(s.nx), int(s.ny)) != (self.nx, self.ny):
                raise ValueError("batched misfit members must share the grid size")
            d = s._domain.desc
            if abs(float(d.north_x)) > 0.0 or float(d.north_y) != 1.0:
                raise NotImplementedError("the adjoint is built for north-up grids only")
            if max(d.bc_north, d.bc_east, d.bc_south, d.bc_west) > 2:
                raise NotImplementedError("the adjoint is built for wall and periodic boundaries only")
        self.n_steps = int(n_steps)
        self.dt = np.float32(s0.dt if dt is None else dt)
        self.obs = obs
        ij = obs.ij_host
        if ij.size and (ij[..., 0].min() < 0 or ij[..., 0].max() >= self.nx or ij[..., 1].min() < 0
                        or ij[..., 1].max() >= self.ny):
            raise ValueError("observation cells must be interior cells")
        self.stream = torch.cuda.Stream()
        self.sh = _native.stream_handle(self.stream)
        M, nx, ny = self.M, self.nx, self.ny
        Pw = _round_up(nx, 32)
        self.wind = torch.zeros((M, 2, ny, Pw), dtype=torch.float32, device="cuda")
        self.lam_wind = torch.zeros((M, 2, ny, Pw), dtype=torch.float32, device="cuda")
        self.wpitch = Pw * 4
        self.h0 = MemberSlab(M, nx, ny)          # current state Q^n (stage 1 in place)
        self.h1 = MemberSlab(M, nx, ny)          # Q*
        self.qn = MemberSlab(M, nx, ny)          # Q^n kept for the adjoint
        self.lam = MemberSlab(M, nx, ny)
        self.scr_star = MemberSlab(M, nx, ny)
        self.scr_qn = MemberSlab(M, nx, ny)
        self.J_dev = torch.zeros(M, dtype=torch.float64, device="cuda")
        self.domains = []
        for m, s in enumerate(self.sims):
            d = s._domain.desc
            dom = _native.Domain(nx, ny, d.dx, d.dy, d.g, d.r, theta=d.theta, desing_eps=d.desing_eps,
                                 flux_slope_eps=d.flux_slope_eps, depth_cutoff=d.depth_cutoff,
                                 bc=(d.bc_north, d.bc_east, d.bc_south, d.bc_west), friction_law=d.friction_law,
                                 north=(d.north_x, d.north_y))
            dom.set_coriolis(s.coriolis_rows)
            dom.set_land(_has_land(s))
            dom.set_wind_field(self.wind[m, 0], self.wind[m, 0], self.wind[m, 1], self.wind[m, 1])
            self.domains.append(dom)
        self.batch = _native.Batch(self.domains)
        for m, s in enumerate(self.sims):
            self.batch.set_member(m, self.dt, tuple(self.h0.t[m, f] for f in range(3)),
                                  tuple(self.h1.t[m, f] for f in range(3)), s.bathymetry.Bi.tensor,
                                  float(s.bathymetry.mask_value), 0.0)
        h = ctypes.c_void_p()
        arr = (ctypes.c_void_p * M)(*[dom.handle.value for dom in self.domains])
        _native.check(lib.go_adjoint_batch_create(arr, M, ctypes.byref(h)))
        self.adj = h
        for m, s in enumerate(self.sims):
            _native.check(lib.go_adjoint_batch_set_member(
                self.adj, m, float(self.dt), self.qn.gs(m), self.h1.gs(m), self.h0.gs(m), self.lam.gs(m),
                self.scr_star.gs(m), self.scr_qn.gs(m), _native.ptr(self.lam_wind[m, 0]),
                _native.ptr(self.lam_wind[m, 1]), self.wpitch, _native.ptr(s.bathymetry.Bi.tensor),
                int(s.bathymetry.Bi.pitch)))
        snap_bytes = self.h0.t.numel() * 4
        if snapshots is None:
            free = torch.cuda.mem_get_info()[0]
            snapshots = max(1, int(free * float(memory_fraction) // snap_bytes))
        self.revolve = Revolve(self.n_steps, min(int(snapshots), self.n_steps))
        self.snap = torch.empty((self.revolve.s,) + tuple(self.h0.t.shape), dtype=torch.float32, device="cuda")
        self.snapshot_bytes = snap_bytes

    def close(self):
        if getattr(self, "adj", None) is not None and self.adj.value:
            _native.load().go_adjoint_batch_destroy(self.adj)
            self.adj = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _misfit(self, step):
        if step not in self.obs.index:
            return
        o, lib = self.obs, _native.load()
        k = o.index[step]
        for m in range(self.M):
            _native.check(lib.go_obs_misfit(self.sh, self.h0.gs(m), self.nx, self.ny, o.n, _native.ptr(o.cells(k)),
                                            _native.ptr(o.values[k]), o.w_eta, o.w_vel,
                                            _native.ptr(self.J_dev[m:m + 1])))

    def _obs_adjoint(self, step):
        if step not in self.obs.index:
            return
        o, lib = self.obs, _native.load()
        k = o.index[step]
        for m in range(self.M):
            _native.check(lib.go_obs_adjoint(self.sh, self.h0.gs(m), self.lam.gs(m), self.nx, self.ny, o.n,
                                             _native.ptr(o.cells(k)), _native.ptr(o.values[k]), o.w_eta, o.w_vel))

    def _advance(self, a, b):
        """h0: Q^a -> Q^b; the misfit of states reached for the first time."""
        cur = a
        if b > self._reached:
            events = sorted({x for x in self.obs.steps if max(a, self._reached) < x <= b})
            for e in events:
                if e > cur:
                    self.batch.step(e - cur, self.stream)
                    cur = e
                self._misfit(e)
            self._reached = b
        if b > cur:
            self.batch.step(b - cur, self.stream)

    def gradient(self, x0, wind):
        """x0: (M, 3, ny, nx) initial interior states; wind: (M, 2, ny, nx)
        wind stress.  Returns (J per member (numpy), dJ/dx0 (M, 3, ny, nx),
        dJ/dwind (M, 2, ny, nx))."""
        torch = _native.require_cuda()
        lib = _native.load()
        self.stream.wait_stream(torch.cuda.current_stream())
        nx, ny = self.nx, self.ny
        with torch.cuda.stream(self.stream):
            self.h0.t.zero_()
            self.h0.interior().copy_(torch.as_tensor(x0, dtype=torch.float32, device="cuda"))
            self.wind[:, :, :, :nx].copy_(torch.as_tensor(wind, dtype=torch.float32, device="cuda"))
            for m, dom in enumerate(self.domains):
                g = self.h0._gs[m]
                _native.check(lib.go_boundary_condition(dom.handle, self.sh, ctypes.c_void_p(g.eta),
                                                        ctypes.c_void_p(g.hu), ctypes.c_void_p(g.hv), g.pitch))
            self.lam.t.zero_()
            self.lam_wind.zero_()
            self.J_dev.zero_()
            self._reached = 0
            self._misfit(0)
            for act in self.revolve.actions:
                kind = act[0]
                if kind == "takeshot":
                    self.snap[act[1]].copy_(self.h0.t)
                elif kind == "restore":
                    self.h0.t.copy_(self.snap[act[1]])
                elif kind == "advance":
                    self._advance(act[1], act[2])
                else:
                    n = act[1]
                    self.qn.t.copy_(self.h0.t)
                    self._advance(n, n + 1)
                    self._obs_adjoint(n + 1)
                    _native.check(lib.go_adjoint_batch_step(self.adj, self.sh))
            if 0 in self.obs.index:
                self.h0.t.copy_(self.snap[0])
                self._obs_adjoint(0)
        self.stream.synchronize()
        return (self.J_dev.cpu().numpy(), self.lam.interior().clone(),
                self.lam_wind[:, :, :, :nx].clone())


def _autograd():
    torch = _native.require_cuda()

    class CDKLM16Misfit(torch.autograd.Function):
        """J = problem.forward(eta0, hu0, hv0, X, Y) as a torch scalar
        (float64) with the adjoint as its backward."""

        @staticmethod
        def forward(ctx, problem, eta0, hu0, hv0, wind_x, wind_y):
            J = problem.forward(eta0.detach(), hu0.detach(), hv0.detach(), wind_x.detach(), wind_y.detach())
            ctx.problem = problem
            return torch.tensor(J, dtype=torch.float64, device=eta0.device)

        @staticmethod
        def backward(ctx, gJ):
            ge, gu, gv, gx, gy = ctx.problem.backward()
            s = gJ.to(torch.float32)
            return None, ge * s, gu * s, gv * s, gx * s, gy * s

    class CDKLM16Step(torch.autograd.Function):
        """One RK2 step (eta, hu, hv, X, Y) -> (eta', hu', hv') of the
        problem's domain; backward through go_adjoint_step."""

        @staticmethod
        def forward(ctx, problem, eta, hu, hv, wind_x, wind_y):
            p = problem
            slab = StateSlab(3, p.nx, p.ny)            # Q^n, Q*, Q^{n+1}
            p.stream.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(p.stream):
                for f, a in enumerate((eta, hu, hv)):
                    slab.interior(0)[f].copy_(a.detach())
                p.wind[0, :, :p.nx].copy_(wind_x.detach())
                p.wind[1, :, :p.nx].copy_(wind_y.detach())
            g = slab._gs[0]
            lib = _native.load()
            _native.check(lib.go_boundary_condition(p.domain.handle, p.sh, ctypes.c_void_p(g.eta),
                                                    ctypes.c_void_p(g.hu), ctypes.c_void_p(g.hv), g.pitch))
            p._traj_step(slab, 0, slab, 1, slab, 2)
            torch.cuda.current_stream().wait_stream(p.stream)
            ctx.problem = p
            ctx.slab = slab
            out = slab.interior(2).clone()
            return out[0], out[1], out[2]

        @staticmethod
        def backward(ctx, le, lu, lv):
            p, slab = ctx.problem, ctx.slab
            lam = StateSlab(3, p.nx, p.ny)
            lw = torch.zeros_like(p.lam_wind)
            p.stream.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(p.stream):
                for f, a in enumerate((le, lu, lv)):
                    if a is not None:
                        lam.interior(0)[f].copy_(a)
            _native.check(_native.load().go_adjoint_step(
                p.domain.handle, p.sh, float(p.dt), slab.gs(0), slab.gs(1), slab.gs(2), lam.gs(0), lam.gs(0),
                lam.gs(1), lam.gs(2), _native.ptr(lw[0]), _native.ptr(lw[1]), p.wpitch, _native.ptr(p.Hi),
                p.Hi_pitch))
            torch.cuda.current_stream().wait_stream(p.stream)
            g = lam.interior(0).clone()
            return None, g[0], g[1], g[2], lw[0, :, :p.nx].clone(), lw[1, :, :p.nx].clone()

    return CDKLM16Misfit, CDKLM16Step


_FUNCS = None


def functions():
    """(CDKLM16Misfit, CDKLM16Step) torch.autograd.Function classes."""
    global _FUNCS
    if _FUNCS is None:
        _FUNCS = _autograd()
    return _FUNCS
