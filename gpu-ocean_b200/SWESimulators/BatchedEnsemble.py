"""Batched stepping of many CDKLM16 simulators.

The reference's ensembles advance their members one at a time
(gpu_ocean/SWESimulators/OceanNoiseEnsemble.py:506-531,
OceanModelEnsemble.py:105-117, EnsembleFromFiles.py:302-324): every member
issues its own 2 step launches (plus boundary launches) per time step from
Python.  ``BatchedCDKLM16`` keeps the members as ordinary ``CDKLM16``
objects (their ``gpu_data`` buffers, ``t`` and ``num_iterations`` stay valid
for the DA code) and advances all of them with one launch per RK stage over
a packed tile list (``go_batch_step``), optionally replayed from a captured
CUDA graph.  Members may have different grid sizes, bathymetry and time
steps; they must share the kernel variant (friction law, grid angle, uniform
or per-cell wind).
"""

import numpy as np

from . import _native


class BatchedCDKLM16:

    def __init__(self, sims, graph_steps=0, launch=None):
        """sims: list of CDKLM16.  graph_steps > 0 captures that many steps
        into a CUDA graph used by ``advance``.  launch: optional (shape,
        rows_per_block, blocks) as chosen by Autotune.tune_batch."""
        torch = _native.require_cuda()
        self.sims = list(sims)
        self.n = len(self.sims)
        self.stream = torch.cuda.Stream()
        self.batch = _native.Batch([s._domain for s in self.sims])
        if launch is not None:
            self.batch.set_launch(*launch)
        for m, s in enumerate(self.sims):
            self._bind(m, s)
        self.graph_steps = 0
        if graph_steps:
            self.capture(graph_steps)

    # -- failure isolation ------------------------------------------------
    def member_status(self, clear=False):
        """Each member's status word (GO_STATUS_* bits, member order); a
        member whose state went non-finite is flagged alone."""
        self.stream.synchronize()
        return self.batch.status(clear)

    def failed_members(self):
        """Indices of the members whose state went non-finite."""
        return [m for m, w in enumerate(self.member_status()) if w & _native.GO_STATUS_NONFINITE]

    def drop(self, members):
        """Removes members (indices into the current member list) from the
        ensemble, as the reference's ensembles stop stepping dead particles
        (BaseOceanStateEnsemble.py:108-110, EnsembleFromFiles.py:315); the
        batch is rebuilt over the remaining members, which step on bit for
        bit as before.  Returns the removed simulators."""
        gone = sorted(set(int(m) for m in members))
        if any(m < 0 or m >= self.n for m in gone):
            raise IndexError("member index out of range")
        self.stream.synchronize()
        removed = [self.sims[m] for m in gone]
        self.sims = [s for m, s in enumerate(self.sims) if m not in gone]
        self.n = len(self.sims)
        self.invalidate_model_error()
        launch = getattr(self.batch, "launch", None)
        self.batch.close()
        self.batch = _native.Batch([s._domain for s in self.sims])
        if launch is not None:
            self.batch.set_launch(*launch)
        for m, s in enumerate(self.sims):
            self._bind(m, s)
        steps = self.graph_steps
        self.graph_steps = 0
        if steps:
            self.capture(steps)
        return removed

    def _bind(self, m, s):
        # the member's wind at its current time (Simulator.update_wind_stress)
        wind_t = np.float32(s.update_wind_stress())
        g = s.gpu_data
        self.batch.set_member(m, np.float32(s.dt), (g.h0.tensor, g.hu0.tensor, g.hv0.tensor),
                              (g.h1.tensor, g.hu1.tensor, g.hv1.tensor), s.bathymetry.Bi.tensor,
                              float(s.bathymetry.mask_value), float(wind_t))

    def _time_varying_wind(self):
        return any(len(s.wind_stress.t) > 1 for s in self.sims)

    def _sync_members(self):
        # work queued on the members' own streams (uploads, perturbations)
        # completes before the batched launch reads their buffers; inside
        # run_events the members are touched only through the batch stream,
        # so the loop orders them once at its start and end
        if getattr(self, "_owned", False):
            return
        for s in self.sims:
            self.stream.wait_stream(s.gpu_stream)

    def _release_members(self):
        # later work on a member's own stream waits for the batch's
        if getattr(self, "_owned", False):
            return
        for s in self.sims:
            s.gpu_stream.wait_stream(self.stream)

    def _first_step_bc(self):
        # on the batch stream, after _sync_members
        for s in self.sims:
            if s.t == 0:
                s.bc_kernel.boundaryCondition(self.stream, s.gpu_data.h0, s.gpu_data.hu0, s.gpu_data.hv0)

    def set_dt(self, dts):
        """Per-member time steps (sequence of n floats)."""
        dts = np.asarray(dts, dtype=np.float32).reshape(-1)
        for s, d in zip(self.sims, dts):
            s.dt = d
        self.batch.set_dt(dts, self.stream)

    def capture(self, n_steps):
        self._sync_members()
        self.batch.capture(int(n_steps), self.stream)
        self.graph_steps = int(n_steps)

    def advance(self, n_steps):
        """n_steps RK2 steps of every member at its own dt (graph replays
        for whole multiples of the captured length, plain launches for the
        rest)."""
        self._sync_members()
        self._first_step_bc()
        if self._time_varying_wind():
            # wind interpolated in time: rebind every member before each step
            for _ in range(int(n_steps)):
                for m, s in enumerate(self.sims):
                    self._bind(m, s)
                self._sync_members()
                self.batch.step(1, self.stream)
                self._account(1)
            return [s.t for s in self.sims]
        done = 0
        if self.graph_steps:
            while n_steps - done >= self.graph_steps:
                done += self.batch.replay(self.stream)
        if n_steps - done:
            self.batch.step(n_steps - done, self.stream)
        self._account(n_steps)
        return [s.t for s in self.sims]

    def _account(self, n_steps):
        self._release_members()
        # t accumulates float64(dt) once per step, as CDKLM16.step does
        # (members sharing t and dt share the sum)
        sums = {}
        for s in self.sims:
            key = (float(s.t), float(np.float32(s.dt)))
            if key not in sums:
                steps = np.full(int(n_steps), np.float64(np.float32(s.dt)))
                sums[key] = float(np.cumsum(np.concatenate([[np.float64(s.t)], steps]))[-1])
            s.t = sums[key]
            s.num_iterations += n_steps

    def step(self, t_end, apply_stochastic_term=True):
        """Every member advances by t_end with the reference's step() loop
        semantics (CDKLM16.py:494-598); the members must share dt.  Members
        built with small_scale_perturbation get their model error after
        every step (CDKLM16.py:580-586), all members in one batched pass."""
        dts = {float(np.float32(s.dt)) for s in self.sims}
        if len(dts) != 1:
            raise ValueError("step(t_end) needs a common dt; use advance(n) for per-member dt")
        perturb = apply_stochastic_term and self._has_model_error()
        dt = np.float32(self.sims[0].dt)
        t_now = 0.0
        full = 0
        while t_now < t_end:
            local_dt = np.float32(min(dt, np.float32(t_end - t_now)))
            if local_dt != dt:
                break
            full += 1
            t_now += np.float64(local_dt)
        if full and perturb:
            for _ in range(full):
                self.advance(1)
                self.perturb_members(boundary_conditions=True)
        elif full:
            self.advance(full)
        if t_now < t_end:
            last = np.float32(min(dt, np.float32(t_end - t_now)))
            self.set_dt([last] * self.n)
            self.advance(1)
            if perturb:
                self.perturb_members(boundary_conditions=True)
            self.set_dt([dt] * self.n)
        return self.sims[0].t

    # -- the members' own model error (OceanStateNoise) ----------------------
    def _has_model_error(self):
        flags = [bool(getattr(s, "small_scale_perturbation", False)) for s in self.sims]
        if any(flags) and not all(flags):
            raise ValueError("either every member or none has small_scale_perturbation")
        return all(flags)

    def _noise_batch(self):
        """go_noise_batch over the members' OceanStateNoise objects.  The
        descriptors point at the members' own buffers and hold each member's
        f, beta, g and q0, so the set is rebuilt when a member's
        OceanStateNoise object is replaced; after changing a member's
        physical parameters or buffers in place, call
        invalidate_model_error()."""
        errs = [s.small_scale_model_error for s in self.sims]
        key = tuple(map(id, errs))
        if getattr(self, "_noise", None) is not None:
            if key == self._noise_key:
                return self._noise
            self.invalidate_model_error()
        import ctypes
        e0, s0 = errs[0], self.sims[0]
        for e, s in zip(errs, self.sims):
            same = (int(e.nx), int(e.ny), int(e.interpolation_factor), bool(e.use_lcg), int(e.periodicNorthSouth),
                    int(e.periodicEastWest), float(e.soar_L), float(e.dx), float(e.dy)) == \
                   (int(e0.nx), int(e0.ny), 1, bool(e0.use_lcg), int(e0.periodicNorthSouth),
                    int(e0.periodicEastWest), float(e0.soar_L), float(e0.dx), float(e0.dy))
            if not same or int(s.ghost_cells_x) != int(s0.ghost_cells_x) or \
                    int(s.ghost_cells_y) != int(s0.ghost_cells_y):
                raise ValueError("batched model error needs one grid, ghost cells, generator, boundary kinds, "
                                 "soar_L and interpolation factor 1 for all members")
        descs = (_native.GoNoiseMember * self.n)(*[e.member_desc(s) for e, s in zip(errs, self.sims)])
        h = ctypes.c_void_p()
        _native.check(_native.load().go_noise_batch_create(
            ctypes.cast(descs, ctypes.c_void_p), self.n, int(e0.nx), int(e0.ny), float(e0.dx), float(e0.dy),
            int(s0.ghost_cells_x), int(s0.ghost_cells_y), float(e0.soar_L), int(e0.periodicNorthSouth),
            int(e0.periodicEastWest), int(bool(e0.use_lcg)), ctypes.byref(h)))
        self._noise = h
        self._noise_key = key
        return h

    def invalidate_model_error(self):
        """Drops the batched model-error descriptors; the next perturbation
        rebuilds them from the members' current OceanStateNoise state."""
        h = getattr(self, "_noise", None)
        self._noise = None
        if h is not None:
            self.stream.synchronize()   # no perturbation in flight reads the descriptors
            _native.load().go_noise_batch_destroy(h)

    def perturb_members(self, q0_scale=1.0, perturbation_scale=1.0, boundary_conditions=False):
        """Every member's OceanStateNoise.perturbSim (OceanStateNoise.py:
        376-397) in three launches for all members (go_noise_batch_perturb),
        each member bit for bit as alone: CDKLM16.perturbState of every
        member (CDKLM16.py:642-644).  boundary_conditions=True also refreshes
        the ghost cells afterwards, as the step loop does (CDKLM16.py:
        580-586)."""
        h = self._noise_batch()
        self._sync_members()
        _native.check(_native.load().go_noise_batch_perturb(h, _native.stream_handle(self.stream), float(q0_scale),
                                                            float(np.float32(perturbation_scale)), 1))
        if boundary_conditions:
            for s in self.sims:
                s.bc_kernel.boundaryCondition(self.stream, s.gpu_data.h0, s.gpu_data.hu0, s.gpu_data.hv0)
        self._release_members()

    def __del__(self):
        h = getattr(self, "_noise", None)
        if h is not None:
            try:
                _native.load().go_noise_batch_destroy(h)
            except Exception:
                pass
            self._noise = None

    def perturb(self, key0, event, std=0.05, corr_cells=15.0):
        """Every member's eta += std * field(key (key0, m), event): one
        batched pass, identical to ModelError.perturb member by member."""
        from . import ModelError
        lib = _native.load()
        n = lib.go_batch_grf_scratch_floats(self.batch.handle, float(corr_cells))
        if n == 0:
            raise ValueError("invalid correlation length")
        self._sync_members()
        buf = ModelError._scratch_for(n, self.stream)
        _native.check(lib.go_batch_grf_perturb(self.batch.handle, _native.stream_handle(self.stream),
                                               int(key0) & 0xFFFFFFFF, int(event) & 0xFFFFFFFF, float(std),
                                               float(corr_cells), _native.ptr(buf), int(buf.numel())))
        ModelError._scratch_used(self.stream)
        self._release_members()

    def model_error(self, event, std=0.05, corr_cells=15.0):
        from . import ModelError
        self.perturb(ModelError.MODEL_ERROR_SEED, event, std, corr_cells)

    def max_dt(self):
        """Exact CFL limit of every member (one batched reduction launch on
        the batch stream, one device-to-host read); numpy array of n.  Each
        value equals the member's own go_max_dt."""
        torch = _native.require_cuda()
        if getattr(self, "_dt_all", None) is None or self._dt_all.numel() != self.n:
            self._dt_all = torch.empty(self.n, dtype=torch.float32, device="cuda")
        self._sync_members()
        _native.check(_native.load().go_batch_max_dt(self.batch.handle, _native.stream_handle(self.stream),
                                                     _native.ptr(self._dt_all)))
        self.stream.synchronize()
        return self._dt_all.cpu().numpy()

    def update_dt(self, courant=0.7):
        """Common dt = courant * min over members of the exact CFL limit."""
        dt = np.float32(courant * float(np.min(self.max_dt())))
        self.set_dt([dt] * self.n)
        return dt

    def run_events(self, first_event, n_events, interval=60.0, std=0.05, corr_cells=15.0, courant=0.7,
                   device_loop=True):
        """The ensemble workload loop: for each event e, every member advances
        `interval` seconds at the common dt (step(t_end) semantics), then
        gets model error for event e, then the common dt is recomputed from
        the members' CFL limits -- what the reference's ensembles do member
        by member (OceanNoiseEnsemble.py:506-531).  Returns the steps taken.

        device_loop: the whole loop runs on the device in one graph launch
        (go_batch_run_events), the host waiting once at the end; the members
        must share dt (update_dt), carry no OceanStateNoise model error of
        their own and no time-varying wind.  Otherwise, or with
        device_loop=False, the host drives each event (one CFL read-back per
        event); both give the same states, times and steps bit for bit."""
        dts = {float(np.float32(s.dt)) for s in self.sims}
        if device_loop and len(dts) == 1 and not self._time_varying_wind() and not self._has_model_error():
            return self._run_events_device(first_event, n_events, interval, std, corr_cells, courant)
        steps = 0
        self._sync_members()
        self._owned = True
        try:
            for e in range(int(first_event), int(first_event) + int(n_events)):
                n0 = self.sims[0].num_iterations
                self.step(interval)
                steps += self.sims[0].num_iterations - n0
                self.model_error(e, std, corr_cells)
                self.update_dt(courant)
        finally:
            self._owned = False
            self._release_members()
        return steps

    def _run_events_device(self, first_event, n_events, interval, std, corr_cells, courant):
        from . import ModelError
        if int(n_events) <= 0:
            return 0
        lib = _native.load()
        n = lib.go_batch_grf_scratch_floats(self.batch.handle, float(corr_cells))
        if n == 0:
            raise ValueError("invalid correlation length")
        self._sync_members()
        self._first_step_bc()
        # the captured graph holds the scratch address: keep one buffer
        buf = getattr(self, "_loop_scratch", None)
        if buf is None or buf.numel() < n:
            torch = _native.require_cuda()
            buf = torch.empty(int(n), dtype=torch.float32, device="cuda")
            self._loop_scratch = buf
        t0 = [float(s.t) for s in self.sims]
        t, steps, dt = self.batch.run_events(self.stream, first_event, n_events, float(interval),
                                             np.float32(self.sims[0].dt), float(courant),
                                             ModelError.MODEL_ERROR_SEED, float(std), float(corr_cells), buf, t0)
        for s, tm in zip(self.sims, t):
            s.t = float(tm)
            s.num_iterations += steps
            s.dt = dt
        self._release_members()
        return steps

    def synchronize(self):
        self.stream.synchronize()
