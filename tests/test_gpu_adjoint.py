"""Adjoint of the CDKLM16 step on a GPU (go_adjoint_stage, go_adjoint_step,
SWESimulators.Adjoint).

1. Each RK stage's adjoint against torch autograd through the FP64 torch
   transcription of the stage (oracle/cdklm16_oracle.py rk_stage), on the
   same FP32 inputs, for wall/periodic boundaries and all friction laws.
2. One RK2 step and the gradient of an observation misfit over many steps
   (every-k checkpointing) against torch autograd through the FP64
   transcription, taken stage by stage along the trajectory the FP32 model
   computes.  (Full FP64 autograd recomputes that trajectory in FP64; the
   two trajectories differ by FP32 rounding, ~1e-4 in hu after one stage,
   which flips near-tie minmod choices at a few percent of the cells, so the
   two gradients differ there by design.  That difference is printed.)
3. FP64 central finite differences of the misfit along random directions
   (eps = 1e-4 ... 1e-9 times |x|); a direction is used at the largest eps
   for which no branch of the scheme (minmod choice, wave speeds, zero-flux
   cut, positivity adjustment, dry clamp) differs between x - h d and
   x + h d.
4. Independence of the checkpoint interval, and the torch.autograd.Function
   wrappers.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

import torch.nn.functional as Fnn  # noqa: E402

from SWESimulators import Adjoint, CDKLM16, Common, SyntheticCases as SC, _native  # noqa: E402
from oracle import cdklm16_oracle as O  # noqa: E402


@pytest.fixture(scope="module")
def ctx():
    return Common.CUDAContext()


def make_sim(ctx, nx, ny, bc=(1, 2, 1, 2), r=3.0e-3, dx=2000.0, spin=4, seed=61000, linear=False,
             seed_bumps=None):
    c = SC.grf(nx, ny=ny, dx=dx, bc=bc, r=r, seed_bathy=seed,
               seed_bumps=seed + 1 if seed_bumps is None else seed_bumps, steps=1)
    sim = CDKLM16.CDKLM16(ctx, dt=c.dt, linear_friction=linear, **c.kwargs())
    for _ in range(spin):
        sim.step(c.dt)
    torch.cuda.synchronize()
    return c, sim


def make_coastal_sim(ctx, nx, ny, bc=(1, 2, 1, 2), r=3.0e-3, linear=False, spin=4, seed=64000):
    """A grid with an island (corners at the land value 1e20) inside a shelf
    3-9 cm deep (cells shallower than desing_eps = 0.1 m) and a patch of dry
    corners (depth 0) at the shelf's edge, so that every branch of the cell
    state map (land, dry, desingularised, wet) occurs.  The shelf depths are
    random: on a flat shelf at rest the two sides of every face are equal and
    the wave-speed maxima of the flux tie, where the FP32 kernel and the FP64
    transcription may take different subgradients."""
    c = SC.grf(nx, ny=ny, dx=2000.0, bc=bc, r=r, seed_bathy=seed, seed_bumps=seed + 1, steps=1)
    Hi = c.Hi.copy()
    j0, i0 = 2 + ny // 2, 2 + nx // 2
    rng = np.random.default_rng(seed + 2)
    Hi[j0 - 7:j0 + 7, i0 - 6:i0 + 8] = 0.03 + 0.06 * rng.random((14, 14))   # shelf
    Hi[j0 - 3:j0 + 3, i0 - 2:i0 + 4] = 1.0e20        # island
    Hi[j0 + 5:j0 + 8, i0 - 9:i0 - 4] = 0.0           # dry patch at the shelf edge
    c.Hi = O.fix_bi_ghost_corners(Hi, c.nx, c.ny, c.bc)
    eta0 = c.eta0.copy()
    eta0[j0 - 10:j0 + 11, i0 - 12:i0 + 12] = 0.0     # still water over the shelf
    c.eta0 = eta0
    sim = CDKLM16.CDKLM16(ctx, dt=c.dt, linear_friction=linear, **c.kwargs())
    for _ in range(spin):
        sim.step(c.dt)
    torch.cuda.synchronize()
    return c, sim


def cell_classes(sim):
    """Counts of land, dry, desingularised and wet interior cells of the
    simulator's current state."""
    eta = sim.download()[0][2:-2, 2:-2].astype(np.float64)
    Bm = sim.downloadBathymetry()[1][2:-2, 2:-2].astype(np.float64)
    land = np.abs(Bm - 1.0e20) <= 1e-3 * 1e20
    h = eta + Bm
    dry = ~land & (h <= 1.0e-5)
    des = ~land & ~dry & (h < 0.1)
    return int(land.sum()), int(dry.sum()), int(des.sum()), int((~land & ~dry & ~des).sum())


def wind_field(c, seed):
    rng = np.random.default_rng(seed)
    X = c.wind[0] * (1.0 + 0.3 * rng.standard_normal((c.ny, c.nx)))
    Y = c.wind[1] * (1.0 + 0.3 * rng.standard_normal((c.ny, c.nx)))
    return (torch.as_tensor(X.astype(np.float32), device="cuda"),
            torch.as_tensor(Y.astype(np.float32), device="cuda"))


class Model:
    """FP64 torch transcription of a CDKLM16 simulator's domain."""

    def __init__(self, sim, c, linear=False):
        self.nx, self.ny = c.nx, c.ny
        self.p = O.Params(c.nx, c.ny, c.dx, c.dy, c.g, c.r, bc=c.bc, linear_friction=linear)
        Bi, Bm = sim.downloadBathymetry()
        like = torch.zeros(1, dtype=torch.float64, device="cuda")
        self.S = O.Static(self.p, Bi, Bm, sim.coriolis_rows, dtype=np.float64, like=like)
        self.xp = self.S.xp

    def full(self, a):
        return O.periodic_wrap(self.xp, Fnn.pad(a, (2, 2, 2, 2)), self.p.bc, self.nx, self.ny)

    def stage(self, q_in, q_n, dt, k, X, Y):
        return O.rk_stage(self.p, [self.full(a) for a in q_in], list(q_n), self.S, float(dt), k, wind=(X, Y))

    def step(self, q, dt, X, Y):
        qs = self.stage(q, q, dt, 0, X, Y)
        return self.stage(qs, q, dt, 1, X, Y)


def vjp_stage(model, q_in, q_n, k, lam, X, Y, dt):
    """FP64 vector-Jacobian product of one stage at the given (FP32) inputs:
    (d q_in, d q_n, d X, d Y) for the output adjoint lam."""
    x = [a.double().clone().requires_grad_(True) for a in q_in]
    qn = [a.double().clone().requires_grad_(True) for a in q_n] if k == 1 else x
    Xd, Yd = X.double().requires_grad_(True), Y.double().requires_grad_(True)
    out = model.stage(x, qn, dt, k, Xd, Yd)
    sum((o * l).sum() for o, l in zip(out, lam)).backward()
    gqn = [a.grad for a in qn] if k == 1 else [torch.zeros_like(a) for a in x]
    return [a.grad for a in x], gqn, Xd.grad, Yd.grad


def vjp_step(model, q_n, q_star, lam, X, Y, dt):
    """FP64 adjoint of one RK2 step along the stored (q_n, q_star)."""
    ls, lqn, gx1, gy1 = vjp_stage(model, q_star, q_n, 1, lam, X, Y, dt)
    l0, _, gx0, gy0 = vjp_stage(model, q_n, q_n, 0, ls, X, Y, dt)
    return [a + b for a, b in zip(l0, lqn)], gx0 + gx1, gy0 + gy1


def rel(a, b):
    a = a.double()
    b = b.double()
    s = b.abs().max().item()
    return (a - b).abs().max().item() / (s if s > 0 else 1.0)


def empty_obs():
    return Adjoint.Observations(np.zeros((0, 2)), [], np.zeros((0, 0, 3)))


def load_state(slab, i, sim):
    g = sim.gpu_data
    for f, a in enumerate((g.h0, g.hu0, g.hv0)):
        slab.full(i)[f].copy_(a.view)


def gs_none():
    return ctypes.cast(None, ctypes.POINTER(_native.GoState))


CASES = {
    # (bc north, east, south, west), r, linear friction
    "walls_ns_periodic_ew_quadratic": ((1, 2, 1, 2), 3.0e-3, False),
    "walls_linear": ((1, 1, 1, 1), 3.0e-3, True),
    "periodic_frictionless": ((2, 2, 2, 2), 0.0, False),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("shape", [(40, 36), (80, 52)])
def test_stage_adjoints_match_fp64_autograd(ctx, name, shape):
    bc, r, linear = CASES[name]
    nx, ny = shape
    c, sim = make_sim(ctx, nx, ny, bc=bc, r=r, linear=linear)
    prob = Adjoint.MisfitProblem(sim, 1, empty_obs())
    model = Model(sim, c, linear)
    lib = _native.load()
    X, Y = wind_field(c, 7)
    prob.wind[0, :, :nx].copy_(X)
    prob.wind[1, :, :nx].copy_(Y)
    slab = Adjoint.StateSlab(3, nx, ny)
    load_state(slab, 0, sim)
    torch.cuda.synchronize()
    dt = np.float32(c.dt)
    prob._traj_step(slab, 0, slab, 1, slab, 2)
    prob.stream.synchronize()

    Xd, Yd = X.double().requires_grad_(True), Y.double().requires_grad_(True)
    # the transcription reproduces the stored forward stages
    q0 = [slab.interior(0)[f].double() for f in range(3)]
    out0 = model.stage(q0, q0, dt, 0, Xd, Yd)
    for f in range(3):      # FP32 vs FP64 of one stage (momentum-flux cancellation ~5e-5)
        assert rel(slab.interior(1)[f], out0[f].detach()) < 5e-4

    gen = torch.Generator(device="cuda").manual_seed(11)
    lam = Adjoint.StateSlab(4, nx, ny)          # lam_out, lam_in, lam_qn, spare
    lam.interior(0).copy_(torch.randn((3, ny, nx), device="cuda", generator=gen))
    lw = torch.zeros_like(prob.lam_wind)
    for k in (0, 1):
        lw.zero_()
        q_in, q_out = (0, 1) if k == 0 else (1, 2)
        torch.cuda.synchronize()             # torch writes above, adjoint on the problem's stream below
        rc = lib.go_adjoint_stage(prob.domain.handle, prob.sh, k, float(dt), slab.gs(q_in), slab.gs(q_out),
                                  lam.gs(0), lam.gs(1), lam.gs(2) if k == 1 else gs_none(),
                                  _native.ptr(lw[0]), _native.ptr(lw[1]), prob.wpitch, _native.ptr(prob.Hi),
                                  prob.Hi_pitch)
        assert rc == 0, lib.go_last_error()
        prob.stream.synchronize()
        x = [slab.interior(q_in)[f].double().clone().requires_grad_(True) for f in range(3)]
        qn = [slab.interior(0)[f].double().clone().requires_grad_(True) for f in range(3)]
        Xk, Yk = X.double().requires_grad_(True), Y.double().requires_grad_(True)
        out = model.stage(x, qn if k == 1 else x, dt, k, Xk, Yk)
        L = sum((o * lam.interior(0)[f].double()).sum() for f, o in enumerate(out))
        L.backward()
        errs = [rel(lam.interior(1)[f], x[f].grad) for f in range(3)]
        errs += [rel(lw[0, :, :nx], Xk.grad), rel(lw[1, :, :nx], Yk.grad)]
        if k == 1:
            errs += [rel(lam.interior(2)[f], qn[f].grad) for f in range(3)]
        print(name, shape, "stage", k, ["%.2e" % e for e in errs])
        assert max(errs) < 1e-4, errs


@pytest.mark.parametrize("name", ["walls_ns_periodic_ew_quadratic", "walls_linear"])
def test_stage_adjoints_with_land_and_shallow_cells_match_fp64_autograd(ctx, name):
    """64 x 64 with an island, a shelf shallower than desing_eps and dry
    cells: both stage adjoints (tile form) against FP64 autograd of the
    transcription, which takes the same branches of the cell state map."""
    bc, r, linear = CASES[name]
    nx = ny = 64
    c, sim = make_coastal_sim(ctx, nx, ny, bc=bc, r=r, linear=linear)
    n_land, n_dry, n_des, n_wet = cell_classes(sim)
    print(name, "land / dry / desingularised / wet cells:", n_land, n_dry, n_des, n_wet)
    assert n_land > 0 and n_dry > 0 and n_des > 0
    prob = Adjoint.MisfitProblem(sim, 1, empty_obs())
    model = Model(sim, c, linear)
    lib = _native.load()
    X, Y = wind_field(c, 8)
    prob.wind[0, :, :nx].copy_(X)
    prob.wind[1, :, :nx].copy_(Y)
    slab = Adjoint.StateSlab(3, nx, ny)
    load_state(slab, 0, sim)
    torch.cuda.synchronize()
    dt = np.float32(c.dt)
    prob._traj_step(slab, 0, slab, 1, slab, 2)
    prob.stream.synchronize()
    gen = torch.Generator(device="cuda").manual_seed(12)
    lam = Adjoint.StateSlab(4, nx, ny)
    lam.interior(0).copy_(torch.randn((3, ny, nx), device="cuda", generator=gen))
    lw = torch.zeros_like(prob.lam_wind)
    for k in (0, 1):
        lw.zero_()
        q_in, q_out = (0, 1) if k == 0 else (1, 2)
        torch.cuda.synchronize()
        rc = lib.go_adjoint_stage(prob.domain.handle, prob.sh, k, float(dt), slab.gs(q_in), slab.gs(q_out),
                                  lam.gs(0), lam.gs(1), lam.gs(2) if k == 1 else gs_none(),
                                  _native.ptr(lw[0]), _native.ptr(lw[1]), prob.wpitch, _native.ptr(prob.Hi),
                                  prob.Hi_pitch)
        assert rc == 0, lib.go_last_error()
        prob.stream.synchronize()
        x = [slab.interior(q_in)[f].double().clone().requires_grad_(True) for f in range(3)]
        qn = [slab.interior(0)[f].double().clone().requires_grad_(True) for f in range(3)]
        Xk, Yk = X.double().requires_grad_(True), Y.double().requires_grad_(True)
        out = model.stage(x, qn if k == 1 else x, dt, k, Xk, Yk)
        L = sum((o * lam.interior(0)[f].double()).sum() for f, o in enumerate(out))
        L.backward()
        errs = [rel(lam.interior(1)[f], x[f].grad) for f in range(3)]
        errs += [rel(lw[0, :, :nx], Xk.grad), rel(lw[1, :, :nx], Yk.grad)]
        if k == 1:
            errs += [rel(lam.interior(2)[f], qn[f].grad) for f in range(3)]
        print(name, "coastal stage", k, ["%.2e" % e for e in errs])
        assert max(errs) < 1e-4, errs


def test_step_adjoint_matches_fp64_autograd(ctx):
    c, sim = make_sim(ctx, 72, 60, spin=6, seed=62000)
    prob = Adjoint.MisfitProblem(sim, 1, empty_obs())
    model = Model(sim, c)
    X, Y = wind_field(c, 8)
    prob.wind[0, :, :c.nx].copy_(X)
    prob.wind[1, :, :c.nx].copy_(Y)
    slab = Adjoint.StateSlab(3, c.nx, c.ny)
    load_state(slab, 0, sim)
    torch.cuda.synchronize()
    dt = np.float32(c.dt)
    prob._traj_step(slab, 0, slab, 1, slab, 2)
    lam = Adjoint.StateSlab(3, c.nx, c.ny)
    gen = torch.Generator(device="cuda").manual_seed(12)
    lam_out = torch.randn((3, c.ny, c.nx), device="cuda", generator=gen)
    prob.stream.synchronize()
    lam.interior(0).copy_(lam_out)
    lw = torch.zeros_like(prob.lam_wind)
    lib = _native.load()
    torch.cuda.synchronize()
    rc = lib.go_adjoint_step(prob.domain.handle, prob.sh, float(dt), slab.gs(0), slab.gs(1), slab.gs(2), lam.gs(0),
                             lam.gs(0), lam.gs(1), lam.gs(2), _native.ptr(lw[0]), _native.ptr(lw[1]), prob.wpitch,
                             _native.ptr(prob.Hi), prob.Hi_pitch)
    assert rc == 0, lib.go_last_error()
    prob.stream.synchronize()
    lam64 = [lam_out[f].double() for f in range(3)]
    g, gx, gy = vjp_step(model, list(slab.interior(0)), list(slab.interior(1)), lam64, X, Y, dt)
    errs = [rel(lam.interior(0)[f], g[f]) for f in range(3)] + [rel(lw[0, :, :c.nx], gx),
                                                                rel(lw[1, :, :c.nx], gy)]
    print("step (along the FP32 trajectory)", ["%.2e" % e for e in errs])
    assert max(errs) < 1e-4, errs
    # full FP64 autograd (FP64 trajectory): differs where near-tie branches flip
    x = [slab.interior(0)[f].double().clone().requires_grad_(True) for f in range(3)]
    out = model.step(x, dt, X.double(), Y.double())
    sum((o * lam64[f]).sum() for f, o in enumerate(out)).backward()
    l2 = [float((lam.interior(0)[f].double() - x[f].grad).norm() / x[f].grad.norm()) for f in range(3)]
    print("step vs full FP64 autograd, relative L2:", ["%.2e" % e for e in l2])


def misfit_setup(ctx, n, dx, n_steps, obs_every, n_obs, k, seed_bg=50002, seed_truth=50001, seed_obs=50003,
                 spin=0):
    """The adjoint workload: background and truth runs differ in their
    initial bumps; observations of the truth at n_obs seeded interior cells
    every obs_every steps.  spin > 0 starts both from their states after
    that many steps (a flow not at rest)."""
    c, sim = make_sim(ctx, n, n, dx=dx, spin=spin, seed=20241, seed_bumps=seed_bg)
    ct, truth = make_sim(ctx, n, n, dx=dx, spin=spin, seed=20241, seed_bumps=seed_truth)
    rng = np.random.default_rng(seed_obs)
    flat = rng.choice((n - 4) * (n - 4), size=n_obs, replace=False)
    ij = np.stack([2 + flat % (n - 4), 2 + flat // (n - 4)], axis=1)
    steps = list(range(obs_every, n_steps + 1, obs_every))
    states = {}
    for s in range(1, n_steps + 1):
        truth.step(ct.dt)
        if s in steps:
            states[s] = truth.download(interior_domain_only=True)
    obs = Adjoint.Observations(ij, steps, Adjoint.Observations.sample(states, ij))
    prob = Adjoint.MisfitProblem(sim, n_steps, obs, dt=c.dt, checkpoint_every=k)
    x0 = [torch.as_tensor(np.ascontiguousarray(a), device="cuda") for a in sim.download(interior_domain_only=True)]
    X, Y = wind_field(c, 9)
    return c, sim, prob, obs, x0, X, Y, ij, steps


def oracle_J(model, obs_vals, ij, steps, x, X, Y, dt, n_steps, w_eta=100.0, w_vel=1.0):
    jj = torch.as_tensor(ij[:, 1], device="cuda")
    ii = torch.as_tensor(ij[:, 0], device="cuda")
    q = list(x)
    J = torch.zeros((), dtype=torch.float64, device="cuda")
    for n in range(1, n_steps + 1):
        q = list(model.step(q, dt, X, Y))
        if n in steps:
            o = obs_vals[steps.index(n)]
            J = J + w_eta * ((q[0][jj, ii] - o[:, 0]) ** 2).sum() + \
                w_vel * (((q[1][jj, ii] - o[:, 1]) ** 2).sum() + ((q[2][jj, ii] - o[:, 2]) ** 2).sum())
    return J


def fp32_trajectory(prob, x0, n_steps):
    """The model's own trajectory (go_traj_step from the initial state),
    as the lists of interior Q^n (n = 0..n_steps) and Q* (n = 0..n_steps-1)."""
    lib = _native.load()
    slab = Adjoint.StateSlab(2 * n_steps + 1, prob.nx, prob.ny)
    for f in range(3):
        slab.interior(0)[f].copy_(x0[f])
    torch.cuda.synchronize()
    g0 = slab._gs[0]
    assert lib.go_boundary_condition(prob.domain.handle, prob.sh, ctypes.c_void_p(g0.eta), ctypes.c_void_p(g0.hu),
                                     ctypes.c_void_p(g0.hv), g0.pitch) == 0
    for n in range(n_steps):
        prob._traj_step(slab, 2 * n, slab, 2 * n + 1, slab, 2 * n + 2)
    prob.stream.synchronize()
    qn = [list(slab.interior(2 * n)) for n in range(n_steps + 1)]
    qs = [list(slab.interior(2 * n + 1)) for n in range(n_steps)]
    return qn, qs, slab


def fp64_tape_adjoint(model, prob, obs, ij, steps, qn, qs, X, Y, dt):
    """FP64 torch-autograd adjoint of the misfit, stage by stage along the
    stored FP32 trajectory (the reverse sweep the GPU adjoint performs)."""
    n_steps = len(qs)
    jj = torch.as_tensor(ij[:, 1], device="cuda")
    ii = torch.as_tensor(ij[:, 0], device="cuda")
    lam = [torch.zeros((prob.ny, prob.nx), dtype=torch.float64, device="cuda") for _ in range(3)]
    gx = torch.zeros_like(lam[0])
    gy = torch.zeros_like(lam[0])
    w = (obs.w_eta, obs.w_vel, obs.w_vel)
    vals = obs.values.double()
    for n in range(n_steps - 1, -1, -1):
        if n + 1 in steps:
            o = vals[steps.index(n + 1)]
            for f in range(3):
                lam[f] = lam[f].index_put((jj, ii), 2.0 * w[f] * (qn[n + 1][f].double()[jj, ii] - o[:, f]),
                                          accumulate=True)
        lam, dx, dy = vjp_step(model, qn[n], qs[n], lam, X, Y, dt)
        gx, gy = gx + dx, gy + dy
    return lam, gx, gy


def test_misfit_gradient_with_checkpoints_matches_fp64_autograd(ctx):
    n_steps = 24
    c, sim, prob, obs, x0, X, Y, ij, steps = misfit_setup(ctx, 48, 4000.0, n_steps, 6, 16, 7)
    J, ge, gu, gv, gx, gy = prob.gradient(*x0, X, Y)
    assert prob.recomputed_steps == 21          # segments 0-7, 7-14, 14-21 recomputed; 21-24 kept
    model = Model(sim, c)
    dt = np.float32(c.dt)
    qn, qs, _ = fp32_trajectory(prob, x0, n_steps)
    lam, rx, ry = fp64_tape_adjoint(model, prob, obs, ij, steps, qn, qs, X, Y, dt)
    errs = [rel(ge, lam[0]), rel(gu, lam[1]), rel(gv, lam[2]), rel(gx, rx), rel(gy, ry)]
    # J of the FP64 transcription (FP64 trajectory) and its full autograd
    x = [a.double().clone().requires_grad_(True) for a in x0]
    Xd, Yd = X.double().requires_grad_(True), Y.double().requires_grad_(True)
    Jr = oracle_J(model, obs.values.double(), ij, steps, x, Xd, Yd, dt, n_steps)
    Jr.backward()
    l2 = [float((a.double() - b.grad).norm() / b.grad.norm()) for a, b in zip((ge, gu, gv, gx, gy), x + [Xd, Yd])]
    print("misfit J %.6e (FP64 %.6e); along the FP32 trajectory" % (J, Jr.item()), ["%.2e" % e for e in errs],
          "; vs full FP64 autograd, relative L2", ["%.2e" % e for e in l2])
    assert abs(J - Jr.item()) / abs(Jr.item()) < 1e-4
    assert max(errs) < 1e-4, errs


def test_gradient_independent_of_checkpoint_interval(ctx):
    grads = []
    for k in (1, 5, 30):
        c, sim, prob, obs, x0, X, Y, ij, steps = misfit_setup(ctx, 40, 4000.0, 30, 10, 12, k)
        J, *g = prob.gradient(*x0, X, Y)
        grads.append(g)
    for g in grads[1:]:
        for a, b in zip(g, grads[0]):
            assert torch.equal(a, b)


def test_finite_differences_fp64_away_from_kinks(ctx):
    """FP64 central differences of the misfit of the FP64 transcription
    along 20 random directions.  In a smooth flow the left and right face
    states nearly tie, so the wave-speed and minmod choices flip somewhere
    for perturbations down to ~1e-8 |x| (measured: ~2e4 flips at 1e-4 |x|,
    ~30 at 1e-7, none at 1e-9 over 8 steps of 64 x 64): each direction takes
    the largest eps in {1e-4 ... 1e-9} |x| for which no branch differs
    between x - h d and x + h d.  The error is |fd - <g, d>| / |g|."""
    n, n_steps = 64, 8
    c, sim, prob, obs, x0, X, Y, ij, steps = misfit_setup(ctx, n, 8000.0, n_steps, 4, 64, 4, spin=5)
    J, *g = prob.gradient(*x0, X, Y)
    model = Model(sim, c)
    vals = obs.values.double()
    dt = np.float32(c.dt)
    xs = [a.double() for a in x0] + [X.double(), Y.double()]
    g64 = [a.double() for a in g]
    gnorm = float(torch.sqrt(sum((a ** 2).sum() for a in g64)))
    # full FP64 autograd of the transcription (FP64 trajectory) as a second reference
    xg = [a.clone().requires_grad_(True) for a in xs]
    oracle_J(model, vals, ij, steps, xg[:3], xg[3], xg[4], dt, n_steps).backward()
    gref = [a.grad for a in xg]
    xnorm = float(torch.sqrt(sum((a ** 2).sum() for a in xs)))
    scales = [0.1, 1.0, 1.0, float(abs(c.wind[0])), float(abs(c.wind[1]))]
    gen = torch.Generator(device="cuda").manual_seed(13)
    errs, errs64, used = [], [], []
    for _ in range(20):
        d = [s * torch.randn(a.shape, dtype=torch.float64, device="cuda", generator=gen) for s, a in zip(scales, xs)]
        dn = float(torch.sqrt(sum((a ** 2).sum() for a in d)))
        d = [a / dn for a in d]
        gd = float(sum((a * b).sum() for a, b in zip(g64, d)))
        gd64 = float(sum((a * b).sum() for a, b in zip(gref, d)))
        for eps in (1e-4, 1e-5, 1e-6, 1e-7, 1e-8, 1e-9):
            h = eps * xnorm
            xp_ = [a + h * b for a, b in zip(xs, d)]
            xm_ = [a - h * b for a, b in zip(xs, d)]
            with torch.no_grad():
                with O.record_branches() as rp:
                    Jp = oracle_J(model, vals, ij, steps, xp_[:3], xp_[3], xp_[4], dt, n_steps).item()
                with O.record_branches() as rm:
                    Jm = oracle_J(model, vals, ij, steps, xm_[:3], xm_[3], xm_[4], dt, n_steps).item()
            if len(rp.masks) == len(rm.masks) and all(torch.equal(a, b) for a, b in zip(rp.masks, rm.masks)):
                fd = (Jp - Jm) / (2.0 * h)
                errs.append(abs(fd - gd) / gnorm)
                errs64.append(abs(fd - gd64) / gnorm)
                used.append(eps)
                break
    print("FD: %d of 20 directions kink-free; eps used %s" % (len(errs), sorted(set(used))))
    print("  |fd - <g_gpu, d>| / |g|: max %.2e median %.2e" % (max(errs), float(np.median(errs))))
    print("  |fd - <g_fp64, d>| / |g|: max %.2e" % max(errs64))
    assert len(errs) >= 15
    assert max(errs64) < 1e-4
    assert max(errs) < 1e-3


def test_autograd_functions(ctx):
    c, sim, prob, obs, x0, X, Y, ij, steps = misfit_setup(ctx, 40, 4000.0, 12, 4, 10, 5)
    Misfit, Step = Adjoint.functions()
    J0, *g0 = prob.gradient(*x0, X, Y)
    leaves = [a.clone().requires_grad_(True) for a in x0] + [X.clone().requires_grad_(True),
                                                             Y.clone().requires_grad_(True)]
    J = Misfit.apply(prob, *leaves)
    (3.0 * J).backward()
    for leaf, ref in zip(leaves, g0):
        assert torch.allclose(leaf.grad, 3.0 * ref, rtol=1e-6, atol=0.0)
    # one step through CDKLM16Step against the FP64 transcription
    model = Model(sim, c)
    leaves = [a.clone().requires_grad_(True) for a in x0] + [X.clone().requires_grad_(True),
                                                             Y.clone().requires_grad_(True)]
    out = Step.apply(prob, *leaves)
    w = [torch.randn_like(o) for o in out]
    sum((o * wi).sum() for o, wi in zip(out, w)).backward()
    with torch.no_grad():
        ref = model.step([a.double() for a in x0], np.float32(c.dt), X.double(), Y.double())
    for o, r in zip(out, ref):
        assert rel(o.detach(), r) < 5e-4
    qn, qs, _ = fp32_trajectory(prob, x0, 1)
    for o, q in zip(out, qn[1]):
        assert torch.equal(o.detach(), q)
    g, gx, gy = vjp_step(model, qn[0], qs[0], [wi.double() for wi in w], X, Y, np.float32(c.dt))
    errs = [rel(leaves[f].grad, g[f]) for f in range(3)] + [rel(leaves[3].grad, gx), rel(leaves[4].grad, gy)]
    assert max(errs) < 1e-4, errs


@pytest.mark.parametrize("nx, ny, bc, coastal", [(100, 70, (1, 2, 1, 2), False), (140, 90, (2, 2, 2, 2), False),
                                                  (70, 130, (1, 1, 1, 1), False), (100, 70, (1, 2, 1, 2), True),
                                                  (70, 90, (1, 1, 1, 1), True)])
def test_adjoint_launch_forms_agree(ctx, nx, ny, bc, coastal):
    """The tile form (tiles of 16, 8 and 12 rows) and the marching forms
    (64/128 columns, several strip heights) give the same stage adjoints to
    FP32 rounding, also with land, dry and desingularised cells."""
    if coastal:
        c, sim = make_coastal_sim(ctx, nx, ny, bc=bc, seed=63500)
    else:
        c, sim = make_sim(ctx, nx, ny, bc=bc, seed=63000)
    prob = Adjoint.MisfitProblem(sim, 1, empty_obs())
    X, Y = wind_field(c, 10)
    prob.wind[0, :, :nx].copy_(X)
    prob.wind[1, :, :nx].copy_(Y)
    slab = Adjoint.StateSlab(3, nx, ny)
    load_state(slab, 0, sim)
    torch.cuda.synchronize()
    dt = float(np.float32(c.dt))
    prob._traj_step(slab, 0, slab, 1, slab, 2)
    prob.stream.synchronize()
    lib = _native.load()
    lam_out = torch.randn((3, ny, nx), device="cuda", generator=torch.Generator(device="cuda").manual_seed(14))
    results = {}
    forms = [(_native.GO_ADJ_TILE, 0), (_native.GO_ADJ_TILE, 8), (_native.GO_ADJ_TILE, 12),
             (_native.GO_ADJ_MARCH64, 0), (_native.GO_ADJ_MARCH64, 8),
             (_native.GO_ADJ_MARCH128, 0), (_native.GO_ADJ_MARCH128, 16), (_native.GO_ADJ_MARCH128, 5)]
    for kind, rows in forms:
        assert lib.go_domain_set_adjoint_launch(prob.domain.handle, kind, rows) == 0
        lam = Adjoint.StateSlab(4, nx, ny)
        lam.interior(0).copy_(lam_out)
        lw = torch.zeros_like(prob.lam_wind)
        torch.cuda.synchronize()
        out = []
        for k in (1, 0):
            q_in, q_out, l_out, l_in = (1, 2, 0, 1) if k == 1 else (0, 1, 1, 3)
            assert lib.go_adjoint_stage(prob.domain.handle, prob.sh, k, dt, slab.gs(q_in), slab.gs(q_out),
                                        lam.gs(l_out), lam.gs(l_in), lam.gs(2), _native.ptr(lw[0]),
                                        _native.ptr(lw[1]), prob.wpitch, _native.ptr(prob.Hi), prob.Hi_pitch) == 0
        prob.stream.synchronize()
        results[(kind, rows)] = [lam.interior(1).clone(), lam.interior(2).clone(), lam.interior(3).clone(),
                                 lw[:, :, :nx].clone()]
    ref = results[forms[0]]
    for key, res in results.items():
        errs = [rel(a, b) for a, b in zip(res, ref)]
        print((nx, ny, bc, coastal), key, ["%.1e" % e for e in errs])
        assert max(errs) < 2e-5, (key, errs)


def _ensemble_setup(ctx, M, n, n_steps, obs_every, n_obs):
    c, sim0, prob0, obs, x0, X, Y, ij, steps = misfit_setup(ctx, n, 4000.0, n_steps, obs_every, n_obs, n_steps,
                                                            spin=2)
    sims = [sim0] + [make_sim(ctx, n, n, dx=4000.0, spin=2, seed=20241, seed_bumps=50010 + m)[1]
                     for m in range(1, M)]
    xs = torch.stack([torch.stack([torch.as_tensor(np.ascontiguousarray(a), device="cuda")
                                   for a in s.download(interior_domain_only=True)]) for s in sims])
    gen = torch.Generator(device="cuda").manual_seed(21)
    winds = torch.stack([torch.stack([X, Y])] * M) * (1.0 + 0.2 * torch.rand((M, 2, n, n), device="cuda",
                                                                               generator=gen))
    return c, sims, obs, xs, winds, steps


def test_batched_adjoint_equals_member_by_member(ctx):
    M, n, n_steps = 3, 48, 12
    c, sims, obs, xs, winds, steps = _ensemble_setup(ctx, M, n, n_steps, 4, 10)
    bp = Adjoint.BatchedMisfitProblem(sims, n_steps, obs, dt=c.dt, snapshots=3)
    assert bp.revolve.s == 3
    J, g, gw = bp.gradient(xs, winds)
    lib = _native.load()
    for m in range(M):
        p = Adjoint.MisfitProblem(sims[m], n_steps, obs, dt=c.dt, checkpoint_every=5)
        assert lib.go_domain_set_adjoint_launch(p.domain.handle, _native.GO_ADJ_MARCH128, 0) == 0
        Jm, ge, gu, gv, gx, gy = p.gradient(xs[m, 0], xs[m, 1], xs[m, 2], winds[m, 0], winds[m, 1])
        assert abs(J[m] - Jm) <= 1e-9 * abs(Jm)
        for a, b in zip((g[m, 0], g[m, 1], g[m, 2], gw[m, 0], gw[m, 1]), (ge, gu, gv, gx, gy)):
            assert torch.equal(a, b)


def test_batched_adjoint_independent_of_snapshots(ctx):
    M, n, n_steps = 2, 40, 16
    c, sims, obs, xs, winds, steps = _ensemble_setup(ctx, M, n, n_steps, 4, 8)
    res = []
    for s in (1, 2, 5, 16):
        bp = Adjoint.BatchedMisfitProblem(sims, n_steps, obs, dt=c.dt, snapshots=s)
        res.append(bp.gradient(xs, winds))
        bp.close()
    for J, g, gw in res[1:]:
        assert np.allclose(J, res[0][0], rtol=1e-12)
        assert torch.equal(g, res[0][1]) and torch.equal(gw, res[0][2])


def test_drifter_misfit(ctx):
    """Drifter-observed currents as the misfit (Observations.from_drifters):
    a truth run with drifters attached gives their positions and the
    currents go_observe_flow reads under them; those are the truth's hu, hv
    at Observations.drifter_cells; and the misfit over moving cells has the
    J and gradient of the sum of one fixed-cell problem per observation
    time (the adjoint is linear in the observation forcing)."""
    from SWESimulators.GPUDrifterCollection import GPUDrifterCollection

    n, dx, n_steps, steps = 40, 4000.0, 12, [4, 8, 12]
    c, sim = make_sim(ctx, n, n, dx=dx, seed=20241, seed_bumps=50002)
    ct, truth = make_sim(ctx, n, n, dx=dx, seed=20241, seed_bumps=50001)
    d = GPUDrifterCollection(ctx, 30, boundaryConditions=truth.boundary_conditions, domain_size_x=n * dx,
                             domain_size_y=n * dx)
    rng = np.random.default_rng(7)
    d.setDrifterPositions(rng.uniform(0.1, 0.9, (30, 2)) * n * dx)
    truth.attachDrifters(d)
    pos, cur = [], []
    for s in range(1, n_steps + 1):
        truth.step(ct.dt)
        if s in steps:
            p = d.getDrifterPositions()
            g = truth.gpu_data
            o = d.observeUnderlyingFlow(g.hu0, g.hv0, n, n, dx, dx)
            _, u, v = truth.download(interior_domain_only=True)
            cells = Adjoint.Observations.drifter_cells(p, n, n, dx, dx)
            assert np.array_equal(o[:, 0], u[cells[:, 1], cells[:, 0]])
            assert np.array_equal(o[:, 1], v[cells[:, 1], cells[:, 0]])
            pos.append(p)
            cur.append(o)
    assert not np.array_equal(pos[0], pos[-1])
    obs = Adjoint.Observations.from_drifters(pos, steps, cur, n, n, dx, dx)
    assert obs.per_step and obs.w_eta == 0.0
    x0 = [torch.as_tensor(np.ascontiguousarray(a), device="cuda") for a in sim.download(interior_domain_only=True)]
    X, Y = wind_field(c, 9)
    J, *g = Adjoint.MisfitProblem(sim, n_steps, obs, dt=c.dt, checkpoint_every=5).gradient(*x0, X, Y)
    J_sum, g_sum = 0.0, None
    vals = obs.values.cpu().numpy()
    for k, s in enumerate(steps):
        ok = Adjoint.Observations(obs.ij_host[k], [s], vals[k:k + 1], w_eta=0.0, w_vel=1.0)
        Jk, *gk = Adjoint.MisfitProblem(sim, n_steps, ok, dt=c.dt, checkpoint_every=5).gradient(*x0, X, Y)
        J_sum += float(Jk)
        g_sum = gk if g_sum is None else [a + b for a, b in zip(g_sum, gk)]
    print("drifter misfit J %.6e, sum of fixed-cell misfits %.6e" % (float(J), J_sum))
    assert float(J) > 0 and abs(float(J) - J_sum) <= 1e-12 * abs(J_sum)
    errs = [rel(a, b) for a, b in zip(g, g_sum)]
    print("gradient rel. differences", ["%.2e" % e for e in errs])
    assert max(errs) < 1e-5, errs
