"""Batched stepping (go_batch_*, BatchedCDKLM16) and the autotuner on a GPU.

The batched launch must give bit-identical states to stepping each member
alone (the reference's member-by-member loop, OceanNoiseEnsemble.py:506-531),
for members of different sizes, bathymetry and time steps, with and without
CUDA-graph replay.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from SWESimulators import Autotune, BatchedEnsemble, CDKLM16, Common, SyntheticCases as SC  # noqa: E402


@pytest.fixture(scope="module")
def ctx():
    return Common.CUDAContext()


def _members(ctx, sizes, seed0=40000):
    sims = []
    for k, n in enumerate(sizes):
        c = SC.grf(n, dx=1000.0, seed_bathy=seed0 + k, seed_bumps=seed0 + 500 + k, steps=1)
        sims.append(CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs()))
    return sims


def _states(sims):
    return [np.stack(s.download()) for s in sims]


def test_mixed_batch_equals_member_by_member(ctx):
    sizes = [128, 256, 96, 200, 160]
    alone = _members(ctx, sizes)
    for s in alone:
        for _ in range(12):
            s.step(s.dt)
    expect = _states(alone)
    sims = _members(ctx, sizes)
    b = BatchedEnsemble.BatchedCDKLM16(sims)
    b.advance(12)
    got = _states(sims)
    for e, g in zip(expect, got):
        assert np.array_equal(e, g)
    for s, a in zip(sims, alone):
        assert s.num_iterations == a.num_iterations
        assert s.t == a.t


@pytest.mark.parametrize("launch", [(5, 16, 0), (5, 3, 148 * 5), (4, 16, 148 * 5), (6, 24, 0), (7, 5, 148 * 3),
                                    (8, 24, 0), (8, 6, 148 * 2)])
def test_batch_launch_shapes_equal_member_by_member(ctx, launch):
    """The batched kernel under the read-ahead shape (5) and a persistent
    grid that walks several tiles per block gives the member-by-member
    states bit for bit."""
    sizes = [256, 200, 320, 128]
    alone = _members(ctx, sizes, seed0=43000)
    for s in alone:
        for _ in range(6):
            s.step(s.dt)
    expect = _states(alone)
    sims = _members(ctx, sizes, seed0=43000)
    b = BatchedEnsemble.BatchedCDKLM16(sims, launch=launch)
    b.advance(6)
    for e, g in zip(expect, _states(sims)):
        assert np.array_equal(e, g)


def _wind_members(ctx, sizes, seed0=45000):
    from SWESimulators.WindStress import WindStress
    sims = []
    for k, n in enumerate(sizes):
        c = SC.grf(n, dx=1000.0, seed_bathy=seed0 + k, seed_bumps=seed0 + 500 + k, steps=1)
        rng = np.random.default_rng(seed0 + 900 + k)
        kw = c.kwargs()
        kw["wind_stress"] = WindStress(t=[0], X=[rng.uniform(-0.2, 0.2, (6, 5)).astype(np.float32)],
                                       Y=[rng.uniform(-0.2, 0.2, (6, 5)).astype(np.float32)])
        sims.append(CDKLM16.CDKLM16(ctx, dt=c.dt, **kw))
    return sims


@pytest.mark.parametrize("launch", [(6, 16, 0), (5, 8, 0), (0, 16, 0), (4, 16, 148 * 5)])
def test_wind_field_batch_equals_member_by_member(ctx, launch):
    """Members with a per-cell wind field run the general kernel variant,
    128-wide whatever the launch shape: the tile list follows the kernel's
    width, and the read-ahead form gives the member-by-member states."""
    sizes = [256, 200, 130]
    alone = _wind_members(ctx, sizes)
    for s in alone:
        for _ in range(5):
            s.step(s.dt)
    expect = _states(alone)
    sims = _wind_members(ctx, sizes)
    b = BatchedEnsemble.BatchedCDKLM16(sims, launch=launch)
    b.advance(5)
    for e, g in zip(expect, _states(sims)):
        assert np.array_equal(e, g)


def test_batched_max_dt_equals_member_max_dt(ctx):
    """The one-launch CFL reduction over all members gives each member's own
    exact limit bit for bit, on uneven sizes, after steps and with land."""
    sims = _members(ctx, [128, 300, 96, 257], seed0=44000)
    c = SC.grf(64, ny=40, dx=1000.0, seed_bathy=44100, steps=1)
    Hi = c.Hi.copy()
    Hi[10:20, 10:30] = 1.0e20                        # a land patch (the mask value)
    kw = c.kwargs()
    kw["H"] = Hi
    sims.append(CDKLM16.CDKLM16(ctx, dt=c.dt, **kw))
    b = BatchedEnsemble.BatchedCDKLM16(sims)
    b.advance(3)
    got = b.max_dt()
    for m, s in enumerate(sims):
        s.updateDt(courant_number=1.0)
        assert np.float32(got[m]) == np.float32(s.dt), (m, got[m], s.dt)


def test_graph_replay_equals_plain_launches(ctx):
    sims_a = _members(ctx, [256] * 4, seed0=41000)
    sims_b = _members(ctx, [256] * 4, seed0=41000)
    a = BatchedEnsemble.BatchedCDKLM16(sims_a)
    b = BatchedEnsemble.BatchedCDKLM16(sims_b, graph_steps=5)
    a.advance(17)
    b.advance(17)            # 3 graph replays + 2 plain steps
    for x, y in zip(_states(sims_a), _states(sims_b)):
        assert np.array_equal(x, y)


def test_batched_step_t_end_semantics(ctx):
    sims = _members(ctx, [128, 128], seed0=42000)
    dt = min(s.dt for s in sims)
    for s in sims:
        s.dt = dt
    alone = _members(ctx, [128, 128], seed0=42000)
    for s in alone:
        s.dt = dt
        s.step(10.5 * dt)
    b = BatchedEnsemble.BatchedCDKLM16(sims)
    b.set_dt([dt, dt])
    b.step(10.5 * dt)
    for x, y in zip(_states(sims), _states(alone)):
        assert np.array_equal(x, y)
    assert sims[0].num_iterations == alone[0].num_iterations == 11


def test_autotune_domain_keeps_state(ctx, tmp_path, monkeypatch):
    monkeypatch.setenv("GOCEAN_TUNE_CACHE", str(tmp_path / "tune.json"))
    c = SC.grf(512, dx=1000.0, steps=1)
    sim = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
    ref = CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs())
    before = np.stack(sim.download())
    best, info = Autotune.tune_domain(sim, steps=3)
    assert np.array_equal(np.stack(sim.download()), before)
    for _ in range(5):
        sim.step(c.dt)
        ref.step(c.dt)
    assert np.array_equal(np.stack(sim.download()), np.stack(ref.download()))
    again, hit = Autotune.tune_domain(sim)           # from the cache
    assert again == best


def test_autotune_batch(ctx, tmp_path, monkeypatch):
    monkeypatch.setenv("GOCEAN_TUNE_CACHE", str(tmp_path / "tune.json"))
    sims = _members(ctx, [256] * 3, seed0=43000)
    b = BatchedEnsemble.BatchedCDKLM16(sims)
    before = _states(sims)
    res = Autotune.tune_batch(b, steps=3, graph_lengths=[4])
    for x, y in zip(before, _states(sims)):
        assert np.array_equal(x, y)
    assert res["graph_steps"] in (0, 4)
    b.advance(6)
    assert sims[0].num_iterations == 6


@pytest.mark.parametrize("lcg", [True, False])
def test_batched_model_error_equals_member_by_member(ctx, lcg):
    """Members with the reference's small-scale model error
    (small_scale_perturbation, OceanStateNoise): BatchedCDKLM16.step perturbs
    all of them after every step in three launches (go_noise_batch_perturb);
    each member ends bit for bit where its twin stepped alone with
    CDKLM16.step ends.  Members differ in f, amplitude and draws; then one
    more perturbation with q0_scale against perturbState."""
    from SWESimulators import CDKLM16, SyntheticCases as SC
    from SWESimulators.BatchedEnsemble import BatchedCDKLM16
    M = 5
    c = SC.grf(64, ny=48, dx=1000.0, bc=(2, 2, 2, 2), steps=1)

    def member(m):
        kw = c.kwargs()
        kw["f"] = np.float32(c.f * (1.0 + 0.1 * m))
        return CDKLM16.CDKLM16(ctx, dt=c.dt, small_scale_perturbation=True,
                               small_scale_perturbation_amplitude=1e-4 * (1 + m), use_lcg=lcg,
                               xorwow_seed=1000 + m, **kw)

    sims = [member(m) for m in range(M)]
    twins = [member(m) for m in range(M)]
    if lcg:
        for s, t in zip(sims, twins):
            seeds = s.small_scale_model_error.getSeed()
            t.small_scale_model_error.seed.upload(t.gpu_stream, seeds)
    ens = BatchedCDKLM16(sims)
    ens.step(7.5 * c.dt)                  # 7 steps and a half step, each perturbed
    ens.synchronize()
    for t in twins:
        t.step(7.5 * c.dt)
    for s, t in zip(sims, twins):
        for x, y in zip(s.download(), t.download()):
            assert np.array_equal(x, y)
        assert s.num_iterations == t.num_iterations == 8
    ens.perturb_members(q0_scale=0.37)
    ens.synchronize()
    for t in twins:
        t.perturbState(q0_scale=0.37)
    for s, t in zip(sims, twins):
        for x, y in zip(s.download(), t.download()):
            assert np.array_equal(x, y)
    e0, e1 = sims[0].download()[0], sims[1].download()[0]
    assert not np.array_equal(e0, e1)


def test_nonfinite_member_flagged_isolated_and_dropped(ctx):
    """A member whose initial eta holds NaN (made on the host) is flagged in
    its own status word; the other members step bit for bit as a batch
    without it, and the ensemble drops it and steps on unchanged
    (BaseOceanStateEnsemble.py:108-110, EnsembleFromFiles.py:315)."""
    sizes = [128, 96, 160, 128]
    sims = _members(ctx, sizes, seed0=47000)
    eta, hu, hv = sims[2].download()
    eta[40, 50] = np.nan
    sims[2].upload(eta, hu, hv)
    keep = [0, 1, 3]
    ref = [m for k, m in enumerate(_members(ctx, sizes, seed0=47000)) if k in keep]
    b = BatchedEnsemble.BatchedCDKLM16(sims)
    b.advance(10)
    b_ref = BatchedEnsemble.BatchedCDKLM16(ref)
    b_ref.advance(10)
    status = b.member_status()
    assert status[2] & 0x1 and all(status[k] == 0 for k in keep)
    assert b.failed_members() == [2]
    for k, r in zip(keep, ref):
        assert np.array_equal(np.stack(sims[k].download()), np.stack(r.download()))
    removed = b.drop(b.failed_members())
    assert removed == [sims[2]] and b.n == 3
    b.advance(7)
    b_ref.advance(7)
    for s, r in zip(b.sims, ref):
        assert np.array_equal(np.stack(s.download()), np.stack(r.download()))
    assert b.member_status() == [0, 0, 0]


def test_batched_members_vs_reference_kernel(ctx):
    """Four members of the config-2 physics on a 96 x 80 grid (beta plane,
    quadratic friction, wind, walls north/south, periodic east/west), each
    with its own GRF bathymetry, bumps and time step, stepped 200 times by
    the batched launch; every member against the reference kernel
    (CDKLM16_kernel.cu:429-1006, rebuilt for this GPU) on the same inputs,
    bit for bit with ghost cells, so the batch is tied to the reference and
    not only to the single-domain path."""
    from oracle import build_ref, ref_kernel
    from oracle import cdklm16_oracle as O
    cfg = build_ref.CONFIGS["small_beta"]
    if not ref_kernel.available(cfg):
        pytest.skip("reference kernel library not built")
    nx, ny = cfg["nx"], cfg["ny"]
    cases = []
    for m in range(4):
        c = SC.grf(nx, dx=500.0, steps=200, seed_bathy=20241 + 7 * m, seed_bumps=20242 + 7 * m)
        c.ny = ny
        c.Hi = O.fix_bi_ghost_corners(np.ascontiguousarray(c.Hi[: ny + 5]), nx, ny, c.bc)
        c.eta0 = np.ascontiguousarray(c.eta0[: ny + 4])
        c.hu0 = np.zeros_like(c.eta0)
        c.hv0 = np.zeros_like(c.eta0)
        c.dt = SC.cfl_dt(c)
        cases.append(c)
    sims = [CDKLM16.CDKLM16(ctx, dt=c.dt, **c.kwargs()) for c in cases]
    b = BatchedEnsemble.BatchedCDKLM16(sims)
    b.advance(200)
    assert b.member_status() == [0, 0, 0, 0]
    for c, s in zip(cases, sims):
        ref = ref_kernel.RefKernelSim(cfg, c.eta0, c.hu0, c.hv0, c.Hi, c.dt, c.f, c.beta, c.bc, wind=c.wind)
        for _ in range(200):
            ref.step(c.dt)
        for a, r in zip(s.download(), ref.download()):
            assert np.array_equal(a, r)
