"""NetCDF output and restart on the GPU (CDKLM16 write_netcdf, writeState,
fromfilename), after the reference's NetCDF test
(gpu_ocean/tests/schemes/NetCDF_test.py): a simulator with the stochastic
model error writes its initial state, is restarted from the file, and the
two agree in every scalar attribute, in their model errors and in their
states, before and after 100 steps.  A run restarted from its last record
continues bit for bit like the uninterrupted run."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from SWESimulators import CDKLM16, Common, SimReader, SyntheticCases as SC  # noqa: E402


@pytest.fixture(scope="module")
def ctx():
    return Common.CUDAContext()


def _kwargs(bc=(2, 2, 2, 2)):
    c = SC.grf(96, ny=80, dx=500.0, bc=bc, steps=1)
    kw = c.kwargs()
    kw["coriolis_beta"] = 0.0
    # the files name the wind's source only, so a restart runs without wind
    # (CDKLM16.py:470-476); so do these runs
    kw.pop("wind_stress", None)
    return c, kw


def _scalars(obj):
    out = {}
    for attr in dir(obj):
        if attr.startswith("_"):
            continue
        v = getattr(obj, attr)
        if np.isscalar(v):
            out[attr] = v
    return out


def test_netcdf_restart_matches_writer(ctx, tmp_path):
    c, kw = _kwargs()
    name = str(tmp_path / "netcdf_test" / "netcdf_test.nc")
    sim = CDKLM16.CDKLM16(ctx, dt=c.dt, write_netcdf=True, netcdf_filename=name, small_scale_perturbation=True,
                          small_scale_perturbation_amplitude=1e-4, use_lcg=True, **kw)
    sim.closeNetCDF()
    file_sim = CDKLM16.CDKLM16.fromfilename(ctx, name, cont_write_netcdf=False, use_lcg=True)
    a, b = _scalars(sim), _scalars(file_sim)
    assert set(a) == set(b)
    for k in a:
        x, y = (round(a[k]), round(b[k])) if k == "t" else (a[k], b[k])
        assert x == y, (k, a[k], b[k])
    ma, mb = _scalars(sim.small_scale_model_error), _scalars(file_sim.small_scale_model_error)
    for k in ma:
        assert ma[k] == mb[k], (k, ma[k], mb[k])
    for x, y in zip(sim.download(), file_sim.download()):
        assert np.array_equal(x, y)
    dt = sim.dt
    sim.step(100 * dt, apply_stochastic_term=False)
    file_sim.step(100 * dt, apply_stochastic_term=False)
    for x, y in zip(sim.download(), file_sim.download()):
        assert np.array_equal(x, y)
    assert np.abs(sim.download()[1]).max() > 0


def test_run_restart_continue(ctx, tmp_path):
    c, kw = _kwargs(bc=(1, 2, 1, 2))
    ref = CDKLM16.CDKLM16(ctx, dt=c.dt, **kw)
    for _ in range(10):
        ref.step(10 * c.dt)
    name = str(tmp_path / "run.nc")
    sim = CDKLM16.CDKLM16(ctx, dt=c.dt, write_netcdf=True, netcdf_filename=str(tmp_path / "run"), **kw)
    for _ in range(5):
        sim.step(10 * c.dt)             # one record per step() call
    sim.writeState()                    # and one more of the same state
    sim.cleanUp()
    r = SimReader.SimNetCDFReader(name, ignore_ghostcells=False)
    assert r.getNumTimeSteps() == 7 and r.getBC().codes() == (1, 2, 1, 2)
    t = r.getTimes()
    assert t[0] == 0 and abs(t[5] - 50 * c.dt) < 1e-3 and t[6] == t[5]
    r.close()
    cont = CDKLM16.CDKLM16.fromfilename(ctx, name, cont_write_netcdf=True,
                                        new_netcdf_filename=str(tmp_path / "cont"))
    for _ in range(5):
        cont.step(10 * c.dt)
    for x, y in zip(ref.download(), cont.download()):
        assert np.array_equal(x, y)
    cont.closeNetCDF()
    r = SimReader.SimNetCDFReader(str(tmp_path / "cont.nc"), ignore_ghostcells=True)
    eta, hu, hv, _ = r.getLastTimeStep()
    assert np.array_equal(hu, ref.download(interior_domain_only=True)[1])
    r.close()
