"""Run the reference's own CDKLM16 kernel on the GPU (test oracle only).

Loads a library built by oracle/build_ref.py and replays the host side of
gpu_ocean/SWESimulators/CDKLM16.py for the RK2 path: Coriolis texture as
the constructor builds it (CDKLM16.py:146-148, 310-345, full resolution),
bathymetry (Common.py:1319-1389), eta0 = max(eta0, -Hm) (CDKLM16.py:237),
and the step() loop (CDKLM16.py:494-598).  Arrays use the reference's
unpadded pitch ((nx+4)*4 bytes, Common.py:546).

Only tests, smoke() and bench.py's reference arm import this module.
"""

import ctypes
import os

import numpy as np

from . import build_ref
from .cdklm16_oracle import coriolis_rows

_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float


def available(cfg, fmad=False):
    return os.path.exists(build_ref.lib_name(cfg, fmad))


def _load(cfg, fmad=False):
    path = build_ref.lib_name(cfg, fmad)
    if not os.path.exists(path):
        raise FileNotFoundError("reference kernel library %s not built (oracle/build_ref.py)" % path)
    lib = ctypes.CDLL(path)
    lib.ref_config.argtypes = [ctypes.POINTER(_I), ctypes.POINTER(_I)] + [ctypes.POINTER(_F)] * 4
    lib.ref_setup.argtypes = [ctypes.POINTER(_F), _I, _I, _F, _F, _F, _F, _F]
    lib.ref_set_wind.argtypes = [ctypes.POINTER(_F)] * 4 + [_I, _I]
    lib.ref_bathymetry.argtypes = [_P, _I, _I, _P, _I, _F, _P, _I]
    lib.ref_boundary.argtypes = [_P, _I, _I, _P, _P, _P, _I]
    lib.ref_stage.argtypes = [_P, _F, _I, _P, _P, _P, _I, _P, _P, _P, _I, _P, _I, _P, _I, _F, _F, _I]
    lib.ref_step.argtypes = [_P, _I, _F, _F, _P, _P, _P, _I, _P, _P, _P, _I, _P, _I, _P, _I, _F, _I]
    lib.ref_max_dt.argtypes = [_P, _P, _P, _P, _I, _P, _I, _F, _P, _P]
    lib.ref_set_drift_wind.argtypes = [ctypes.POINTER(_F)] * 4 + [_I, _I]
    lib.ref_set_open_bc.argtypes = [ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_F), ctypes.POINTER(_F),
                                    _I, ctypes.POINTER(_F), ctypes.POINTER(_F), _I, _F]
    lib.ref_set_bc_t.argtypes = [_F]
    lib.refr_drift.argtypes = [_P, _I, _I, _F, _F, _F, _I, _I, _P, _I, _P, _I, _P, _I, _P, _I, _I, _I, _I, _P, _I,
                               _F, _F, _F]
    lib.refr_enforce_bc.argtypes = [_P, _F, _F, _I, _I, _I, _P, _I]
    lib.refr_observe.argtypes = [_P, _I, _I, _F, _F, _I, _I, _P, _I, _P, _I, _P, _I, _F, _I, _P, _I, _P, _I]
    lib.ref_noise_textures.argtypes = [ctypes.POINTER(_F), _I, _I, ctypes.POINTER(_F), _I, _I]
    lib.refn_lcg.argtypes = [_P, _I, _I, _I, _I, _P, _I, _P, _I]
    lib.refn_soar.argtypes = [_P, _I, _I, _F, _F, _F, _F, _F, _I, _I, _P, _I, _P, _I, _I]
    lib.refn_geostrophic.argtypes = [_P, _I, _I, _F, _F, _I, _I, _F, _F, _F, _F, _P, _I, _P, _I, _P, _I, _P, _I,
                                     _P, _I, _F]
    lib.refn_bicubic.argtypes = [_P, _I, _I, _I, _I, _F, _F, _I, _I, _I, _I, _F, _F, _I, _I, _F, _F, _F, _F, _P, _I,
                                 _P, _I, _P, _I, _P, _I, _P, _I, _F]
    lib.refn_make_perpendicular.argtypes = [_P, _I, _I, _P, _I, _P, _I, _P]
    return lib


def _chk(rc, what):
    if rc != 0:
        raise RuntimeError("reference kernel call %s failed with CUDA error %d" % (what, rc))


def _p(t):
    return ctypes.c_void_p(int(t.data_ptr()))


class RefKernelSim:
    """Reference CDKLM16 RK2 simulation on the GPU (wall/periodic, f- or
    beta-plane, uniform wind or wind arrays, a constant grid angle)."""

    def __init__(self, cfg, eta0, hu0, hv0, Hi, dt, f, coriolis_beta=0.0, bc=(1, 1, 1, 1),
                 wind=(0.0, 0.0), fmad=False, f_rows=None, wind_fields=None, angle=0.0):
        import torch
        self.torch = torch
        self.lib = _load(cfg, fmad)
        nx, ny = cfg["nx"], cfg["ny"]
        self.nx, self.ny = nx, ny
        self.bc = tuple(int(b) for b in bc)
        self.bc_packed = (self.bc[0] << 24) | (self.bc[2] << 16) | (self.bc[1] << 8) | self.bc[3]
        if f_rows is None:
            if coriolis_beta == 0.0:
                ftex = np.array([[np.float32(f)]], dtype=np.float32)
            else:
                f_rows = coriolis_rows(f, coriolis_beta, ny, cfg["dy"])
        if f_rows is not None:
            ftex = np.ascontiguousarray(np.repeat(np.asarray(f_rows, np.float32)[:, None], nx + 4, axis=1))
        fh, fw = ftex.shape
        _chk(self.lib.ref_setup(ftex.ctypes.data_as(ctypes.POINTER(_F)), fw, fh, float(np.float32(angle)),
                                float(wind[0]), float(wind[0]), float(wind[1]), float(wind[1])), "setup")
        if wind_fields is not None:
            # (X current, X next, Y current, Y next) arrays of one shape
            arrs = [np.ascontiguousarray(np.asarray(a, dtype=np.float32)) for a in wind_fields]
            wh, ww = arrs[0].shape
            _chk(self.lib.ref_set_wind(*[a.ctypes.data_as(ctypes.POINTER(_F)) for a in arrs], ww, wh),
                 "set_wind")
            self._wind_fields = arrs
        dev = "cuda"
        self.stream = torch.cuda.current_stream()
        s = ctypes.c_void_p(int(self.stream.cuda_stream))
        self.s = s
        self.Hi = torch.from_numpy(np.ascontiguousarray(Hi, dtype=np.float32)).to(dev)
        self.Bm = torch.zeros((ny + 4, nx + 4), dtype=torch.float32, device=dev)
        self.land = np.float32(1e20)
        _chk(self.lib.ref_bathymetry(s, self.bc[0], self.bc[1], _p(self.Hi), (nx + 5) * 4, float(self.land),
                                     _p(self.Bm), (nx + 4) * 4), "bathymetry")
        Bm = self.Bm.cpu().numpy()
        eta0 = np.maximum(np.asarray(eta0, np.float32), -Bm)
        self.h0 = [torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev) for a in (eta0, hu0, hv0)]
        self.h1 = [a.clone() for a in self.h0]
        self.pitch = (nx + 4) * 4
        self.dt = dt
        self.t = 0.0
        self.num_iterations = 0
        self.dt_blocks = torch.zeros(((ny + 31) // 32) * ((nx + 11) // 12) + 1, dtype=torch.float32, device=dev)
        self.dt_out = torch.zeros(1, dtype=torch.float32, device=dev)

    def boundary(self, Q):
        _chk(self.lib.ref_boundary(self.s, self.bc[0], self.bc[1], _p(Q[0]), _p(Q[1]), _p(Q[2]), self.pitch),
             "boundary")

    def run_steps(self, n, dt, wind_t=0.0):
        h0, h1 = self.h0, self.h1
        _chk(self.lib.ref_step(self.s, int(n), float(dt), float(wind_t), _p(h0[0]), _p(h0[1]), _p(h0[2]),
                               self.pitch, _p(h1[0]), _p(h1[1]), _p(h1[2]), self.pitch, _p(self.Hi),
                               (self.nx + 5) * 4, _p(self.Bm), self.pitch, float(self.land), self.bc_packed),
             "step")

    def stage(self, rk_step, dt, Qin, Qout, wind_t=0.0):
        _chk(self.lib.ref_stage(self.s, float(dt), int(rk_step), _p(Qin[0]), _p(Qin[1]), _p(Qin[2]), self.pitch,
                                _p(Qout[0]), _p(Qout[1]), _p(Qout[2]), self.pitch, _p(self.Hi), (self.nx + 5) * 4,
                                _p(self.Bm), self.pitch, float(self.land), float(wind_t), self.bc_packed), "stage")

    def set_open_bc(self, codes, sponge, t, ns, ew):
        """Open boundaries: codes and sponge widths (north, east, south,
        west); the exterior solution at two times t = (t0, t1) as NS texels
        [(2, L, 4) per time: row 0 south, row 1 north] and EW texels
        [(L, 2, 4): column 0 west, column 1 east], as
        BoundaryConditionsArakawaA.update_bc_values packs them."""
        self._open_t = (float(t[0]), float(t[1]))
        ns = [np.ascontiguousarray(a, dtype=np.float32) for a in ns]
        ew = [np.ascontiguousarray(a, dtype=np.float32) for a in ew]
        self._open_data = (ns, ew)
        c = (_I * 4)(*[int(x) for x in codes])
        sp = (_I * 4)(*[int(x) for x in sponge])
        P = lambda a: a.ctypes.data_as(ctypes.POINTER(_F))
        _chk(self.lib.ref_set_open_bc(c, sp, P(ns[0]), P(ns[1]), ns[0].shape[1], P(ew[0]), P(ew[1]), ew[0].shape[0],
                                      float(self._bc_t(0.0))), "set_open_bc")

    def _bc_t(self, t):
        t0, t1 = self._open_t
        return np.float32(max(0.0, min(1.0, (t - t0) / max(1.0e-10, t1 - t0))))

    def step(self, t_end):
        """CDKLM16.step(t_end) (CDKLM16.py:494-598) with constant wind."""
        open_bc = getattr(self, "_open_t", None) is not None
        if self.t == 0:
            if open_bc:
                self.lib.ref_set_bc_t(float(self._bc_t(self.t)))
            self.boundary(self.h0)
        t_now = 0.0
        while t_now < t_end:
            local_dt = np.float32(min(self.dt, np.float32(t_end - t_now)))
            if open_bc:
                self.lib.ref_set_bc_t(float(self._bc_t(self.t)))
            self.run_steps(1, local_dt)
            self.t += np.float64(local_dt)
            t_now += np.float64(local_dt)
            self.num_iterations += 1
        return self.t

    def max_dt(self):
        Q = self.h0
        _chk(self.lib.ref_max_dt(self.s, _p(Q[0]), _p(Q[1]), _p(Q[2]), self.pitch, _p(self.Bm), self.pitch,
                                 float(self.land), _p(self.dt_blocks), _p(self.dt_out)), "max_dt")
        return float(self.dt_out.cpu().numpy()[0])

    def download(self):
        self.torch.cuda.synchronize()
        return tuple(a.cpu().numpy() for a in self.h0)

    def download_prev(self):
        self.torch.cuda.synchronize()
        return tuple(a.cpu().numpy() for a in self.h1)


class RefDrifters:
    """The reference's drifter kernels (passiveDrifterKernel,
    enforceBoundaryConditions, observeUnderlyingFlow) on their own device
    positions: (n + 1) x 2 float32, the last row the observation.  Flow
    arrays are (tensor, pitch in bytes) pairs of the ghost-inclusive grid."""

    def __init__(self, cfg, positions, observation, wind_fields=None):
        import torch
        self.torch = torch
        self.lib = _load(cfg)
        rows = np.concatenate([np.asarray(positions, np.float32).reshape(-1, 2),
                               np.asarray(observation, np.float32).reshape(1, 2)])
        self.n = rows.shape[0] - 1
        self.pos = torch.from_numpy(np.ascontiguousarray(rows)).cuda()
        self.s = ctypes.c_void_p(int(torch.cuda.current_stream().cuda_stream))
        if wind_fields is not None:
            arrs = [np.ascontiguousarray(np.asarray(a, dtype=np.float32)) for a in wind_fields]
            wh, ww = arrs[0].shape
            _chk(self.lib.ref_set_drift_wind(*[a.ctypes.data_as(ctypes.POINTER(_F)) for a in arrs], ww, wh),
                 "set_drift_wind")
            self._wind = arrs

    def drift(self, eta, hu, hv, Hm, nx, ny, dx, dy, dt, periodic_ns, periodic_ew, sensitivity=1.0,
              wind_t=0.0, wind_drift_factor=0.0):
        _chk(self.lib.refr_drift(self.s, nx, ny, float(dx), float(dy), float(dt), 2, 2, _p(eta[0]), eta[1],
                                 _p(hu[0]), hu[1], _p(hv[0]), hv[1], _p(Hm[0]), Hm[1], int(periodic_ns),
                                 int(periodic_ew), self.n, _p(self.pos), 8, float(sensitivity), float(wind_t),
                                 float(wind_drift_factor)), "drift")

    def enforce_bc(self, size_x, size_y, periodic_ns, periodic_ew):
        _chk(self.lib.refr_enforce_bc(self.s, float(size_x), float(size_y), int(periodic_ns), int(periodic_ew),
                                      self.n, _p(self.pos), 8), "enforce_bc")

    def observe(self, eta, hu, hv, nx, ny, dx, dy):
        out = self.torch.zeros((max(self.n, 1), 2), dtype=self.torch.float32, device="cuda")
        _chk(self.lib.refr_observe(self.s, nx, ny, float(dx), float(dy), 2, 2, _p(eta[0]), eta[1], _p(hu[0]), hu[1],
                                   _p(hv[0]), hv[1], 0.0, self.n, _p(self.pos), 8, _p(out), 8), "observe")
        self.torch.cuda.synchronize()
        return out[:self.n].cpu().numpy()

    def positions(self):
        self.torch.cuda.synchronize()
        return self.pos.cpu().numpy()


class RefNoise:
    """The reference's model-error kernels (normalDistribution,
    uniformDistribution, SOAR, geostrophicBalance, bicubicInterpolation,
    makePerpendicular from ocean_noise.cu, --use_fast_math) on caller
    tensors given as (tensor, pitch in bytes) pairs, on the current torch
    stream.  The angle and Coriolis textures are host arrays."""

    def __init__(self, cfg, angle=((0.0,),), coriolis=((0.0,),)):
        import torch
        self.torch = torch
        self.lib = _load(cfg)
        self.s = ctypes.c_void_p(int(torch.cuda.current_stream().cuda_stream))
        a = np.ascontiguousarray(np.asarray(angle, dtype=np.float32))
        c = np.ascontiguousarray(np.asarray(coriolis, dtype=np.float32))
        self._tex = (a, c)
        _chk(self.lib.ref_noise_textures(a.ctypes.data_as(ctypes.POINTER(_F)), a.shape[1], a.shape[0],
                                         c.ctypes.data_as(ctypes.POINTER(_F)), c.shape[1], c.shape[0]), "textures")

    def lcg(self, normal, seed_nx, seed_ny, random_nx, seed, random):
        _chk(self.lib.refn_lcg(self.s, int(normal), seed_nx, seed_ny, random_nx, _p(seed[0]), seed[1],
                               _p(random[0]), random[1]), "lcg")

    def soar(self, cnx, cny, cdx, cdy, q0, L, scale, pns, pew, random, coarse, additive=0):
        _chk(self.lib.refn_soar(self.s, cnx, cny, float(cdx), float(cdy), float(q0), float(L), float(scale),
                                int(pns), int(pew), _p(random[0]), random[1], _p(coarse[0]), coarse[1],
                                int(additive)), "soar")

    def geostrophic(self, nx, ny, dx, dy, g, f, beta, coarse, eta, hu, hv, Hi, land=1e20, gx=2, gy=2):
        _chk(self.lib.refn_geostrophic(self.s, nx, ny, float(dx), float(dy), gx, gy, float(g), float(f),
                                       float(beta), 0.0, _p(coarse[0]), coarse[1], _p(eta[0]), eta[1], _p(hu[0]),
                                       hu[1], _p(hv[0]), hv[1], _p(Hi[0]), Hi[1], float(land)), "geostrophic")

    def bicubic(self, nx, ny, dx, dy, cnx, cny, cdx, cdy, oi, oj, g, f, beta, coarse, eta, hu, hv, Hi, land=1e20,
                gx=2, gy=2):
        _chk(self.lib.refn_bicubic(self.s, nx, ny, gx, gy, float(dx), float(dy), cnx, cny, gx, gy, float(cdx),
                                   float(cdy), int(oi), int(oj), float(g), float(f), float(beta), 0.0, _p(coarse[0]),
                                   coarse[1], _p(eta[0]), eta[1], _p(hu[0]), hu[1], _p(hv[0]), hv[1], _p(Hi[0]),
                                   Hi[1], float(land)), "bicubic")

    def make_perpendicular(self, nx, ny, xi, nu, red):
        _chk(self.lib.refn_make_perpendicular(self.s, nx, ny, _p(xi[0]), xi[1], _p(nu[0]), nu[1], _p(red)),
             "make_perpendicular")
