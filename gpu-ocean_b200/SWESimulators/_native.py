"""ctypes binding of the in-tree C ABI (include/gocean.h, lib/libgocean.so).

There is no CPU fallback: if the shared library is missing, or no CUDA
device is present when a kernel is called, the call raises.
"""

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libgocean.so")
# GOCEAN_DEBUG_BOUNDS=1 selects the checked-index build of the stage kernels
# (lib/libgocean_debug.so: every global access and shared ring read tests its
# index, flags GO_STATUS_BOUNDS and skips the access when it is outside)
if os.environ.get("GOCEAN_DEBUG_BOUNDS") == "1":
    LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libgocean_debug.so")

GO_OK = 0
GO_BC_WALL = 1
GO_BC_PERIODIC = 2
GO_FRICTION_QUADRATIC = 0
GO_FRICTION_LINEAR = 1
GO_STATUS_NONFINITE = 0x1
GO_STATUS_ADJ_SCOPE = 0x2
GO_STATUS_TIMEOUT = 0x4
GO_STATUS_BOUNDS = 0x8
GO_DEBUG_SKIP_TMA = 0x1
GO_ERR_INVALID = -1
GO_ERR_CUDA = -2
GO_ERR_UNSUPPORTED = -3
GO_ARITH_EXACT = 0
GO_ARITH_RCP = 1
GO_ADJ_AUTO = 0
GO_ADJ_TILE = 1
GO_ADJ_MARCH64 = 2
GO_ADJ_MARCH128 = 3

_c_float_p = ctypes.c_void_p  # device pointers travel as integers


class GoDomainDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("dx", ctypes.c_float), ("dy", ctypes.c_float),
        ("g", ctypes.c_float), ("r", ctypes.c_float),
        ("theta", ctypes.c_float),
        ("desing_eps", ctypes.c_float), ("flux_slope_eps", ctypes.c_float),
        ("depth_cutoff", ctypes.c_float),
        ("rk_order", ctypes.c_int),
        ("bc_north", ctypes.c_int), ("bc_east", ctypes.c_int),
        ("bc_south", ctypes.c_int), ("bc_west", ctypes.c_int),
        ("friction_law", ctypes.c_int),
        ("north_x", ctypes.c_float), ("north_y", ctypes.c_float),
    ]


class GoState(ctypes.Structure):
    """go_state: three device arrays sharing a pitch in bytes."""
    _fields_ = [("eta", ctypes.c_void_p), ("hu", ctypes.c_void_p), ("hv", ctypes.c_void_p),
                ("pitch", ctypes.c_int)]


_SP = ctypes.POINTER(GoState)


class GoNoiseMember(ctypes.Structure):
    """go_noise_member: one ensemble member's model-error buffers."""
    _fields_ = [("seed", ctypes.c_void_p), ("xorwow_states", ctypes.c_void_p), ("random", ctypes.c_void_p),
                ("coarse", ctypes.c_void_p), ("eta", ctypes.c_void_p), ("hu", ctypes.c_void_p),
                ("hv", ctypes.c_void_p), ("Hi", ctypes.c_void_p), ("angle_texture", ctypes.c_uint64),
                ("coriolis_texture", ctypes.c_uint64), ("seed_pitch", ctypes.c_int), ("random_pitch", ctypes.c_int),
                ("coarse_pitch", ctypes.c_int), ("eta_pitch", ctypes.c_int), ("hu_pitch", ctypes.c_int),
                ("hv_pitch", ctypes.c_int), ("Hi_pitch", ctypes.c_int), ("n_generators", ctypes.c_int),
                ("soar_q0", ctypes.c_float), ("g", ctypes.c_float), ("f", ctypes.c_float), ("beta", ctypes.c_float),
                ("land_value", ctypes.c_float), ("reserved", ctypes.c_float)]

# name -> (restype, argtypes)
_P = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
SIGNATURES = {
    "go_domain_create": (_I, [ctypes.POINTER(GoDomainDesc), ctypes.POINTER(ctypes.c_void_p)]),
    "go_domain_destroy": (_I, [_P]),
    "go_domain_set_coriolis": (_I, [_P, ctypes.POINTER(ctypes.c_float), _I]),
    "go_domain_set_wind_uniform": (_I, [_P, _F, _F, _F, _F]),
    "go_domain_set_wind_field": (_I, [_P, _P, _P, _P, _P, _I]),
    "go_domain_set_launch": (_I, [_P, _I, _I]),
    "go_domain_set_arith": (_I, [_P, _I]),
    "go_check_quotients": (_I, [_P, _P, _P, _I, _P, _P]),
    "go_domain_set_land": (_I, [_P, _I]),
    "go_init_bathymetry": (_I, [_P, _P, _P, _I, _P, _I, _F]),
    "go_boundary_condition": (_I, [_P, _P, _P, _P, _P, _I]),
    "go_cdklm_swe_2D": (_I, [_P, _P, _F, _I, _P, _I, _P, _I, _P, _I, _P, _I, _P, _I, _P, _I,
                             _P, _I, _P, _I, _F, _F, _I]),
    "go_cdklm_step": (_I, [_P, _P, _I, _F, _F, _P, _P, _P, _I, _P, _P, _P, _I, _P, _I, _F]),
    "go_cdklm_step_static": (_I, [ctypes.POINTER(GoDomainDesc), _P, ctypes.POINTER(ctypes.c_float), _I, _F, _F,
                                  _I, _F, _P, _P, _P, _I, _P, _P, _P, _I, _P, _I, _F,
                                  ctypes.POINTER(ctypes.c_uint32)]),
    "go_domain_set_adjoint_launch": (_I, [_P, _I, _I]),
    "go_adjoint_batch_create": (_I, [ctypes.POINTER(ctypes.c_void_p), _I, ctypes.POINTER(ctypes.c_void_p)]),
    "go_adjoint_batch_destroy": (_I, [_P]),
    "go_adjoint_batch_set_launch": (_I, [_P, _I, _I]),
    "go_adjoint_batch_set_member": (_I, [_P, _I, _F, _SP, _SP, _SP, _SP, _SP, _SP, _P, _P, _I, _P, _I]),
    "go_adjoint_batch_step": (_I, [_P, _P]),
    "go_traj_step": (_I, [_P, _P, _F, _F, _SP, _SP, _SP, _P, _I, _F]),
    "go_adjoint_stage": (_I, [_P, _P, _I, _F, _SP, _SP, _SP, _SP, _SP, _P, _P, _I, _P, _I]),
    "go_adjoint_step": (_I, [_P, _P, _F, _SP, _SP, _SP, _SP, _SP, _SP, _SP, _P, _P, _I, _P, _I]),
    "go_obs_misfit": (_I, [_P, _SP, _I, _I, _I, _P, _P, _F, _F, _P]),
    "go_obs_adjoint": (_I, [_P, _SP, _SP, _I, _I, _I, _P, _P, _F, _F]),
    "go_grf_scratch_floats": (ctypes.c_size_t, [_I, _I, _F]),
    "go_grf_perturb": (_I, [_P, _P, _P, _I, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _F, _F, _P,
                            ctypes.c_size_t]),
    "go_batch_grf_scratch_floats": (ctypes.c_size_t, [_P, _F]),
    "go_batch_grf_perturb": (_I, [_P, _P, ctypes.c_uint32, ctypes.c_uint32, _F, _F, _P, ctypes.c_size_t]),
    "go_max_dt": (_I, [_P, _P, _P, _P, _P, _I, _P, _I, _F, _P]),
    "go_batch_max_dt": (_I, [_P, _P, _P]),
    "go_sample_wind": (_I, [_P, _P, _I, _I, _I, _I, _P, _I]),
    "go_north_vector": (_I, [_F, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    "go_wind_texture_create": (_I, [_P, _I, _I, ctypes.POINTER(ctypes.c_uint64)]),
    "go_wind_texture_destroy": (_I, [ctypes.c_uint64]),
    "go_drift_passive": (_I, [_P, _I, _I, _F, _F, _F, _I, _I, _P, _I, _P, _I, _P, _I, _P, _I, _I, _I, _I, _P, _I,
                              _F, _F, _F, _P]),
    "go_drift_enforce_bc": (_I, [_P, _F, _F, _I, _I, _I, _P, _I]),
    "go_observe_flow": (_I, [_P, _I, _I, _F, _F, _I, _I, _P, _I, _P, _I, _I, _P, _I, _P, _I]),
    "go_domain_set_sponge": (_I, [_P, _I, _I, _I, _I]),
    "go_bc_texture_create": (_I, [_P, _I, _I, ctypes.POINTER(ctypes.c_uint64)]),
    "go_domain_set_open_bc": (_I, [_P, _P, _F]),
    "go_domain_status": (_I, [_P, ctypes.POINTER(ctypes.c_uint32), _I]),
    "go_batch_status": (_I, [_P, _P, _I]),
    "go_domain_stage_launches": (_I, [_P, _P]),
    "go_domain_set_debug": (_I, [_P, ctypes.c_uint32]),
    "go_batch_run_events": (_I, [_P, _P, ctypes.c_uint32, _I, ctypes.c_double, _F, ctypes.c_double,
                                 ctypes.c_uint32, _F, _F, _P, ctypes.c_size_t, _P, _P, _P]),
    "go_noise_lcg": (_I, [_P, _I, _I, _I, _I, _P, _I, _P, _I]),
    "go_noise_xorwow_state_bytes": (ctypes.c_size_t, []),
    "go_noise_xorwow_init": (_I, [_P, ctypes.c_uint64, _I, _P]),
    "go_noise_xorwow_fill": (_I, [_P, _I, _I, _P, _I, _I, _P, _I]),
    "go_noise_soar": (_I, [_P, _I, _I, _F, _F, _F, _F, _F, _I, _I, _P, _I, _P, _I, _I]),
    "go_noise_geostrophic": (_I, [_P, _I, _I, _F, _F, _I, _I, _F, _F, _F, _F, _P, _I, _P, _I, _P, _I, _P, _I,
                                  _P, _I, _F, ctypes.c_uint64, ctypes.c_uint64]),
    "go_noise_bicubic": (_I, [_P, _I, _I, _I, _I, _F, _F, _I, _I, _I, _I, _F, _F, _I, _I, _F, _F, _F, _F, _P, _I,
                              _P, _I, _P, _I, _P, _I, _P, _I, _F, ctypes.c_uint64, ctypes.c_uint64]),
    "go_noise_batch_create": (_I, [_P, _I, _I, _I, _F, _F, _I, _I, _F, _I, _I, _I, ctypes.POINTER(ctypes.c_void_p)]),
    "go_noise_batch_destroy": (_I, [_P]),
    "go_noise_batch_perturb": (_I, [_P, _P, ctypes.c_double, _F, _I]),
    "go_noise_reduce_scratch_bytes": (ctypes.c_size_t, []),
    "go_noise_square_sums": (_I, [_P, _I, _I, _P, _I, _P, _I, _P, _P, ctypes.c_size_t]),
    "go_noise_make_perpendicular": (_I, [_P, _I, _I, _P, _I, _P, _I, _P]),
    "go_batch_create": (_I, [ctypes.POINTER(ctypes.c_void_p), _I, ctypes.POINTER(ctypes.c_void_p)]),
    "go_batch_destroy": (_I, [_P]),
    "go_batch_set_member": (_I, [_P, _I, _F, _P, _P, _P, _I, _P, _P, _P, _I, _P, _I, _F, _F]),
    "go_batch_set_launch": (_I, [_P, _I, _I, _I]),
    "go_batch_set_arith": (_I, [_P, _I]),
    "go_batch_set_dt": (_I, [_P, _P, ctypes.POINTER(ctypes.c_float)]),
    "go_batch_tiles": (_I, [_P, ctypes.POINTER(_I)]),
    "go_batch_step": (_I, [_P, _P, _I]),
    "go_batch_graph_capture": (_I, [_P, _P, _I]),
    "go_batch_graph_launch": (_I, [_P, _P, ctypes.POINTER(_I)]),
    "go_last_error": (ctypes.c_char_p, []),
    "go_version": (ctypes.c_char_p, []),
}

_lib = None


class NativeError(RuntimeError):
    pass


def load():
    """Load lib/libgocean.so (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NativeError("CUDA library %s is missing; build it with gpu-ocean_b200/build.py" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc):
    if rc != GO_OK:
        msg = load().go_last_error().decode()
        raise NativeError("gocean error %d: %s" % (rc, msg))
    return rc


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise NativeError("no CUDA device: the CDKLM16 step runs on the GPU only")
    return torch


def ptr(t):
    return ctypes.c_void_p(int(t.data_ptr()))


def stream_handle(stream):
    if stream is None:
        return ctypes.c_void_p(0)
    return ctypes.c_void_p(int(stream.cuda_stream))


def north_vector(angle):
    """(sin a, cos a) of a float32 grid angle as the device computes it
    (go_north_vector)."""
    nx_, ny_ = ctypes.c_float(), ctypes.c_float()
    check(load().go_north_vector(float(np.float32(angle)), ctypes.byref(nx_), ctypes.byref(ny_)))
    return np.float32(nx_.value), np.float32(ny_.value)


def pack_bc(north, east, south, west):
    """The packed boundary code of CDKLM16.callKernel (CDKLM16.py:620-624)."""
    return (int(north) << 24) | (int(south) << 16) | (int(east) << 8) | int(west)


class Domain:
    """Owner of one go_domain handle (scheme constants, Coriolis table, wind)."""

    def __init__(self, nx, ny, dx, dy, g, r=0.0, theta=1.3, desing_eps=0.1,
                 flux_slope_eps=0.1, depth_cutoff=1.0e-5, bc=(1, 1, 1, 1),
                 friction_law=GO_FRICTION_QUADRATIC, north=(0.0, 1.0), rk_order=2):
        lib = load()
        d = GoDomainDesc()
        d.nx, d.ny = int(nx), int(ny)
        d.dx, d.dy, d.g, d.r, d.theta = float(dx), float(dy), float(g), float(r), float(theta)
        d.desing_eps, d.flux_slope_eps, d.depth_cutoff = float(desing_eps), float(flux_slope_eps), float(depth_cutoff)
        d.rk_order = int(rk_order)
        d.bc_north, d.bc_east, d.bc_south, d.bc_west = (int(b) for b in bc)
        d.friction_law = int(friction_law)
        d.north_x, d.north_y = float(north[0]), float(north[1])
        h = ctypes.c_void_p()
        check(lib.go_domain_create(ctypes.byref(d), ctypes.byref(h)))
        self.desc = d
        self.handle = h
        self.nx, self.ny = int(nx), int(ny)
        self.bc = tuple(int(b) for b in bc)
        self.bc_packed = pack_bc(*self.bc)

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            load().go_domain_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_coriolis(self, f_rows):
        a = np.ascontiguousarray(np.asarray(f_rows, dtype=np.float32).reshape(-1))
        check(load().go_domain_set_coriolis(self.handle, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), a.size))

    def set_wind_uniform(self, x_cur, x_next, y_cur, y_next):
        check(load().go_domain_set_wind_uniform(self.handle, float(x_cur), float(x_next), float(y_cur), float(y_next)))

    def set_wind_field(self, x_cur, x_next, y_cur, y_next):
        """Four device tensors (ny, nx) float32 with a common row stride."""
        if x_cur is None:
            check(load().go_domain_set_wind_field(self.handle, None, None, None, None, 0))
            return
        pitch = x_cur.stride(0) * 4
        for t in (x_next, y_cur, y_next):
            assert t.stride(0) * 4 == pitch
        check(load().go_domain_set_wind_field(self.handle, ptr(x_cur), ptr(x_next), ptr(y_cur), ptr(y_next), pitch))

    def set_sponge(self, north, east, south, west):
        check(load().go_domain_set_sponge(self.handle, int(north), int(east), int(south), int(west)))

    def set_open_bc(self, textures, bc_t):
        arr = (ctypes.c_uint64 * 4)(*[int(t) for t in textures])
        check(load().go_domain_set_open_bc(self.handle, arr, float(np.float32(bc_t))))

    def set_launch(self, shape=0, rows_per_block=0):
        check(load().go_domain_set_launch(self.handle, int(shape), int(rows_per_block)))

    def set_arith(self, mode):
        check(load().go_domain_set_arith(self.handle, int(mode)))

    def set_land(self, may_have_land):
        check(load().go_domain_set_land(self.handle, int(bool(may_have_land))))

    def status(self, clear=False):
        v = ctypes.c_uint32()
        check(load().go_domain_status(self.handle, ctypes.byref(v), int(bool(clear))))
        return int(v.value)

    def set_debug(self, flags):
        """Test hooks (GO_DEBUG_*; 0 in normal runs)."""
        check(load().go_domain_set_debug(self.handle, int(flags)))

    def stage_launches(self):
        """Kernel launches of the last RK stage (go_domain_stage_launches)."""
        v = ctypes.c_int()
        check(load().go_domain_stage_launches(self.handle, ctypes.byref(v)))
        return int(v.value)


class Batch:
    """Owner of one go_batch handle over a list of ``Domain`` objects."""

    def __init__(self, domains):
        lib = load()
        self.domains = list(domains)
        arr = (ctypes.c_void_p * len(self.domains))(*[d.handle.value for d in self.domains])
        h = ctypes.c_void_p()
        check(lib.go_batch_create(arr, len(self.domains), ctypes.byref(h)))
        self.handle = h
        self.n = len(self.domains)

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            load().go_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_member(self, m, dt, h0, h1, Hi, land_value=1e20, wind_t=0.0):
        """h0, h1: (eta, hu, hv) device tensors sharing a row stride; Hi a
        device tensor of corners."""
        p0 = h0[0].stride(0) * 4
        p1 = h1[0].stride(0) * 4
        check(load().go_batch_set_member(self.handle, int(m), float(dt), ptr(h0[0]), ptr(h0[1]), ptr(h0[2]), p0,
                                         ptr(h1[0]), ptr(h1[1]), ptr(h1[2]), p1, ptr(Hi), Hi.stride(0) * 4,
                                         float(land_value), float(wind_t)))

    def set_launch(self, shape=0, rows_per_block=0, blocks=0):
        check(load().go_batch_set_launch(self.handle, int(shape), int(rows_per_block), int(blocks)))
        self.launch = (int(shape), int(rows_per_block), int(blocks))

    def set_arith(self, mode):
        check(load().go_batch_set_arith(self.handle, int(mode)))

    def set_dt(self, dts, stream=None):
        a = np.ascontiguousarray(np.asarray(dts, dtype=np.float32).reshape(-1))
        assert a.size == self.n
        check(load().go_batch_set_dt(self.handle, stream_handle(stream),
                                     a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def tiles(self):
        n = ctypes.c_int()
        check(load().go_batch_tiles(self.handle, ctypes.byref(n)))
        return n.value

    def status(self, clear=False):
        """Per-member status words (GO_STATUS_* bits), member order."""
        out = (ctypes.c_uint32 * self.n)()
        check(load().go_batch_status(self.handle, ctypes.cast(out, ctypes.c_void_p), int(bool(clear))))
        return [int(v) for v in out]

    def step(self, n_steps, stream=None):
        check(load().go_batch_step(self.handle, stream_handle(stream), int(n_steps)))

    def capture(self, n_steps, stream):
        check(load().go_batch_graph_capture(self.handle, stream_handle(stream), int(n_steps)))

    def replay(self, stream):
        n = ctypes.c_int()
        check(load().go_batch_graph_launch(self.handle, stream_handle(stream), ctypes.byref(n)))
        return n.value

    def run_events(self, stream, first_event, n_events, interval, dt, courant, key0, std, corr_cells, scratch, t):
        """go_batch_run_events; t: the members' model times (float64, member
        order).  Returns (t after, steps per member, common dt after)."""
        tt = np.ascontiguousarray(np.asarray(t, dtype=np.float64).reshape(-1))
        assert tt.size == self.n
        steps = ctypes.c_longlong()
        dt_out = ctypes.c_float()
        check(load().go_batch_run_events(self.handle, stream_handle(stream), int(first_event) & 0xFFFFFFFF,
                                         int(n_events), float(interval), float(np.float32(dt)), float(courant),
                                         int(key0) & 0xFFFFFFFF, float(std), float(corr_cells), ptr(scratch),
                                         int(scratch.numel()), tt.ctypes.data_as(ctypes.c_void_p),
                                         ctypes.byref(steps), ctypes.byref(dt_out)))
        return tt, int(steps.value), np.float32(dt_out.value)
