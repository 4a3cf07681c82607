"""flowcontrast_b200: B200-native fractional-step lattice Boltzmann pipe solver.

Python mirror of the C ABI in include/fslbm.h (libfslbm.so, built in place by
`flowcontrast_b200.build.build()`). The compute path is the native library; importing this
package without it raises, and no operation falls back to Python or the CPU.

Axes follow the reference (PipeDemoStandalone/FSLBM.cu): x, y span the cross-section, z is
streamwise; numpy field arrays are shaped (lz, ly, lx). The stored velocity is the negated
physical one, as in the reference.
"""
import ctypes
import os

import numpy as np

__all__ = ["Context", "Solve", "Batch", "Server", "Domain", "Params", "FslbmError", "lib",
           "F64", "F32", "F16", "pipe_m_mask", "read_pipe_txt", "write_pipe_txt",
           "read_param_txt", "write_param_txt", "ref_mask_to_core", "init_poiseuille",
           "LIB_PATH"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfslbm.so")

F64, F32, F16 = 0, 1, 2
_NP = {F64: np.float64, F32: np.float32}


class FslbmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"fslbm error {code}: {msg}")
        self.code = code


class Domain(ctypes.Structure):
    _fields_ = [("lx", ctypes.c_int), ("ly", ctypes.c_int), ("lz", ctypes.c_int),
                ("mask", ctypes.c_void_p), ("radius", ctypes.c_double),
                ("cx", ctypes.c_double), ("cy", ctypes.c_double),
                ("buffer_depth", ctypes.c_int), ("mask_planes", ctypes.c_int),
                ("periodic_xy", ctypes.c_int)]


class Params(ctypes.Structure):
    _fields_ = [("tblend", ctypes.c_double), ("pin", ctypes.c_double),
                ("nu", ctypes.c_double), ("d1", ctypes.c_int), ("delta", ctypes.c_int),
                ("blend", ctypes.c_double), ("monitor_every", ctypes.c_int),
                ("force", ctypes.c_double * 3), ("fd_order", ctypes.c_int)]

    @classmethod
    def make(cls, tblend=1.0, pin=0.003, nu=0.004006, d1=2, delta=1, blend=0.0,
             monitor_every=50, force=(0.0, 0.0, 0.0), fd_order=0):
        """Defaults are pipe.m's param.txt (pipe.m:68) and the reference's 50-step monitor;
        fd_order 0 is the reference's active 4<->2 corrector blend."""
        return cls(tblend, pin, nu, d1, delta, blend, monitor_every, (ctypes.c_double * 3)(*force),
                   int(fd_order))

    def as_dict(self):
        return dict(tblend=self.tblend, pin=self.pin, nu=self.nu, d1=self.d1, delta=self.delta,
                    blend=self.blend, monitor_every=self.monitor_every, force=tuple(self.force),
                    fd_order=self.fd_order)


class Monitor(ctypes.Structure):
    _fields_ = [("step", ctypes.c_int64), ("q1", ctypes.c_double), ("q2", ctypes.c_double),
                ("p1", ctypes.c_double), ("p2", ctypes.c_double), ("f", ctypes.c_double),
                ("sample", ctypes.c_double), ("re", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Info(ctypes.Structure):
    _fields_ = [("cells", ctypes.c_int64), ("fluid_cells", ctypes.c_int64),
                ("bytes_device", ctypes.c_int64), ("steps", ctypes.c_int64),
                ("lx_pitch", ctypes.c_int), ("dtype", ctypes.c_int),
                ("last_step_ms", ctypes.c_double), ("kernel_launches", ctypes.c_int64)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_int64), ("max_resident", ctypes.c_int),
                ("quantum", ctypes.c_int), ("policy", ctypes.c_int),
                ("round_cells", ctypes.c_int64)]


SERVE_ALL, SERVE_LEAST_WORK = 0, 1


class InitSpec(ctypes.Structure):
    _fields_ = [("umax", ctypes.c_double), ("noise", ctypes.c_double), ("modes", ctypes.c_int),
                ("mode_amp", ctypes.c_double), ("seed", ctypes.c_uint64)]


class Request(ctypes.Structure):
    _fields_ = [("domain", Domain), ("params", Params), ("dtype", ctypes.c_int),
                ("nsteps", ctypes.c_int64), ("init", ctypes.c_void_p * 4),
                ("init_spec", InitSpec), ("out", ctypes.c_void_p * 4)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("error", ctypes.c_int),
                ("steps_done", ctypes.c_int64), ("t_submit", ctypes.c_double),
                ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double),
                ("bytes_device", ctypes.c_int64), ("cells", ctypes.c_int64),
                ("last", Monitor)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "last"}
        d["last"] = self.last.as_dict()
        return d


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64),
                ("failed", ctypes.c_int64), ("queued", ctypes.c_int64),
                ("resident", ctypes.c_int64), ("bytes_resident", ctypes.c_int64),
                ("bytes_peak", ctypes.c_int64), ("rounds", ctypes.c_int64),
                ("cell_steps", ctypes.c_double), ("busy_seconds", ctypes.c_double),
                ("t_admit", ctypes.c_double), ("t_regroup", ctypes.c_double),
                ("t_launch", ctypes.c_double), ("t_wait", ctypes.c_double),
                ("t_retire", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3

_lib = None
_vp = ctypes.c_void_p
_i = ctypes.c_int


def lib():
    """The loaded native library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run flowcontrast_b200.build.build() "
                              "(the solver has no non-native path)")
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "fslbm_version": ([], ctypes.c_char_p),
            "fslbm_last_error": ([ctypes.c_char_p, ctypes.c_size_t], _i),
            "fslbm_ctx_create": ([_i, ctypes.POINTER(_vp)], _i),
            "fslbm_ctx_destroy": ([_vp], _i),
            "fslbm_selftest_waits": ([_vp, ctypes.c_double, ctypes.POINTER(ctypes.c_uint)], _i),
            "fslbm_solve_create": ([_vp, ctypes.POINTER(Domain), ctypes.POINTER(Params), _i,
                                    ctypes.POINTER(_vp)], _i),
            "fslbm_solve_destroy": ([_vp], _i),
            "fslbm_solve_set_params": ([_vp, ctypes.POINTER(Params)], _i),
            "fslbm_solve_set_fields": ([_vp, _i, _vp, _vp, _vp, _vp], _i),
            "fslbm_solve_get_fields": ([_vp, _i, _vp, _vp, _vp, _vp], _i),
            "fslbm_solve_step": ([_vp, ctypes.c_int64], _i),
            "fslbm_solve_sync": ([_vp], _i),
            "fslbm_solve_monitor": ([_vp, ctypes.POINTER(Monitor)], _i),
            "fslbm_solve_monitor_log": ([_vp, ctypes.POINTER(Monitor), _i, ctypes.POINTER(_i)], _i),
            "fslbm_solve_check": ([_vp, ctypes.POINTER(ctypes.c_double)], _i),
            "fslbm_solve_info": ([_vp, ctypes.POINTER(Info)], _i),
            "fslbm_solve_set_timing": ([_vp, _i], _i),
            "fslbm_solve_kernel_time": ([_vp, ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_int64)], _i),
            "fslbm_solve_device_fields": ([_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                                           ctypes.POINTER(_vp), ctypes.POINTER(_vp)], _i),
            "fslbm_solve_get_fields_ref": ([_vp, _vp, _vp, _vp, _vp], _i),
            "fslbm_solve_set_fields_ref": ([_vp, _vp, _vp, _vp, _vp], _i),
            "fslbm_solve_get_plane": ([_vp, _i, _i, _vp], _i),
            "fslbm_stats_sample": ([_vp], _i),
            "fslbm_stats_get": ([_vp, _vp, ctypes.POINTER(_i), ctypes.POINTER(_i)], _i),
            "fslbm_stats_set": ([_vp, _vp, _i, _i], _i),
            "fslbm_profile_sample": ([_vp], _i),
            "fslbm_profile_get": ([_vp, _vp, ctypes.POINTER(ctypes.c_int64)], _i),
            "fslbm_profile_reset": ([_vp], _i),
            "fslbm_batch_create": ([_vp, ctypes.POINTER(_vp), _i, ctypes.POINTER(_vp)], _i),
            "fslbm_batch_destroy": ([_vp], _i),
            "fslbm_batch_step": ([_vp, ctypes.c_int64, _i], _i),
            "fslbm_batch_sync": ([_vp], _i),
            "fslbm_batch_elapsed": ([_vp, ctypes.POINTER(ctypes.c_double)], _i),
            "fslbm_batch_set_stop": ([_vp, _i, ctypes.c_int64], _i),
            "fslbm_batch_set_tiling": ([_vp, _i, _i, _i], _i),
            "fslbm_batch_load_tiling": ([_vp, ctypes.c_char_p], _i),
            "fslbm_batch_autotune": ([_vp, _i, ctypes.c_char_p], _i),
            "fslbm_solve_init_poiseuille": ([_vp, ctypes.c_double, ctypes.c_double, _i,
                                             ctypes.c_double, ctypes.c_uint64], _i),
            "fslbm_solve_footprint": ([ctypes.POINTER(Domain), _i, ctypes.POINTER(ctypes.c_int64)], _i),
            "fslbm_fd_coefficients": ([_i, ctypes.c_double, _i, _vp, ctypes.POINTER(_i)], _i),
            "fslbm_server_create": ([_i, ctypes.POINTER(ServerConfig), ctypes.POINTER(_vp)], _i),
            "fslbm_server_destroy": ([_vp], _i),
            "fslbm_server_submit": ([_vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_int64)], _i),
            "fslbm_server_poll": ([_vp, ctypes.c_int64, ctypes.POINTER(Result)], _i),
            "fslbm_server_wait": ([_vp, ctypes.c_int64, ctypes.c_double, ctypes.POINTER(Result)], _i),
            "fslbm_server_drain": ([_vp, ctypes.c_double], _i),
            "fslbm_server_release": ([_vp, ctypes.c_int64], _i),
            "fslbm_server_stats_get": ([_vp, ctypes.POINTER(ServerStats)], _i),
            "fslbm_read_pipe_txt": ([ctypes.c_char_p, _i, _i, _i, _vp], _i),
            "fslbm_write_pipe_txt": ([ctypes.c_char_p, _i, _i, _i, _vp], _i),
            "fslbm_read_param_txt": ([ctypes.c_char_p, ctypes.POINTER(Params)], _i),
            "fslbm_write_param_txt": ([ctypes.c_char_p, ctypes.POINTER(Params)], _i),
            "fslbm_pipe_m_mask": ([_i, _i, _i, _vp], _i),
            "fslbm_ref_mask_to_core": ([_vp, _i, _i, _i, _i, _vp], _i),
            "fslbm_ref_mask_to_core3d": ([_vp, _i, _i, _i, _i, _vp], _i),
            "fslbm_init_poiseuille": ([ctypes.POINTER(Domain), ctypes.c_double, ctypes.c_double,
                                       _i, ctypes.c_double, ctypes.c_uint64, _vp, _vp, _vp, _vp], _i),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        buf = ctypes.create_string_buffer(1024)
        lib().fslbm_last_error(buf, 1024)
        raise FslbmError(rc, buf.value.decode(errors="replace"))


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


# ---------------------------------------------------------------------------------------
# formats and generators
# ---------------------------------------------------------------------------------------
def pipe_m_mask(lx0=100, l0=300, d=10):
    """pipe.m geometry in the reference layout, shape (l0+2d, lx0+2d, lx0+2d)."""
    lx, lz = lx0 + 2 * d, l0 + 2 * d
    out = np.empty((lz, lx, lx), np.uint8)
    _check(lib().fslbm_pipe_m_mask(lx0, l0, d, _ptr(out)))
    return out


def read_pipe_txt(path, lx, ly, lz):
    out = np.empty((lz, ly, lx), np.uint8)
    _check(lib().fslbm_read_pipe_txt(os.fsencode(path), lx, ly, lz, _ptr(out)))
    return out


def write_pipe_txt(path, mask):
    mask = np.ascontiguousarray(mask, np.uint8)
    lz, ly, lx = mask.shape
    _check(lib().fslbm_write_pipe_txt(os.fsencode(path), lx, ly, lz, _ptr(mask)))


def read_param_txt(path, base=None):
    p = base if base is not None else Params.make()
    p = Params.from_buffer_copy(p)
    _check(lib().fslbm_read_param_txt(os.fsencode(path), ctypes.byref(p)))
    return p


def write_param_txt(path, prm):
    _check(lib().fslbm_write_param_txt(os.fsencode(path), ctypes.byref(prm)))


def ref_mask_to_core(mask3d, d2=10):
    mask3d = np.ascontiguousarray(mask3d, np.uint8)
    lz, ly, lx = mask3d.shape
    out = np.empty((ly, lx), np.uint8)
    _check(lib().fslbm_ref_mask_to_core(_ptr(mask3d), lx, ly, lz, d2, _ptr(out)))
    return out


def ref_mask_to_core3d(mask3d, d2=10):
    """Reference-layout mask (lz_ref, ly, lx) -> core masks (lz_ref - 2*d2, ly, lx), one
    cross-section per core plane (buffers must copy the wrapped core planes)."""
    mask3d = np.ascontiguousarray(mask3d, np.uint8)
    lz, ly, lx = mask3d.shape
    out = np.empty((lz - 2 * d2, ly, lx), np.uint8)
    _check(lib().fslbm_ref_mask_to_core3d(_ptr(mask3d), lx, ly, lz, d2, _ptr(out)))
    return out


def make_domain(lx, ly, lz, mask=None, radius=0.0, cx=None, cy=None, buffer_depth=10,
                periodic_xy=0):
    """Domain struct; keeps a reference to the mask array on the struct. mask: (ly, lx) for a
    cross-section extruded along z, or (lz, ly, lx) for one cross-section per plane.
    periodic_xy = G: cross-section periodic in x and y behind a G-wide ghost band."""
    d = Domain(lx, ly, lz, None, float(radius),
               float((lx - 1) / 2 if cx is None else cx), float((ly - 1) / 2 if cy is None else cy),
               int(buffer_depth), 0, int(periodic_xy))
    if mask is not None:
        m = np.ascontiguousarray(mask, np.uint8)
        if m.ndim == 3:
            m = m.reshape(lz, ly, lx)
            d.mask_planes = lz
        else:
            m = m.reshape(ly, lx)
        d.mask = m.ctypes.data
        d._mask_ref = m
    return d


def init_poiseuille(domain, umax, noise=1e-3, modes=0, mode_amp=0.0, seed=1):
    """Seeded initial fields (4, lz, ly, lx) float64: Poiseuille w plus noise and modes."""
    f = np.empty((4, domain.lz, domain.ly, domain.lx), np.float64)
    _check(lib().fslbm_init_poiseuille(ctypes.byref(domain), umax, noise, modes, mode_amp, seed,
                                       _ptr(f[0]), _ptr(f[1]), _ptr(f[2]), _ptr(f[3])))
    return f


# ---------------------------------------------------------------------------------------
# runtime
# ---------------------------------------------------------------------------------------
class Context:
    """One device and one stream (the reference's cudaSetDevice(0), FSLBM.cu:490)."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        _check(lib().fslbm_ctx_create(device, ctypes.byref(h)))
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            _check(lib().fslbm_ctx_destroy(self.handle))
            self.handle = None

    def selftest_waits(self, limit_ms=2.0):
        """Runs the device-side bounded waits against conditions nothing satisfies
        (fslbm_selftest_waits); returns (status code, bits of the waits that gave up)."""
        bits = ctypes.c_uint(0)
        rc = lib().fslbm_selftest_waits(self.handle, float(limit_ms), ctypes.byref(bits))
        return rc, bits.value

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Solve:
    """A periodic pipe solve (replaces the set-up and time loop of FSLBM.cu:489-905)."""

    def __init__(self, ctx, domain, params, dtype=F32):
        h = ctypes.c_void_p()
        self.domain, self.params, self.dtype, self.ctx = domain, params, dtype, ctx
        _check(lib().fslbm_solve_create(ctx.handle, ctypes.byref(domain), ctypes.byref(params),
                                        dtype, ctypes.byref(h)))
        self.handle = h
        self.shape = (domain.lz, domain.ly, domain.lx)

    def close(self):
        if self.handle:
            _check(lib().fslbm_solve_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params):
        _check(lib().fslbm_solve_set_params(self.handle, ctypes.byref(params)))
        self.params = params

    def set_fields(self, f):
        """f: (4, lz, ly, lx) float64 or float32 host array (or four arrays)."""
        arrs = [np.ascontiguousarray(a) for a in f]
        dt = F64 if arrs[0].dtype == np.float64 else F32
        arrs = [a.astype(_NP[dt], copy=False) for a in arrs]
        for a in arrs:
            if a.shape != self.shape:
                raise ValueError(f"field shape {a.shape} != {self.shape}")
        _check(lib().fslbm_solve_set_fields(self.handle, dt, *(_ptr(a) for a in arrs)))

    def init_poiseuille(self, umax, noise=1e-3, modes=0, mode_amp=0.0, seed=1):
        """The seeded start of init_poiseuille(), generated on the device."""
        _check(lib().fslbm_solve_init_poiseuille(self.handle, float(umax), float(noise), int(modes),
                                                 float(mode_amp), int(seed)))

    def set_fields_host(self, host_dtype, p, u, v, w):
        """Raw pointers (e.g. pinned host buffers) of the four fields."""
        _check(lib().fslbm_solve_set_fields(self.handle, host_dtype, p, u, v, w))

    def get_fields(self, dtype=np.float64):
        dt = F64 if np.dtype(dtype) == np.float64 else F32
        f = np.empty((4,) + self.shape, _NP[dt])
        _check(lib().fslbm_solve_get_fields(self.handle, dt, *(_ptr(f[k]) for k in range(4))))
        return f

    def get_fields_host(self, host_dtype, p, u, v, w):
        _check(lib().fslbm_solve_get_fields(self.handle, host_dtype, p, u, v, w))

    def step(self, n=1):
        _check(lib().fslbm_solve_step(self.handle, int(n)))

    def sync(self):
        _check(lib().fslbm_solve_sync(self.handle))

    def monitor(self):
        m = Monitor()
        _check(lib().fslbm_solve_monitor(self.handle, ctypes.byref(m)))
        return m.as_dict()

    def monitor_log(self, max_records=100000):
        buf = (Monitor * max_records)()
        n = ctypes.c_int()
        _check(lib().fslbm_solve_monitor_log(self.handle, buf, max_records, ctypes.byref(n)))
        return [buf[k].as_dict() for k in range(n.value)]

    def check(self):
        m = ctypes.c_double()
        _check(lib().fslbm_solve_check(self.handle, ctypes.byref(m)))
        return m.value

    def info(self):
        i = Info()
        _check(lib().fslbm_solve_info(self.handle, ctypes.byref(i)))
        return {k: getattr(i, k) for k, _ in Info._fields_}

    def set_timing(self, enable=True):
        _check(lib().fslbm_solve_set_timing(self.handle, int(bool(enable))))

    def kernel_time(self):
        """(summed step-kernel milliseconds, launches) since the previous call."""
        ms, n = ctypes.c_double(), ctypes.c_int64()
        _check(lib().fslbm_solve_kernel_time(self.handle, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def device_fields(self):
        ps = [ctypes.c_void_p() for _ in range(4)]
        _check(lib().fslbm_solve_device_fields(self.handle, *(ctypes.byref(p) for p in ps)))
        return [p.value for p in ps]

    # reference layout ------------------------------------------------------------------
    def get_fields_ref(self):
        d2 = self.domain.buffer_depth
        shp = (self.domain.lz + 2 * d2, self.domain.ly, self.domain.lx)
        f = np.empty((4,) + shp, np.float32)
        _check(lib().fslbm_solve_get_fields_ref(self.handle, *(_ptr(f[k]) for k in range(4))))
        return f

    def set_fields_ref(self, f):
        arrs = [np.ascontiguousarray(a, np.float32) for a in f]
        _check(lib().fslbm_solve_set_fields_ref(self.handle, *(_ptr(a) for a in arrs)))

    def get_plane(self, kind, comp):
        d2 = self.domain.buffer_depth
        if kind == 0:
            out = np.empty((self.domain.lz + 2 * d2) * self.domain.ly, np.float32)
        else:
            out = np.empty(self.domain.ly * self.domain.lx, np.float32)
        _check(lib().fslbm_solve_get_plane(self.handle, kind, comp, _ptr(out)))
        return out

    # statistics --------------------------------------------------------------------------
    def stats_sample(self):
        _check(lib().fslbm_stats_sample(self.handle))

    def stats_get(self):
        d2 = self.domain.buffer_depth
        n = self.domain.ly * (self.domain.lz + 2 * d2)
        out = np.empty((11, n), np.float64)
        c1, c2 = ctypes.c_int(), ctypes.c_int()
        _check(lib().fslbm_stats_get(self.handle, _ptr(out), ctypes.byref(c1), ctypes.byref(c2)))
        return out, c1.value, c2.value

    def stats_set(self, means, cnt, cnt2):
        m = np.ascontiguousarray(means, np.float64)
        _check(lib().fslbm_stats_set(self.handle, _ptr(m), int(cnt), int(cnt2)))

    def profile_sample(self):
        _check(lib().fslbm_profile_sample(self.handle))

    def profile_get(self):
        out = np.empty((10, self.domain.ly, self.domain.lx), np.float64)
        n = ctypes.c_int64()
        _check(lib().fslbm_profile_get(self.handle, _ptr(out), ctypes.byref(n)))
        return out, n.value

    def profile_reset(self):
        _check(lib().fslbm_profile_reset(self.handle))


class Batch:
    """Many solves of one context advanced together."""

    def __init__(self, ctx, solves):
        arr = (ctypes.c_void_p * len(solves))(*[s.handle.value for s in solves])
        h = ctypes.c_void_p()
        _check(lib().fslbm_batch_create(ctx.handle, arr, len(solves), ctypes.byref(h)))
        self.handle, self.solves = h, list(solves)

    def step(self, n, use_graph=True):
        _check(lib().fslbm_batch_step(self.handle, int(n), int(bool(use_graph))))

    def sync(self):
        _check(lib().fslbm_batch_sync(self.handle))

    def set_stop(self, member, stop_step):
        """Member `member` stops stepping once its step count reaches stop_step (-1: never)."""
        _check(lib().fslbm_batch_set_stop(self.handle, int(member), int(stop_step)))

    def set_tiling(self, member, chunk, warp_shape=1):
        """warp_shape: 0 = 32 x 2 cells, 1 = 16 x 4, 2 = 8 x 8."""
        _check(lib().fslbm_batch_set_tiling(self.handle, int(member), int(chunk), int(warp_shape)))

    def load_tiling(self, path):
        _check(lib().fslbm_batch_load_tiling(self.handle, os.fsencode(path)))

    def autotune(self, trial_steps=20, path=None):
        """Per-size-class tiling timed on this batch (state restored afterwards); with `path`
        the table is also written there as JSON and returned as a dict."""
        _check(lib().fslbm_batch_autotune(self.handle, int(trial_steps),
                                          os.fsencode(path) if path else None))
        if path:
            import json
            with open(path) as f:
                return json.load(f)["classes"]
        return None

    def elapsed_ms(self):
        ms = ctypes.c_double()
        _check(lib().fslbm_batch_elapsed(self.handle, ctypes.byref(ms)))
        return ms.value

    def close(self):
        if self.handle:
            _check(lib().fslbm_batch_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Served solves with continuous batching (fslbm_server_*): its own context and worker
    thread on `device`. submit() returns a request id; results come back in FP32 arrays."""

    def __init__(self, device=0, hbm_budget=0, max_resident=0, quantum=0, policy=SERVE_ALL,
                 round_cells=0):
        """policy SERVE_ALL advances every resident request each round; SERVE_LEAST_WORK the
        ones with the least work left, up to round_cells box cells per round."""
        cfg = ServerConfig(int(hbm_budget), int(max_resident), int(quantum), int(policy),
                           int(round_cells))
        h = ctypes.c_void_p()
        _check(lib().fslbm_server_create(int(device), ctypes.byref(cfg), ctypes.byref(h)))
        self.handle = h
        self._out = {}

    def submit(self, domain, params, dtype, nsteps, init=None, init_spec=None, want_fields=True):
        """init: (4, lz, ly, lx) host fields (copied), or None with init_spec = dict(umax,
        noise, modes, mode_amp, seed) for the device-generated start."""
        r = Request()
        r.domain = domain
        r.params = params
        r.dtype = int(dtype)
        r.nsteps = int(nsteps)
        keep = []
        if init is not None:
            a = np.ascontiguousarray(init, np.float32)
            keep.append(a)
            for k in range(4):
                r.init[k] = a[k].ctypes.data
        else:
            q = dict(umax=0.1, noise=1e-3, modes=0, mode_amp=0.0, seed=1)
            q.update(init_spec or {})
            r.init_spec = InitSpec(q["umax"], q["noise"], int(q["modes"]), q["mode_amp"],
                                   int(q["seed"]))
        out = None
        if want_fields:
            out = np.empty((4, domain.lz, domain.ly, domain.lx), np.float32)
            for k in range(4):
                r.out[k] = out[k].ctypes.data
        rid = ctypes.c_int64()
        _check(lib().fslbm_server_submit(self.handle, ctypes.byref(r), ctypes.byref(rid)))
        self._out[rid.value] = out
        return rid.value

    def poll(self, rid):
        res = Result()
        _check(lib().fslbm_server_poll(self.handle, int(rid), ctypes.byref(res)))
        return res.as_dict()

    def wait(self, rid, timeout=600.0):
        res = Result()
        _check(lib().fslbm_server_wait(self.handle, int(rid), float(timeout), ctypes.byref(res)))
        return res.as_dict()

    def fields(self, rid):
        """Final fields (4, lz, ly, lx) FP32 of a finished request submitted with want_fields."""
        return self._out.get(rid)

    def drain(self, timeout=3600.0):
        _check(lib().fslbm_server_drain(self.handle, float(timeout)))

    def release(self, rid):
        _check(lib().fslbm_server_release(self.handle, int(rid)))
        return self._out.pop(rid, None)

    def stats(self):
        st = ServerStats()
        _check(lib().fslbm_server_stats_get(self.handle, ctypes.byref(st)))
        return st.as_dict()

    def close(self):
        if self.handle:
            _check(lib().fslbm_server_destroy(self.handle))
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def fd_coefficients(order, blend=0.0, dtype=F64):
    """Corrector coefficients c0..cK of `order` as a solve of `dtype` uses them."""
    c = np.zeros(9)
    k = ctypes.c_int()
    _check(lib().fslbm_fd_coefficients(int(order), float(blend), int(dtype), _ptr(c), ctypes.byref(k)))
    return c[:k.value + 1]
