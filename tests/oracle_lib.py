"""ctypes binding of the test-only oracle (oracle/liboracle.so) for the test-suite.

The oracle is the CPU restatement of the reference method; it is a checker and is never
called by the product.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "liboracle.so")

_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.check_call(["make", "-s", "-C", ORACLE_DIR, "all"])
        L = ctypes.CDLL(LIB_PATH)
        i, l, d = ctypes.c_int, ctypes.c_long, ctypes.c_double
        L.oracle_check_ref_mask.argtypes = [_u8p, i, i, i, i]
        L.oracle_step_ref_f64.argtypes = [_u8p, i, i, i, i, _f64p, _f64p, _f64p, i]
        L.oracle_step_ref_f32.argtypes = [_u8p, i, i, i, i, _f64p, _f32p, _f32p, i]
        L.oracle_monitor_ref_f64.argtypes = [_u8p, i, i, i, i, d, d, _f64p, _f64p]
        L.oracle_monitor_ref_f32.argtypes = [_u8p, i, i, i, i, d, d, _f32p, _f64p]
        L.oracle_run_core_f64.argtypes = [_u8p, i, i, i, _f64p, i, d, l, _f64p, ctypes.c_void_p, i]
        L.oracle_run_core_f32.argtypes = [_u8p, i, i, i, _f64p, i, d, l, _f32p, ctypes.c_void_p, i]
        L.oracle_run_core3d_f64.argtypes = [_u8p, i, i, i, _f64p, i, d, l, _f64p, ctypes.c_void_p, i]
        L.oracle_run_core3d_f32.argtypes = [_u8p, i, i, i, _f64p, i, d, l, _f32p, ctypes.c_void_p, i]
        L.oracle_run_core_periodic_f64.argtypes = [_u8p, i, i, i, i, _f64p, i, d, l, _f64p,
                                                   ctypes.c_void_p, i]
        L.oracle_run_core_periodic_f32.argtypes = [_u8p, i, i, i, i, _f64p, i, d, l, _f32p,
                                                   ctypes.c_void_p, i]
        L.oracle_stats_accumulate.argtypes = [l, _f64p, _f64p, _f64p, _f64p, i, _f64p]
        L.oracle_stats_accumulate.restype = None
        L.oracle_pipe_m_mask.argtypes = [i, i, i, _u8p]
        L.oracle_max_threads.argtypes = []
        L.oracle_fd_coefficients.argtypes = [i, d, _f64p]
        L.oracle_init_poiseuille.argtypes = [i, i, i, d, d, d, d, d, i, d, ctypes.c_uint64, _f64p]
        _lib = L
    return _lib


def threads():
    return int(lib().oracle_max_threads())


def pipe_m_mask(lx0=100, l0=300, d=10):
    """pipe.m geometry (reference layout), shape (lz, ly, lx)."""
    lx, lz = lx0 + 2 * d, l0 + 2 * d
    out = np.zeros(lx * lx * lz, np.uint8)
    lib().oracle_pipe_m_mask(lx0, l0, d, out)
    return out.reshape(lz, lx, lx)


def step_ref(io, fields, prm, dtype=np.float64, nthreads=0):
    """One reference-layout step. io (lz,ly,lx) uint8; fields (4,lz,ly,lx); prm = dict."""
    lz, ly, lx = io.shape
    d2 = prm.get("d2", 10)
    p = np.array([prm["tblend"], prm["pin"], prm["nu"], prm["d1"], prm["blend"],
                  prm.get("gauge", 0.0), *prm.get("force", (0.0, 0.0, 0.0)),
                  prm.get("fd_order", 0)], np.float64)
    src = np.ascontiguousarray(fields, dtype=dtype)
    out = np.empty_like(src)
    fn = lib().oracle_step_ref_f64 if dtype == np.float64 else lib().oracle_step_ref_f32
    rc = fn(np.ascontiguousarray(io), lx, ly, lz, d2, p, src.ravel(), out.ravel(),
            nthreads or threads())
    if rc:
        raise ValueError(f"oracle_step_ref rejected the case: code {rc}")
    return out


def monitor_ref(io, fields, nu, radius, d2=10):
    lz, ly, lx = io.shape
    out = np.zeros(7)
    if fields.dtype == np.float64:
        lib().oracle_monitor_ref_f64(io, lx, ly, lz, d2, nu, radius, np.ascontiguousarray(fields).ravel(), out)
    else:
        lib().oracle_monitor_ref_f32(io, lx, ly, lz, d2, nu, radius, np.ascontiguousarray(fields).ravel(), out)
    return out


def run_core(mask2d, L, fields, prm, nsteps, monitor_every=50, radius=0.0, dtype=np.float64,
             nthreads=0):
    """Periodic-core run. mask2d (ly,lx) 0/125, or (L,ly,lx) for a mask per core plane;
    fields (4,L,ly,lx). Returns (fields, monitor)."""
    three_d = mask2d.ndim == 3
    ly, lx = mask2d.shape[-2:]
    p = np.array([prm["tblend"], prm["pin"], prm["nu"], prm["d1"], prm["blend"],
                  *prm.get("force", (0.0, 0.0, 0.0)), prm.get("fd_order", 0)], np.float64)
    f = np.array(fields, dtype=dtype, order="C", copy=True)
    nmon = nsteps // monitor_every if monitor_every > 0 else 0
    mon = np.zeros((max(nmon, 1), 7))
    if three_d:
        fn = lib().oracle_run_core3d_f64 if dtype == np.float64 else lib().oracle_run_core3d_f32
    else:
        fn = lib().oracle_run_core_f64 if dtype == np.float64 else lib().oracle_run_core_f32
    rc = fn(np.ascontiguousarray(mask2d, np.uint8).ravel(), lx, ly, L, p, monitor_every,
            float(radius), nsteps, f.ravel(), mon.ctypes.data, nthreads or threads())
    if rc < 0:
        raise ValueError(f"oracle_run_core rejected the case: code {rc}")
    return f, mon[:nmon]


def stats_accumulate(acc, p, u, v, w, cnt):
    n = p.size
    lib().oracle_stats_accumulate(n, *(np.ascontiguousarray(a, np.float64).ravel() for a in (p, u, v, w)),
                                  int(cnt), acc.ravel())


def init_poiseuille(lx, ly, L, radius, cx, cy, umax, noise=0.0, modes=0, mode_amp=0.0, seed=0):
    """Seeded start of the benchmark workloads on a circular pipe, (4, L, ly, lx) float64; the
    same fields as the library's fslbm_init_poiseuille, without loading the library."""
    out = np.zeros(4 * L * ly * lx)
    rc = lib().oracle_init_poiseuille(lx, ly, L, float(radius), float(cx), float(cy), float(umax),
                                      float(noise), int(modes), float(mode_amp), int(seed), out)
    if rc:
        raise ValueError(f"oracle_init_poiseuille rejected the case: code {rc}")
    return out.reshape(4, L, ly, lx)


def fd_coefficients(order, blend=0.0):
    """Corrector coefficients c0..cK of an order (the reference's sets), FP64 forms."""
    c = np.zeros(9)
    k = lib().oracle_fd_coefficients(int(order), float(blend), c)
    if k == 0:
        raise ValueError(f"no corrector of order {order}")
    return c[:k + 1]


def periodic_mask(nx, ny, G, inner=None):
    """Cross-section periodic in x and y: interior nx x ny (0 fluid / 125 wall, all fluid by
    default) inside a G-wide ghost band (2 where the periodic image is fluid)."""
    lx, ly = nx + 2 * G, ny + 2 * G
    inner = np.zeros((ny, nx), np.uint8) if inner is None else np.asarray(inner, np.uint8)
    m = np.empty((ly, lx), np.uint8)
    for y in range(ly):
        for x in range(lx):
            v = inner[(y - G) % ny, (x - G) % nx]
            inside = G <= x < lx - G and G <= y < ly - G
            m[y, x] = v if inside else (125 if v == 125 else 2)
    return m


def run_periodic(mask2d, L, G, fields, prm, nsteps, monitor_every=0, radius=0.0,
                 dtype=np.float64, nthreads=0):
    """Periodic-core run with a cross-section periodic in x and y (ghost band G)."""
    ly, lx = mask2d.shape
    p = np.array([prm["tblend"], prm["pin"], prm["nu"], prm["d1"], prm["blend"],
                  *prm.get("force", (0.0, 0.0, 0.0)), prm.get("fd_order", 0)], np.float64)
    f = np.array(fields, dtype=dtype, order="C", copy=True)
    nmon = nsteps // monitor_every if monitor_every > 0 else 0
    mon = np.zeros((max(nmon, 1), 7))
    fn = lib().oracle_run_core_periodic_f64 if dtype == np.float64 else lib().oracle_run_core_periodic_f32
    rc = fn(np.ascontiguousarray(mask2d, np.uint8).ravel(), lx, ly, L, G, p, monitor_every,
            float(radius), nsteps, f.ravel(), mon.ctypes.data, nthreads or threads())
    if rc < 0:
        raise ValueError(f"oracle_run_core_periodic rejected the case: code {rc}")
    return f, mon[:nmon]
