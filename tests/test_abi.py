"""C-ABI boundary tests that need no GPU: the library loads, exports every declared entry
point, and its host-side formats and generators behave (pipe.txt, param.txt, pipe.m geometry,
reference-mask split, seeded initial fields)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(fslbm_[a-z0-9_]+)\s*\(", txt))
    return names


def test_every_declared_symbol_is_exported(built):
    names = _declared()
    assert len(names) > 30
    lib = ctypes.CDLL(built.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_buffer(built):
    assert built.lib().fslbm_version().startswith(b"fslbm")
    with pytest.raises(built.FslbmError) as e:
        built.read_pipe_txt("/nonexistent/pipe.txt", 4, 4, 4)
    assert e.value.code == -4 and "cannot open" in str(e.value)


def test_pipe_txt_round_trip_and_exact_count(built, tmp_path):
    m = built.pipe_m_mask(12, 16, 10)
    p = tmp_path / "pipe.txt"
    built.write_pipe_txt(str(p), m)
    lines = p.read_text().splitlines()
    assert len(lines) == m.size and lines[0] == "125"
    back = built.read_pipe_txt(str(p), 32, 32, 36)
    assert np.array_equal(back, m)
    # one value short, one value too many, a non-byte value: all rejected (FSLBM.cu:481-484
    # would write past its buffer or silently keep stale bytes)
    p.write_text("\n".join(lines[:-1]) + "\n")
    with pytest.raises(built.FslbmError):
        built.read_pipe_txt(str(p), 32, 32, 36)
    p.write_text("\n".join(lines + ["0"]) + "\n")
    with pytest.raises(built.FslbmError):
        built.read_pipe_txt(str(p), 32, 32, 36)
    p.write_text("\n".join(lines[:-1] + ["300"]) + "\n")
    with pytest.raises(built.FslbmError):
        built.read_pipe_txt(str(p), 32, 32, 36)


def test_param_txt_pipe_m_format(built, tmp_path):
    p = tmp_path / "param.txt"
    # pipe.m:68 output (the sixth value reuses the first format, %f)
    p.write_text("1.000000\n0.003000\n0.004006\n2\n1\n0.000000\n")
    prm = built.read_param_txt(str(p))
    assert prm.tblend == 1.0 and prm.d1 == 2 and prm.delta == 1 and prm.blend == 0.0
    # floats are read into FP32 like the reference's fscanf("%e", &float)
    assert prm.pin == float(np.float32(0.003)) and prm.nu == float(np.float32(0.004006))
    # a trailing save-path line is ignored (FSLBM.cu:508)
    p.write_text("0.5\n0.01\n0.02\n1\n2\n0.25\n/some/path/\n")
    prm = built.read_param_txt(str(p))
    assert (prm.tblend, prm.d1, prm.delta, prm.blend) == (0.5, 1, 2, 0.25)
    built.write_param_txt(str(p), prm)
    assert built.read_param_txt(str(p)).as_dict() == prm.as_dict()
    p.write_text("1.0\n0.003\n")
    with pytest.raises(built.FslbmError):
        built.read_param_txt(str(p))
    p.write_text("1.0\n0.003\nabc\n2\n1\n0\n")
    with pytest.raises(built.FslbmError):
        built.read_param_txt(str(p))


def test_ref_mask_to_core(built):
    m = built.pipe_m_mask(12, 16, 10)
    core = built.ref_mask_to_core(m, 10)
    assert np.array_equal(core, np.where(m[10] == 125, 125, 0))
    bad = m.copy(); bad[20, 16, 16] = 125          # one plane differs
    with pytest.raises(built.FslbmError):
        built.ref_mask_to_core(bad, 10)
    bad = m.copy(); bad[2, 16, 16] = 0             # fluid inside a buffer
    with pytest.raises(built.FslbmError):
        built.ref_mask_to_core(bad, 10)
    bad = m.copy(); bad[:, 0, 12] = np.where(bad[:, 0, 12] == 125, 0, bad[:, 0, 12])
    with pytest.raises(built.FslbmError):
        built.ref_mask_to_core(bad, 10)


def test_init_poiseuille_seeded(built):
    d = built.make_domain(32, 32, 16, radius=15.0, cx=15.5, cy=15.5)
    a = built.init_poiseuille(d, 0.1, noise=1e-3, modes=3, mode_amp=0.1, seed=7)
    b = built.init_poiseuille(d, 0.1, noise=1e-3, modes=3, mode_amp=0.1, seed=7)
    c = built.init_poiseuille(d, 0.1, noise=1e-3, modes=3, mode_amp=0.1, seed=8)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    y, x = np.mgrid[0:32, 0:32]
    wall = (x - 15.5) ** 2 + (y - 15.5) ** 2 > 15.0 ** 2
    assert (a[:, :, wall] == 0).all()
    # stored streamwise velocity is negative (physical flow towards +z); centre near -umax
    assert a[3, :, 15, 15].mean() < -0.09
    assert (a[0] == 0).all()


def test_ctx_create_without_gpu_reports_error(built):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(built.FslbmError) as e:
        built.Context(0)
    assert e.value.code == -2


def test_server_without_gpu_reports_error(built):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(built.FslbmError) as e:
        built.Server(0)
    assert e.value.code == -2


def test_server_refuses_unknown_policy_before_touching_a_device(built):
    with pytest.raises(built.FslbmError) as e:
        built.Server(0, policy=7)
    assert e.value.code == -1


def test_solve_footprint_counts_state_ping_pong(built):
    import ctypes
    fb = built
    dom = fb.make_domain(128, 128, 512, radius=63, cx=63.5, cy=63.5)
    out = {}
    for dt in (fb.F64, fb.F32, fb.F16):
        b = ctypes.c_int64()
        fb._check(fb.lib().fslbm_solve_footprint(ctypes.byref(dom), dt, ctypes.byref(b)))
        out[dt] = b.value
    state = 2 * 4 * 128 * 128 * 512
    for dt, es in ((fb.F64, 8), (fb.F32, 4), (fb.F16, 2)):
        assert state * es <= out[dt] <= state * es + 4 * 2 ** 20


def test_noalloc_argument_checks_need_no_device(built):
    """fslbm_step_f32_noalloc refuses, before touching a device: a cross-section beyond its
    65 536-cell scratch, d1 != 2, and an output that overlaps the input or the mask (the step
    reads its input while other blocks write the output, so it cannot run in place). The
    pointers are never dereferenced on these paths."""
    import ctypes
    fb = built
    fn = fb.lib().fslbm_step_f32_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int, ctypes.POINTER(fb.Params), ctypes.c_double,
                   ctypes.c_void_p]
    prm = fb.Params.make(d1=2, blend=1.0)
    lx, ly, lz, pitch = 32, 32, 40, 32
    nbytes = 4 * lz * ly * pitch * 4
    a, b, m = 1 << 32, (1 << 32) + 2 * nbytes, (1 << 32) + 4 * nbytes
    buf = ctypes.create_string_buffer(256)

    def call(*args, **kw):
        rc = fn(*args, ctypes.byref(kw.get("prm", prm)), 0.0, None)
        fb.lib().fslbm_last_error(buf, 256)
        return rc, buf.value.decode()

    rc, msg = call(a, b, m, 264, 256, lz, 264)           # 264 * 256 > 65536 cells
    assert rc == -1 and "65536" in msg
    rc, msg = call(a, b, m, lx, ly, lz, pitch, prm=fb.Params.make(d1=3))
    assert rc == -1 and "d1" in msg
    rc, msg = call(a, a, m, lx, ly, lz, pitch)           # in place
    assert rc == -1 and "overlaps" in msg
    rc, msg = call(a, a + nbytes // 2, m, lx, ly, lz, pitch)   # partly overlapping
    assert rc == -1 and "overlaps" in msg
    rc, msg = call(a, b, b + 64, lx, ly, lz, pitch)      # mask inside the output
    assert rc == -1 and "overlaps" in msg
