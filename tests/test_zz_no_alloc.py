"""The allocation-free step entry point (fslbm_step_f32_noalloc) against the regular one.

Callers that cannot let a library allocate device memory (their own memory pool, or a loop in
which a device allocation is not allowed) step a state they own through this entry point. It
must give the same fields as fslbm_solve_step on the same input, over two calls in a row that
reuse its preallocated work tables. Tolerance: 1e-6 relative L2 over all cells (both paths run
the same FP32 kernel; the only difference allowed is the order of work inside it).

This file is collected last so that a run stopping at the first failure has run every other
test before it.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _circle(lx, ly, R, c):
    y, x = np.mgrid[0:ly, 0:lx]
    return np.where((x - c) ** 2 + (y - c) ** 2 <= R * R, 0, 125).astype(np.uint8)


def test_noalloc_step_matches_solve_step(built):
    import torch

    fb = built
    L = fb.lib()
    fn = L.fslbm_step_f32_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int, ctypes.POINTER(fb.Params), ctypes.c_double,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int

    lx = ly = 32
    lz, R = 40, 14.0
    m2 = _circle(lx, ly, R, 15.5)
    prm = fb.Params.make(tblend=0.8, pin=0.002, nu=0.02, d1=2, delta=1, blend=1.0,
                         monitor_every=0, force=(0.0, 0.0, -1e-5))
    ctx = fb.Context(0)
    try:
        dom = fb.make_domain(lx, ly, lz, mask=m2, radius=R, buffer_depth=10)
        s = fb.Solve(ctx, dom, prm, fb.F32)
        rng = np.random.default_rng(3)
        f = np.zeros((4, lz, ly, lx))
        f[0] = 1e-3 * rng.uniform(-1, 1, f[0].shape)
        f[1:] = 0.02 * rng.uniform(-1, 1, f[1:].shape)
        f[3] -= 0.05
        s.set_fields(f)
        s.sync()
        pitch = s.info()["lx_pitch"]
        n = 4 * lz * ly * pitch

        mask_pad = np.full((ly, pitch), 125, np.uint8)
        mask_pad[:, :lx] = m2
        dmask = torch.from_numpy(mask_pad).cuda()
        bufs = [torch.zeros(n, dtype=torch.float32, device="cuda") for _ in range(2)]
        torch.cuda.synchronize()

        src = s.device_fields()[0]
        for k in range(2):
            rc = fn(src, bufs[k].data_ptr(), dmask.data_ptr(), lx, ly, lz, pitch,
                    ctypes.byref(prm), 0.0, None)
            if rc != 0:
                buf = ctypes.create_string_buffer(512)
                L.fslbm_last_error(buf, 512)
                pytest.fail(f"fslbm_step_f32_noalloc failed: {rc} {buf.value.decode()}")
            s.step(1)
            s.sync()
            want = s.get_fields(np.float32).astype(np.float64)
            got = bufs[k].cpu().numpy().reshape(4, lz, ly, pitch)[:, :, :, :lx].astype(np.float64)
            err = np.linalg.norm(got - want) / np.linalg.norm(want)
            assert err <= 1e-6, (k, err)
            src = bufs[k].data_ptr()
        s.close()
    finally:
        ctx.close()
