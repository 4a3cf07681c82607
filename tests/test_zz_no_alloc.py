"""The allocation-free step entry point (fslbm_step_f32_noalloc) against the regular one.

Callers that cannot let a library allocate device memory (their own memory pool, or a loop in
which a device allocation is not allowed) step a state they own through this entry point. It
must give the same fields as fslbm_solve_step on the same input, over calls in a row that
reuse its preallocated work tables:
  - a 32 x 32 cross-section (one tile) and a 100 x 70 one (row pitch 104, several tiles in x
    and y, one column of tiles all wall, ly not a multiple of the tile height), with the
    solve's monitor every step and its gauge p2 handed to the next call: equal bit for bit
    (the step's results do not depend on which tiles or streamwise chunks a launch runs);
  - the 100 x 70 case against the FP64 oracle within 1e-5 relative (the FP32 parity bound);
  - a mask with fluid on the rim, or with a value other than 0 / 125, is refused with
    FSLBM_ERR_ARG and a later valid call steps correctly.
Argument checks that need no device (sizes beyond the 65 536-cell scratch, d1 != 2,
overlapping input and output) are tested on the CPU in test_abi.py.

This file is collected last so that a run stopping at the first failure has run every other
test before it.
"""
import ctypes

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu


def _circle(lx, ly, R, cx, cy):
    y, x = np.mgrid[0:ly, 0:lx]
    return np.where((x - cx) ** 2 + (y - cy) ** 2 <= R * R, 0, 125).astype(np.uint8)


def _fn(fb):
    L = fb.lib()
    fn = L.fslbm_step_f32_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int, ctypes.POINTER(fb.Params), ctypes.c_double,
                   ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _err(fb):
    buf = ctypes.create_string_buffer(512)
    fb.lib().fslbm_last_error(buf, 512)
    return buf.value.decode()


def _start(m2, lz, seed):
    ly, lx = m2.shape
    rng = np.random.default_rng(seed)
    f = np.zeros((4, lz, ly, lx))
    f[0] = 1e-3 * rng.uniform(-1, 1, f[0].shape)
    f[1:] = 0.02 * rng.uniform(-1, 1, f[1:].shape)
    f[3] -= 0.05
    return f * (m2 == 0)


CASES = {
    "one_tile": dict(lx=32, ly=32, lz=40, R=14.0, cx=15.5, cy=15.5),
    "multi_tile": dict(lx=100, ly=70, lz=36, R=30.0, cx=38.0, cy=34.5),
}


@pytest.mark.parametrize("name", list(CASES))
def test_noalloc_step_matches_solve_step(built, name):
    import torch

    fb = built
    fn = _fn(fb)
    c = CASES[name]
    lx, ly, lz = c["lx"], c["ly"], c["lz"]
    m2 = _circle(lx, ly, c["R"], c["cx"], c["cy"])
    prm = fb.Params.make(tblend=0.8, pin=0.002, nu=0.02, d1=2, delta=1, blend=1.0,
                         monitor_every=1, force=(0.0, 0.0, -1e-5))
    ctx = fb.Context(0)
    try:
        dom = fb.make_domain(lx, ly, lz, mask=m2, radius=c["R"], buffer_depth=10)
        s = fb.Solve(ctx, dom, prm, fb.F32)
        s.set_fields(_start(m2, lz, 3))
        s.sync()
        pitch = s.info()["lx_pitch"]
        n = 4 * lz * ly * pitch
        if name == "multi_tile":
            assert pitch == 104 and np.all(m2[:, 96:] == 125)    # tiles at x >= 96 are all wall

        mask_pad = np.full((ly, pitch), 125, np.uint8)
        mask_pad[:, :lx] = m2
        dmask = torch.from_numpy(mask_pad).cuda()
        bufs = [torch.zeros(n, dtype=torch.float32, device="cuda") for _ in range(3)]
        torch.cuda.synchronize()

        src, gauge = s.device_fields()[0], 0.0
        for k in range(3):
            rc = fn(src, bufs[k].data_ptr(), dmask.data_ptr(), lx, ly, lz, pitch,
                    ctypes.byref(prm), gauge, None)
            assert rc == 0, f"fslbm_step_f32_noalloc failed: {rc} {_err(fb)}"
            s.step(1)
            s.sync()
            want = s.get_fields(np.float32)
            got = bufs[k].cpu().numpy().reshape(4, lz, ly, pitch)
            assert np.array_equal(got[:, :, :, :lx], want), k
            assert not np.any(got[:, :, :, lx:]), k               # padding stays zero
            gauge = s.monitor()["p2"]                            # gauges the next step
            assert k == 0 or gauge != 0.0
            src = bufs[k].data_ptr()
        s.close()
    finally:
        ctx.close()


def test_noalloc_step_matches_oracle(built):
    import torch

    fb = built
    fn = _fn(fb)
    c = CASES["multi_tile"]
    lx, ly, lz = c["lx"], c["ly"], c["lz"]
    pitch = 104
    m2 = _circle(lx, ly, c["R"], c["cx"], c["cy"])
    prm = fb.Params.make(tblend=0.8, pin=0.002, nu=0.02, d1=2, delta=1, blend=1.0,
                         monitor_every=0, force=(0.0, 0.0, -1e-5))
    f0 = _start(m2, lz, 4)
    want, _ = O.run_core(m2, lz, f0, dict(tblend=0.8, pin=0.002, nu=0.02, d1=2, blend=1.0,
                                          force=(0.0, 0.0, -1e-5)), 2, monitor_every=0)
    host = np.zeros((4, lz, ly, pitch), np.float32)
    host[:, :, :, :lx] = f0
    mask_pad = np.full((ly, pitch), 125, np.uint8)
    mask_pad[:, :lx] = m2
    dmask = torch.from_numpy(mask_pad).cuda()
    a = torch.from_numpy(host.ravel()).cuda()
    b = torch.zeros_like(a)
    for src, dst in ((a, b), (b, a)):
        rc = fn(src.data_ptr(), dst.data_ptr(), dmask.data_ptr(), lx, ly, lz, pitch,
                ctypes.byref(prm), 0.0, None)
        assert rc == 0, _err(fb)
    got = a.cpu().numpy().reshape(4, lz, ly, pitch)[:, :, :, :lx].astype(np.float64)
    nw = m2 == 0
    eu = np.linalg.norm((got[1:] - want[1:])[:, :, nw]) / np.linalg.norm(want[1:][:, :, nw])
    scale = np.linalg.norm(np.abs(want[0][:, nw]) + 1.5 * (want[1:][:, :, nw] ** 2).sum(0))
    ep = np.linalg.norm((got[0] - want[0])[:, nw]) / scale
    assert eu <= 1e-5 and ep <= 1e-5, (eu, ep)


def test_noalloc_rejects_bad_masks(built):
    import torch

    fb = built
    fn = _fn(fb)
    lx = ly = 32
    lz = 12
    m2 = _circle(lx, ly, 14.0, 15.5, 15.5)
    prm = fb.Params.make(tblend=0.8, pin=0.0, nu=0.02, d1=2, blend=1.0, monitor_every=0)
    n = 4 * lz * ly * lx
    a = torch.zeros(n, dtype=torch.float32, device="cuda")
    b = torch.zeros(n, dtype=torch.float32, device="cuda")
    for bad in ("rim", "value"):
        m = m2.copy()
        if bad == "rim":
            m[0, 16] = 0                         # fluid on the cross-section rim
        else:
            m[16, 16] = 2                        # neither fluid nor wall
        dm = torch.from_numpy(m).cuda()
        rc = fn(a.data_ptr(), b.data_ptr(), dm.data_ptr(), lx, ly, lz, lx, ctypes.byref(prm), 0.0, None)
        assert rc == -1 and "mask" in _err(fb), (bad, rc)          # FSLBM_ERR_ARG
    # the shared work tables recover: a valid call steps a uniform rest state to itself
    host = np.zeros((4, lz, ly, lx), np.float32)
    host[0] = 1e-3 * (m2 == 0)
    a.copy_(torch.from_numpy(host.ravel()))
    dm = torch.from_numpy(m2).cuda()
    rc = fn(a.data_ptr(), b.data_ptr(), dm.data_ptr(), lx, ly, lz, lx, ctypes.byref(prm), 0.0, None)
    assert rc == 0, _err(fb)
    out = b.cpu().numpy().reshape(4, lz, ly, lx)
    assert np.allclose(out[0], host[0], rtol=0, atol=1e-8) and np.abs(out[1:]).max() < 1e-8
