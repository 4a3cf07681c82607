"""Geometry varying along the pipe on the GPU (one cross-section per plane; one-column kernel
with per-cell wall sums). Against the oracle over 60 steps with the seam pressure jump and the
monitor gauge: FP64 1e-12, FP32 1e-5 relative L2 (p scaled as in the parity tests). The
monitor's l1 is the reference's buffer-cell count over 2*d2 planes, which for such geometry
depends on the buffer depth: the domains here use the oracle's padding depth max(1, K*d1)."""
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as O
from flowcontrast_b200 import workloads as wl
from test_gpu_parity import errors, run_gpu

pytestmark = pytest.mark.gpu


def rough_case(seed=5):
    n, L, R = 32, 28, 13.0
    m3 = wl.rough_pipe_mask(n, L, R, amplitude=1.5, seed=seed)
    rng = np.random.default_rng(seed)
    f = np.zeros((4, L, n, n))
    f[0] = 1e-3 * rng.uniform(-1, 1, f[0].shape)
    f[1:] = 0.02 * rng.uniform(-1, 1, f[1:].shape)
    f[3] -= 0.08
    f *= (m3 == 0)
    prm = dict(tblend=0.8, pin=0.002, nu=0.03, d1=2, blend=1.0, force=(0.0, 0.0, -1e-5))
    return m3, n, L, R, f, prm


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_rough_pipe_parity(built, ctx, dt):
    fb = built
    m3, n, L, R, f, prm = rough_case()
    dom = fb.make_domain(n, n, L, mask=m3, radius=R, buffer_depth=4)
    ref, mon = O.run_core(m3, L, f, prm, 60, monitor_every=25, radius=R)
    got, log = run_gpu(fb, ctx, dom, prm, fb.F64 if dt == "f64" else fb.F32, f, 60, monitor_every=25)
    nw = np.all(m3 == 0, axis=0)                  # compare on columns fluid in every plane
    _, eu, eps = errors(got, ref, np.where(nw, 0, 125))
    tol = 1e-12 if dt == "f64" else 1e-5
    assert eu <= tol and eps <= tol, (eu, eps)
    assert np.all(got[:, m3 != 0] == 0)           # walls stay zero, plane by plane
    assert [r["step"] for r in log] == [25, 50]
    for r, m in zip(log, mon):
        assert abs(r["q1"] - m[0]) <= (1e-10 if dt == "f64" else 1e-5) * abs(m[0])


def test_extruded_mask_given_per_plane(built, ctx):
    fb = built
    m3, n, L, R, f, prm = rough_case()
    m3[:] = m3[0]
    f *= (m3 == 0)
    a, _ = run_gpu(fb, ctx, fb.make_domain(n, n, L, mask=m3[0], radius=R), prm, fb.F64, f, 30)
    b, _ = run_gpu(fb, ctx, fb.make_domain(n, n, L, mask=m3, radius=R), prm, fb.F64, f, 30)
    assert np.allclose(a, b, rtol=0, atol=1e-13)


def test_cli_rough_pipe(built, ctx, tmp_path):
    """pipe.txt whose planes differ runs through fslbm_pipe and matches the library."""
    fb = built
    from test_cli import CLI
    core = wl.rough_pipe_mask(40, 40, 17.0, amplitude=1.5, seed=7)
    d2 = 10
    ref = np.concatenate([core[-d2:], core, core[:d2]])
    for sl in (slice(0, d2), slice(-d2, None)):
        part = ref[sl]
        part[part == 0] = 1
    d = str(tmp_path)
    fb.write_pipe_txt(os.path.join(d, "pipe.txt"), ref)
    fb.write_param_txt(os.path.join(d, "param.txt"),
                       fb.Params.make(tblend=1.0, pin=0.003, nu=0.03, d1=2, delta=1, blend=0.0))
    r = subprocess.run([CLI, "--lx", "40", "--ly", "40", "--lz", "60", "--radius", "17",
                        "--steps", "100", "--backup", "100", "--dump", "100", "--quiet"],
                       cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    raw = [np.fromfile(os.path.join(d, k), np.float32).reshape(60, 40, 40)
           for k in ("p3Dii", "ux3Dii", "uy3Dii", "uz3Dii")]
    dom = fb.make_domain(40, 40, 40, mask=core, radius=17.0, buffer_depth=d2)
    prm = fb.read_param_txt(os.path.join(d, "param.txt"))
    prm.monitor_every = 50
    s = fb.Solve(ctx, dom, prm, fb.F32)
    f = np.zeros((4, 60, 40, 40), np.float32)
    z = np.arange(60, dtype=np.float32)
    f[0] = (np.float32(np.float32(0.003) * (np.float32(50) - z)) / np.float32(40))[:, None, None]
    s.set_fields_ref(f)
    s.step(100)
    s.sync()
    want = s.get_fields_ref()
    s.close()
    for k in range(4):
        assert np.array_equal(raw[k], want[k]), k
