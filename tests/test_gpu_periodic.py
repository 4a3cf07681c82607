"""Cross-section periodic in x and y on the GPU: against the oracle (a periodic array of
cylinders with the seam jump, force and monitors; 40 steps, FP64 1e-12 / FP32 1e-5), and the
Taylor-Green vortex decay (effective viscosity within 1 % of nu on a 64^2 box)."""
import numpy as np
import pytest

import oracle_lib as O
from test_gpu_parity import errors, run_gpu

pytestmark = pytest.mark.gpu


def cylinders(n=32, G=4, L=16, seed=3):
    inner = np.zeros((n, n), np.uint8)
    y, x = np.mgrid[0:n, 0:n]
    inner[(x - 15.5) ** 2 + (y - 15.5) ** 2 <= 6.0 ** 2] = 125
    m = O.periodic_mask(n, n, G, inner)
    rng = np.random.default_rng(seed)
    f = np.zeros((4, L, n + 2 * G, n + 2 * G))
    f[:, :, G:-G, G:-G] = 0.01 * rng.uniform(-1, 1, (4, L, n, n)) * (inner == 0)
    f[3, :, G:-G, G:-G] -= 0.05 * (inner == 0)
    prm = dict(tblend=0.8, pin=0.002, nu=0.05, d1=2, blend=1.0, force=(0.0, 0.0, -1e-5))
    return inner, m, f, prm, n, G, L


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_periodic_cylinders_parity(built, ctx, dt):
    fb = built
    inner, m, f, prm, n, G, L = cylinders()
    full = np.zeros((n + 2 * G, n + 2 * G), np.uint8)
    full[G:-G, G:-G] = inner
    dom = fb.make_domain(n + 2 * G, n + 2 * G, L, mask=full, radius=10.0, periodic_xy=G,
                         buffer_depth=4)
    ref, mon = O.run_periodic(m, L, G, f, prm, 40, monitor_every=20, radius=10.0)
    got, log = run_gpu(fb, ctx, dom, prm, fb.F64 if dt == "f64" else fb.F32, f, 40, monitor_every=20)
    _, eu, eps = errors(got, ref, np.where(m == 0, 0, 125))
    tol = 1e-12 if dt == "f64" else 1e-5
    assert eu <= tol and eps <= tol, (eu, eps)
    assert np.allclose(got[:, :, :G, G:-G], got[:, :, -2 * G:-G, G:-G])   # ghosts are images
    for r, w in zip(log, mon):
        assert abs(r["q1"] - w[0]) <= (1e-10 if dt == "f64" else 1e-5) * abs(w[0])


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_taylor_green_on_gpu(built, ctx, dt):
    fb = built
    n, G, L, A, nu, steps = 64, 4, 8, 1e-4, 0.05, 40
    lx = n + 2 * G
    y, x = np.mgrid[0:lx, 0:lx]
    k = 2 * np.pi / n
    f = np.zeros((4, L, lx, lx))
    f[1] = (A * np.sin(k * (x - G)) * np.cos(k * (y - G)))[None]
    f[2] = (-A * np.cos(k * (x - G)) * np.sin(k * (y - G)))[None]
    dom = fb.make_domain(lx, lx, L, periodic_xy=G, buffer_depth=4)
    prm = dict(tblend=1.0, pin=0.0, nu=nu, d1=2, blend=1.0)
    got, _ = run_gpu(fb, ctx, dom, prm, fb.F64 if dt == "f64" else fb.F32, f, steps, monitor_every=0)
    inner = (slice(None), slice(G, -G), slice(G, -G))
    e0 = (f[1][inner] ** 2 + f[2][inner] ** 2).sum()
    e1 = (got[1][inner] ** 2 + got[2][inner] ** 2).sum()
    nu_eff = -np.log(e1 / e0) / (2 * 2 * k * k * steps)
    assert abs(nu_eff - nu) <= 0.01 * nu, nu_eff


def test_periodic_band_too_narrow(built, ctx):
    fb = built
    dom = fb.make_domain(40, 40, 8, periodic_xy=2)            # d1 = 2: the corrector reaches 4
    with pytest.raises(fb.FslbmError):
        fb.Solve(ctx, dom, fb.Params.make(d1=2), fb.F32)
