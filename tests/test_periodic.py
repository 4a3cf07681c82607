"""Cross-section periodic in x and y (ghost band) in the oracle: the Taylor-Green vortex, the
benchmark the reference's README names next, and translation invariance (no GPU)."""
import numpy as np
import pytest

import oracle_lib as O


def taylor_green(n, G=4, L=8, A=1e-4):
    m = O.periodic_mask(n, n, G)
    ly, lx = m.shape
    y, x = np.mgrid[0:ly, 0:lx]
    k = 2 * np.pi / n
    f = np.zeros((4, L, ly, lx))
    f[1] = (A * np.sin(k * (x - G)) * np.cos(k * (y - G)))[None]
    f[2] = (-A * np.cos(k * (x - G)) * np.sin(k * (y - G)))[None]
    return m, f, k


def nu_effective(n, nu, blend, steps=20, G=4):
    m, f, k = taylor_green(n, G)
    g, _ = O.run_periodic(m, 8, G, f, dict(tblend=1.0, pin=0.0, nu=nu, d1=2, blend=blend), steps)
    ly, lx = m.shape
    inner = (slice(None), slice(G, ly - G), slice(G, lx - G))
    e0 = (f[1][inner] ** 2 + f[2][inner] ** 2).sum()
    e1 = (g[1][inner] ** 2 + g[2][inner] ** 2).sum()
    assert np.abs(g[3]).max() < 1e-15                # a two-dimensional flow stays so
    return -np.log(e1 / e0) / (2 * 2 * k * k * steps)


@pytest.mark.parametrize("blend", [0.0, 1.0])
def test_taylor_green_viscosity(blend):
    """Small-amplitude Taylor-Green vortex: kinetic energy decays as exp(-2 nu |k|^2 t) (one
    time unit per step at tblend 1). The effective viscosity is within 3 % of nu on a 32^2 box
    and converges with resolution (64^2 at least three times closer)."""
    nu = 0.05
    e32 = abs(nu_effective(32, nu, blend) - nu) / nu
    e64 = abs(nu_effective(64, nu, blend) - nu) / nu
    assert e32 <= 0.03, e32
    assert e64 <= e32 / 3, (e32, e64)


def test_periodic_roll_equivariance():
    """The periodic box commutes with a roll of the interior along x (seam jump and gauge on)."""
    n, G, L = 24, 4, 10
    rng = np.random.default_rng(2)
    inner = np.zeros((n, n), np.uint8)
    inner[8:13, 9:14] = 125                            # an obstacle
    m = O.periodic_mask(n, n, G, inner)
    f = np.zeros((4, L, n + 2 * G, n + 2 * G))
    f[:, :, G:-G, G:-G] = 0.01 * rng.uniform(-1, 1, (4, L, n, n)) * (inner == 0)
    prm = dict(tblend=0.8, pin=0.002, nu=0.05, d1=2, blend=1.0, force=(0.0, 0.0, -1e-5))
    a, ma = O.run_periodic(m, L, G, f, prm, 6, monitor_every=3, radius=10.0)
    r = 7
    m2 = O.periodic_mask(n, n, G, np.roll(inner, r, axis=1))
    f2 = np.zeros_like(f)
    f2[:, :, G:-G, G:-G] = np.roll(f[:, :, G:-G, G:-G], r, axis=3)
    b, mb = O.run_periodic(m2, L, G, f2, prm, 6, monitor_every=3, radius=10.0)
    assert np.allclose(np.roll(a[:, :, G:-G, G:-G], r, axis=3), b[:, :, G:-G, G:-G], rtol=0, atol=1e-14)
    keep = [0, 1, 2, 3, 4, 6]                       # all but the fixed-cell sample
    assert np.allclose(ma[:, keep], mb[:, keep], rtol=1e-12)
