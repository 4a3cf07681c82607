"""Statistics on the device against the oracle.

Plane statistics (FSLBM.cu:683-768): on the YZ plane x = lx/2 of the reference layout (buffer
planes rebuilt as bcond's copies with +-pin), running sums of p, u, v, w, the mean absolute
deviation from the running mean and the cross products of the velocity deviations, with the
`delta` reset policy applied before each sample (0: everything restarts, 1: the fluctuation
sums restart, 2: nothing does). A pipe of 40 x 40 cross-section and 40 core planes (a 40x40x60
reference box) is sampled every 25 steps through a delta schedule 2,2,1,2,0,2,2,1,2 while the
flow develops; after every sample fslbm_stats_get must equal the oracle's
oracle_stats_accumulate fed the same plane values (taken from the solve's own state), with the
reset policy applied on the host as the reference does.

Full-volume profile statistics: per cross-section cell, sums over z and samples of
p, u, v, w and the six second moments against NumPy sums of the same states.

Tolerance: 1e-12 relative (both sides are FP64 sums of the same stored values; they differ
only in the order of additions and the device's compensated sums), for FP64 and FP32 storage.
"""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

TOL = 1e-12


def ref_plane(f, mask2d, L, d2, pin, xs, fp32):
    """The YZ plane x = xs of the reference layout from core fields f (4, L, ly, lx): values
    ordered y + ly * z_ref, buffer planes wrapped with +pin (inlet) / -pin (outlet) on non-wall
    cells, formed in the storage type's arithmetic."""
    zr = np.arange(L + 2 * d2)
    zc = (zr - d2) % L
    pl = f[:, zc][..., xs]                                     # (4, L + 2 d2, ly)
    jump = np.where(zr < d2, 1.0, np.where(zr >= d2 + L, -1.0, 0.0))[:, None]
    off = jump * (mask2d[:, xs] != 125)[None, :]
    if fp32:
        p = (pl[0].astype(np.float32) + off.astype(np.float32) * np.float32(pin)).astype(np.float64)
    else:
        p = pl[0] + off * pin
    return [p.ravel(), pl[1].ravel(), pl[2].ravel(), pl[3].ravel()]


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_plane_statistics_match_oracle(built, ctx, dtype):
    fb = built
    lx = ly = 40
    L, d2, R = 40, 10, 17.0
    y, x = np.mgrid[0:ly, 0:lx]
    m2 = np.where((x - 19.5) ** 2 + (y - 19.5) ** 2 <= R * R, 0, 125).astype(np.uint8)
    dom = fb.make_domain(lx, ly, L, mask=m2, radius=R, buffer_depth=d2)
    prm = fb.Params.make(tblend=0.7, pin=0.003, nu=0.02, d1=2, delta=2, blend=1.0,
                         monitor_every=50, force=(0.0, 0.0, -2e-6))
    dt = fb.F64 if dtype == "f64" else fb.F32
    s = fb.Solve(ctx, dom, prm, dt)
    try:
        rng = np.random.default_rng(21)
        f = np.zeros((4, L, ly, lx))
        f[0] = 2e-3 * rng.uniform(-1, 1, f[0].shape)
        f[1:3] = 0.01 * rng.uniform(-1, 1, f[1:3].shape)
        f[3] = -0.05 + 0.01 * rng.uniform(-1, 1, f[3].shape)
        f *= (m2 == 0)
        s.set_fields(f)
        n = ly * (L + 2 * d2)
        acc = np.zeros(11 * n)
        cnt = cnt2 = 0
        for delta in (2, 2, 1, 2, 0, 2, 2, 1, 2):
            s.step(25)
            prm.delta = delta
            s.set_params(prm)
            if delta == 0:                      # FSLBM.cu:683-686
                acc[:] = 0.0
                cnt = cnt2 = 0
            elif delta == 1:                    # FSLBM.cu:688-690
                acc[4 * n:] = 0.0
                cnt2 = 0
            cnt += 1
            cnt2 += 1
            state = s.get_fields(np.float64)
            O.stats_accumulate(acc, *ref_plane(state, m2, L, d2, prm.pin, lx // 2, dt == fb.F32), cnt)
            s.stats_sample()
            got, c1, c2 = s.stats_get()
            assert (c1, c2) == (cnt, cnt2)
            want = np.concatenate([acc[:4 * n] / cnt, acc[4 * n:] / cnt2]).reshape(11, n)
            for k in range(11):
                assert rel(got[k], want[k]) <= TOL, (delta, k, rel(got[k], want[k]))
        assert np.abs(want[4:8]).max() > 0 and np.abs(want[8:]).max() > 0
    finally:
        s.close()


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_profile_statistics_match_sums(built, ctx, dtype):
    fb = built
    lx, ly, L, R = 37, 29, 48, 12.5
    y, x = np.mgrid[0:ly, 0:lx]
    m2 = np.where((x - 18.0) ** 2 + (y - 14.0) ** 2 <= R * R, 0, 125).astype(np.uint8)
    dom = fb.make_domain(lx, ly, L, mask=m2, radius=R, buffer_depth=4)
    prm = fb.Params.make(tblend=0.8, pin=0.0, nu=0.03, d1=2, delta=1, blend=1.0,
                         monitor_every=0, force=(0.0, 0.0, -5e-6))
    dt = fb.F64 if dtype == "f64" else fb.F32
    s = fb.Solve(ctx, dom, prm, dt)
    try:
        rng = np.random.default_rng(22)
        f = np.zeros((4, L, ly, lx))
        f[1:] = 0.02 * rng.uniform(-1, 1, f[1:].shape)
        f[3] -= 0.04
        f[0] = 1e-3 * rng.uniform(-1, 1, f[0].shape)
        f *= (m2 == 0)
        s.set_fields(f)
        want = np.zeros((10, ly, lx))
        for _ in range(5):
            s.step(20)
            s.profile_sample()
            g = s.get_fields(np.float64)
            p, u, v, w = g
            for k, a in enumerate((p, u, v, w, u * u, v * v, w * w, u * v, u * w, v * w)):
                want[k] += a.sum(axis=0)
        got, ns = s.profile_get()
        assert ns == 5
        for k in range(10):
            assert rel(got[k], want[k]) <= TOL, (k, rel(got[k], want[k]))
    finally:
        s.close()
