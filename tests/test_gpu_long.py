"""Long horizon on the production pipe: 512 x 128 x 128, R = 63, bulk Re ~ 5300 forcing (Re_tau
180), 20 000 steps from a seeded Poiseuille start with random-phase modes. Full-volume
statistics are sampled every 100 steps over the second half (100 samples) and reduced to radial
profiles. The FP64 solve, pinned to the oracle on short horizons, is the reference.
Tolerances: mean axial velocity profile <= 1 % relative L2, Reynolds stresses <= 5 %, for
FP32 and for FP16 storage.
"""
import numpy as np
import pytest

from flowcontrast_b200 import stats as st

pytestmark = pytest.mark.gpu

STEPS, EVERY = 20000, 100


def profiles(fb, ctx, dtype):
    R, nu = 63.0, 0.0111
    dom = fb.make_domain(128, 128, 512, radius=R, cx=63.5, cy=63.5)
    ub = 5300 * nu / (2 * R)
    ut = 180 * nu / R
    prm = fb.Params.make(tblend=0.02, pin=0.0, nu=nu, d1=2, delta=1, blend=1.0, monitor_every=50,
                         force=(0.0, 0.0, -2 * ut * ut / R))
    s = fb.Solve(ctx, dom, prm, dtype)
    s.init_poiseuille(2 * ub, noise=1e-3, modes=4, mode_amp=0.05, seed=20261203)
    s.step(STEPS // 2)
    s.profile_reset()
    for _ in range(STEPS // 2 // EVERY):
        s.step(EVERY)
        s.profile_sample()
    s.sync()
    sums, n = s.profile_get()
    assert np.isfinite(s.check())
    s.close()
    return st.radial_profiles(sums, n, 512, 63.5, 63.5, R)


def test_long_horizon_statistics(built, ctx):
    fb = built
    ref = profiles(fb, ctx, fb.F64)
    assert ref["w"][0] > ref["w"][-1] > 0           # axial flow, slowest at the wall
    assert ref["ww"].max() > 1e-4                    # the flow carries fluctuations
    for dt in (fb.F32, fb.F16):
        got = profiles(fb, ctx, dt)
        err = {k: st.profile_error(got, ref, k, ref["counts"]) for k in ("w", "uu_r", "uu_t", "ww", "uw_r")}
        print(f"dtype {dt}: {err}")
        assert err["w"] <= 0.01, err
        assert max(err[k] for k in ("uu_r", "uu_t", "ww", "uw_r")) <= 0.05, err
