"""Radial profile reduction of the full-volume statistics (host logic, no GPU)."""
import numpy as np

from flowcontrast_b200 import stats as st


def test_radial_profiles_known_field():
    lx = ly = 64
    cx = cy = 31.5
    R, L, n = 30.0, 8, 5
    y, x = np.mgrid[0:ly, 0:lx]
    r = np.hypot(x - cx, y - cy)
    fluid = r <= R
    wmean = np.where(fluid, -0.5 * (1 - (r / R) ** 2), 0.0)     # stored (negated) axial velocity
    sig2 = 1e-3                                                   # <w'w'> everywhere in the fluid
    uw = 2e-4                                                     # <u'w'>, zero mean u
    sums = np.zeros((10, ly, lx))
    scale = n * L
    sums[3] = wmean * scale
    sums[6] = (wmean ** 2 + np.where(fluid, sig2, 0.0)) * scale
    sums[8] = np.where(fluid, uw, 0.0) * scale
    prof = st.radial_profiles(sums, n, L, cx, cy, R, nbins=10)
    rc = prof["r"]
    assert np.all(prof["counts"] > 0)
    assert np.allclose(prof["w"], 0.5 * (1 - rc ** 2), atol=0.02)
    assert np.allclose(prof["ww"], sig2, rtol=1e-12)
    # <u_r' w'> = cos(theta) <u'w'> averages to about zero over full rings
    assert np.all(np.abs(prof["uw_r"]) < 0.1 * uw)
    assert st.profile_error(prof, prof, "w") == 0.0
