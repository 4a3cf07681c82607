"""Geometry varying along the pipe (host logic and oracle, no GPU)."""
import numpy as np
import pytest

import oracle_lib as O
from flowcontrast_b200 import workloads as wl


def fields(mask3d, seed=3):
    L, ly, lx = mask3d.shape
    rng = np.random.default_rng(seed)
    f = np.zeros((4, L, ly, lx))
    f[0] = 1e-3 * rng.uniform(-1, 1, f[0].shape)
    f[1:] = 0.02 * rng.uniform(-1, 1, f[1:].shape)
    f[3] -= 0.05
    return f * (mask3d == 0)


PRM = dict(tblend=0.8, pin=0.002, nu=0.03, d1=2, blend=1.0, force=(0.0, 0.0, -1e-5))


def test_extruded_mask_per_plane_equals_cross_section():
    m3 = wl.rough_pipe_mask(24, 16, 9.5, amplitude=0.0)
    assert np.all(m3 == m3[0])
    f = fields(m3)
    a, ma = O.run_core(m3[0], 16, f, PRM, 12, monitor_every=5, radius=9.5)
    b, mb = O.run_core(m3, 16, f, PRM, 12, monitor_every=5, radius=9.5)
    assert np.array_equal(a, b) and np.array_equal(ma, mb)


def test_rough_pipe_roll_equivariance():
    """Without the seam jump and the gauge the step commutes with a streamwise roll."""
    m3 = wl.rough_pipe_mask(24, 20, 9.0, amplitude=1.5, seed=4)
    assert not np.all(m3 == m3[0])
    f = fields(m3)
    prm = dict(PRM, pin=0.0)
    a, _ = O.run_core(m3, 20, f, prm, 6, monitor_every=0)
    b, _ = O.run_core(np.roll(m3, 7, axis=0), 20, np.roll(f, 7, axis=1), prm, 6, monitor_every=0)
    assert np.allclose(np.roll(a, 7, axis=1), b, rtol=0, atol=1e-15)


def test_ref_mask_round_trip(built):
    fb = built
    core = wl.rough_pipe_mask(20, 12, 8.0, amplitude=1.0, seed=2)
    d2 = 3
    ref = np.concatenate([core[-d2:], core, core[:d2]])
    ref[:d2][ref[:d2] == 0] = 1
    ref[-d2:][ref[-d2:] == 0] = 1
    assert np.array_equal(fb.ref_mask_to_core3d(ref, d2), core)
    with pytest.raises(fb.FslbmError):
        fb.ref_mask_to_core(ref, d2)          # planes differ: not one extruded cross-section
    bad = ref.copy()
    bad[0][bad[0] == 1] = 125                 # buffer no longer a copy of its core plane
    with pytest.raises(fb.FslbmError):
        fb.ref_mask_to_core3d(bad, d2)
