"""Known-answer tests of the CPU oracle (the restatement of FSLBM.cu), no GPU needed.

The reference ships no tests or fixtures; these KATs follow from the method (PDF eqs. 1-10) and
from the reference's code structure. Golden outputs of the reference's own kernels are checked
separately in test_oracle_golden.py.
"""
import numpy as np
import pytest

import oracle_lib as O
import ref_cases as RC


def _mask2d_circle(lx, ly, r, cx=None, cy=None):
    cx = (lx - 1) / 2 if cx is None else cx
    cy = (ly - 1) / 2 if cy is None else cy
    y, x = np.mgrid[0:ly, 0:lx]
    return np.where((x - cx) ** 2 + (y - cy) ** 2 <= r * r, 0, 125).astype(np.uint8)


def test_pipe_m_restatements_agree(built):
    """pipe.m:36-60 restated three times (oracle C, test numpy, product C) must agree."""
    for lx0, l0, d in [(100, 300, 10), (12, 16, 10), (7, 5, 3)]:
        a = O.pipe_m_mask(lx0, l0, d)
        b = RC.pipe_m_mask(lx0, l0, d)
        c = built.pipe_m_mask(lx0, l0, d)
        assert np.array_equal(a, b) and np.array_equal(a, c)
    m = O.pipe_m_mask(100, 300, 10)
    assert m.shape == (320, 120, 120)
    # buffer planes carry the fluid pattern of the core planes as value 1
    assert ((m[10] == 0) == (m[0] == 1)).all() and ((m[10] == 0) == (m[-1] == 1)).all()
    assert 0.75 < (m[10] == 0).sum() / (np.pi * 50 ** 2) < 1.05
    assert set(np.unique(m)) == {0, 1, 125}
    assert (m[:, :10] == 125).all() and (m[:, :, :10] == 125).all()


def test_rest_state_is_fixed_point():
    """p = const, u = 0 is preserved (sum of W * 1.5 weights = 1)."""
    io = RC.pipe_m_mask(12, 16)
    f = np.zeros((4,) + io.shape)
    f[0] = 0.01 * (io != 125)
    prm = dict(tblend=0.7, pin=0.0, nu=0.01, d1=2, blend=0.5, d2=10)
    g = O.step_ref(io, f, prm)
    assert np.abs(g - f).max() < 1e-16


def test_uniform_flow_preserved_away_from_walls():
    """Uniform (p,u) is a fixed point where all 27 neighbours and corrector taps are fluid."""
    io = RC.pipe_m_mask(40, 30)
    f = np.zeros((4,) + io.shape)
    nw = io != 125
    f[0], f[1], f[2], f[3] = 0.002 * nw, 0.01 * nw, -0.02 * nw, 0.03 * nw
    prm = dict(tblend=1.0, pin=0.0, nu=0.05, d1=2, blend=1.0, d2=10)
    g = O.step_ref(io, f, prm)
    z, y, x = np.mgrid[0:io.shape[0], 0:io.shape[1], 0:io.shape[2]]
    far = ((x - 29.5) ** 2 + (y - 29.5) ** 2 < 12 ** 2) & (z >= 15) & (z < io.shape[0] - 15)
    assert np.abs(g[:, far] - f[:, far]).max() < 1e-15


def test_shear_wave_linear_decay():
    """u_x(z) = A sin(kz) evolves by the exact linear factor of predictor + corrector:
    G(k) = (4 + 2 cos k)/6 + dtddy*m*(c1*(2cos(d1 k) - 2) + c2*(2cos(2 d1 k) - 2))."""
    L, lx0 = 32, 48
    io0 = RC.pipe_m_mask(lx0, L)
    mask2d = np.where(io0[10] == 125, 125, 0).astype(np.uint8)
    ly, lx = mask2d.shape
    zc = np.arange(L)
    k = 2 * np.pi / L
    A = 1e-4
    f = np.zeros((4, L, ly, lx))
    f[1] = (A * np.sin(k * zc))[:, None, None] * (mask2d == 0)
    for d1, blend, nu in [(2, 0.0, 0.02), (2, 1.0, 0.05), (1, 0.0, 0.12)]:
        prm = dict(tblend=1.0, pin=0.0, nu=nu, d1=d1, blend=blend)
        steps = 3
        g, _ = O.run_core(mask2d, L, f, prm, steps, monitor_every=0)
        c1, c2 = 1 + 0.3333333333 * blend, -0.0833333333 * blend
        dtddy, m = nu - 0.16666666, 1.0 / d1 ** 2
        G = (4 + 2 * np.cos(k)) / 6 + dtddy * m * (c1 * (2 * np.cos(d1 * k) - 2) +
                                                  c2 * (2 * np.cos(2 * d1 * k) - 2))
        y, x = np.mgrid[0:ly, 0:lx]
        centre = (x - (lx - 1) / 2) ** 2 + (y - (ly - 1) / 2) ** 2 < 6 ** 2
        want = f[1][:, centre] * G ** steps
        got = g[1][:, centre]
        assert np.abs(got - want).max() < 1e-12 * A * 1e4, (d1, blend)


def test_roll_equivariance_without_jump():
    """With pin = 0 the periodic core is translation invariant along z."""
    io0 = RC.pipe_m_mask(12, 20)
    mask2d = np.where(io0[10] == 125, 125, 0).astype(np.uint8)
    f = RC.core_state(mask2d, 20, 3, 0.05, 0.01, 1e-3, dtype=np.float64)
    prm = dict(tblend=0.8, pin=0.0, nu=0.03, d1=2, blend=0.6)
    a, _ = O.run_core(mask2d, 20, f, prm, 4, monitor_every=0)
    b, _ = O.run_core(mask2d, 20, np.roll(f, 7, axis=1), prm, 4, monitor_every=0)
    assert np.abs(np.roll(a, 7, axis=1) - b).max() < 1e-15


def test_pressure_jump_equals_seam_offset():
    """The +-pin buffer copies equal a periodic core whose p jumps by pin across the seam:
    running the core with pin and with the equivalent ramp-free field agrees with a direct
    reference-layout step on the padded field."""
    c = RC.CASES["pipe_m_r6"]
    io, _, prm = RC.inputs("pipe_m_r6")
    mask2d = np.where(io[10] == 125, 125, 0).astype(np.uint8)
    core = RC.core_state(mask2d, c["l0"], c["seed"], c["u0"], c["noise"], c["pnoise"],
                         dtype=np.float64)
    ref64 = RC.pad_reference(core, mask2d, prm["pin"])
    a = O.step_ref(io, ref64, prm)[:, 10:-10]
    b, _ = O.run_core(mask2d, c["l0"], core, prm, 1, monitor_every=0)
    assert np.abs(a - b).max() < 1e-15


def test_mirror_symmetry():
    """A circle centred in the box: reflecting x and negating u commutes with the step."""
    lx, ly, L = 24, 24, 12
    mask2d = _mask2d_circle(lx, ly, 9.6)
    rng = np.random.default_rng(5)
    f = rng.uniform(-1e-2, 1e-2, (4, L, ly, lx)) * (mask2d == 0)
    prm = dict(tblend=0.9, pin=0.001, nu=0.02, d1=2, blend=0.3)
    a, _ = O.run_core(mask2d, L, f, prm, 3, monitor_every=0)
    fr = f[:, :, :, ::-1].copy()
    fr[1] *= -1
    b, _ = O.run_core(mask2d, L, fr, prm, 3, monitor_every=0)
    br = b[:, :, :, ::-1].copy()
    br[1] *= -1
    assert np.abs(a - br).max() < 1e-15


def test_float_and_double_instantiations_track():
    io, ref, prm = RC.inputs("paper_tb002")
    a = ref.astype(np.float64)
    b = ref.astype(np.float32)
    for _ in range(10):
        a = O.step_ref(io, a, prm)
        b = O.step_ref(io, b, prm, dtype=np.float32)
    nw = io != 125
    assert np.linalg.norm((a - b)[:, nw]) / np.linalg.norm(a[:, nw]) < 1e-6


def test_mask_contract_rejections():
    io = RC.pipe_m_mask(12, 16)
    bad = io.copy(); bad[15, 0, 5] = 0          # fluid on the rim
    assert O.lib().oracle_check_ref_mask(bad, 32, 32, 36, 10) == -4
    bad = io.copy(); bad[3, 16, 16] = 0         # fluid inside a buffer plane
    assert O.lib().oracle_check_ref_mask(bad, 32, 32, 36, 10) == -3
    bad = io.copy(); bad[15, 16, 16] = 7        # unknown cell type
    assert O.lib().oracle_check_ref_mask(bad, 32, 32, 36, 10) == -2
    assert O.lib().oracle_check_ref_mask(io, 32, 32, 36, 10) == 0


def test_monitor_formulas():
    """FSLBM.cu:632-666 on the reference layout: q2 == q1 (the outlet buffer copies plane d2),
    p1 - p2 == pin, f = (p1-p2)*4r/(3 q1^2 L), Re = 2 r q1 / nu."""
    io, ref, prm = RC.inputs("pipe_m_r6")
    f = O.step_ref(io, ref.astype(np.float64), prm)
    m = O.monitor_ref(io, f, prm["nu"], radius=6.0)
    q1, q2, p1, p2, ff, sample, re = m
    assert q1 == q2
    assert abs((p1 - p2) - prm["pin"]) < 1e-15
    L = io.shape[0] - 20
    assert abs(ff - (p1 - p2) / q1 / q1 / 3 * 4 * 6.0 / L) < 1e-12 * abs(ff)
    assert abs(re - 2 * 6.0 * q1 / prm["nu"]) < 1e-12 * abs(re)
    lz, ly, lx = io.shape
    assert sample == f[3, lz // 2].ravel()[(ly * lx) // 2 + lx // 2]


def _stats_numpy(acc, planes, cnt):
    """FSLBM.cu:715-748 restated in numpy (independent of the oracle's C version)."""
    p, u, v, w = planes
    pav, uxav, uyav, uzav, p2av, ux2av, uy2av, uz2av, uxyav, uxzav, uyzav = acc
    pav += p; dd1 = pav / cnt - p
    uxav += u; dd2 = uxav / cnt - u
    uyav += v; dd3 = uyav / cnt - v
    uzav += w; dd4 = uzav / cnt - w
    p2av += np.abs(dd1); ux2av += np.abs(dd2); uy2av += np.abs(dd3); uz2av += np.abs(dd4)
    uxyav += dd2 * dd3; uxzav += dd2 * dd4; uyzav += dd4 * dd3


def test_stats_accumulation_restatements_agree():
    rng = np.random.default_rng(9)
    n = 500
    a = np.zeros((11, n)); b = np.zeros((11, n))
    for cnt in range(1, 6):
        planes = rng.normal(size=(4, n))
        O.stats_accumulate(a, *planes, cnt)
        _stats_numpy(b, planes, cnt)
    assert np.abs(a - b).max() < 1e-13
