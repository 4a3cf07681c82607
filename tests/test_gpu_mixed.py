"""FP16 storage with FP32 arithmetic (dtype F16) against the oracle.

The FP16 form computes each step in FP32 exactly as the FP32 form does and rounds the four
stored fields stochastically to FP16 (unbiased; noise seeded by cell and step only). p, u and
v are stored as they are (p is already the deviation rho - 1 from rest); w is stored as the
deviation from a per-column FP32 base (the streamwise mean of the fields it was given), so its
rounding is relative to the flow's departure from that profile, not to the profile itself.
Stated tolerances:
  one step from an FP16-exact state: every stored value within one FP16 ulp (plus 2e-7, the
    FP32 reassociation of pressure's O(0.1) terms) of the FP32 oracle's value (stochastic
    rounding picks one of the two neighbours), and the rounding unbiased: |mean error| <=
    0.02 ulp over all values;
  per-step increments far below half an FP16 ulp survive: over 100 steps of a pure body-force
    drift the FP16 core-mean change matches the FP32 change within 5 % (round-to-nearest
    storage would keep it at zero);
  200 steps of the small Poiseuille pipe (64 x 32 x 32, Re 100): relative L2 error of u and of
    p (scaled as in the FP32 parity tests) <= 1e-4 against the FP64 oracle, the mixed-precision
    bar of the FP32 form;
  set/get round trip: p, u, v as their FP16 values; w within half an FP16 ulp of its deviation
    from the column's base.
"""
import numpy as np
import pytest

import oracle_lib as O
from test_gpu_parity import circle_mask, config1, errors, run_gpu, to_params

pytestmark = pytest.mark.gpu


def f16_ulp(x):
    a = np.maximum(np.abs(x), 2.0 ** -14)
    return 2.0 ** (np.floor(np.log2(a)) - 10)


def test_fp16_one_step_within_one_ulp_and_unbiased(built, ctx):
    fb = built
    lx = ly = 32
    L, R, c = 24, 14.0, 15.5
    m2 = circle_mask(lx, ly, R, c, c)
    dom = fb.make_domain(lx, ly, L, radius=R, cx=c, cy=c)
    rng = np.random.default_rng(11)
    f = np.zeros((4, L, ly, lx))
    f[0] = 2e-3 * rng.uniform(-1, 1, f[0].shape)
    f[1:3] = 0.03 * rng.uniform(-1, 1, f[1:3].shape)
    f[3] = -0.4 + 0.05 * rng.uniform(-1, 1, f[3].shape)
    f[:, :, m2 != 0] = 0.0
    f = f.astype(np.float16).astype(np.float64)
    prm = dict(tblend=0.8, pin=0.002, nu=0.02, d1=2, blend=1.0, force=(0.0, 0.0, -1e-5))
    # the oracle steps the state the solve holds: p, u, v as given (FP16-exact), w as the
    # column's base plus the stored FP16 deviation (one rounding at set_fields)
    sv = fb.Solve(ctx, dom, to_params(fb, prm, 0), fb.F16)
    sv.set_fields(f)
    held = sv.get_fields()
    sv.step(1)
    sv.sync()
    got = sv.get_fields()
    sv.close()
    assert np.array_equal(held[:3], f[:3])
    ref, _ = O.run_core(m2, L, held.astype(np.float32), prm, 1, monitor_every=0, dtype=np.float32)
    ref = ref.astype(np.float64)
    nw = m2 == 0
    d = (got - ref)[:, :, nw]
    ulp = f16_ulp(np.maximum(np.abs(got), np.abs(ref)))[:, :, nw]
    worst = float(np.max(np.abs(d) / (ulp + 2e-7)))
    assert worst <= 1.0, worst
    bias = float(np.mean(d / ulp))
    assert abs(bias) <= 0.02, bias
    assert np.all(got[:, :, ~nw] == 0.0)


def test_fp16_small_increments_survive(built, ctx):
    """Uniform streamwise flow in a pipe core under a body force: each step adds tblend*g =
    1e-6, about 1/500 of an FP16 ulp at |w| = 0.4."""
    fb = built
    lx = ly = 48
    L, R, c = 64, 22.0, 23.5
    m2 = circle_mask(lx, ly, R, c, c)
    dom = fb.make_domain(lx, ly, L, radius=R, cx=c, cy=c)
    f = np.zeros((4, L, ly, lx))
    f[3][:, m2 == 0] = -0.4
    prm = dict(tblend=0.5, pin=0.0, nu=0.05, d1=2, blend=1.0, force=(0.0, 0.0, -2e-6))
    n = 100
    core = np.zeros((ly, lx), bool)
    y, x = np.mgrid[0:ly, 0:lx]
    core[(x - c) ** 2 + (y - c) ** 2 <= 8.0 ** 2] = True
    out = {}
    for name, dt in (("f32", fb.F32), ("f16", fb.F16)):
        s = fb.Solve(ctx, dom, to_params(fb, prm, 0), dt)
        s.set_fields(f)
        w0 = float(np.mean(s.get_fields()[3][:, core]))       # -0.4 as stored (FP16: rounded)
        s.step(n)
        s.sync()
        out[name] = float(np.mean(s.get_fields()[3][:, core])) - w0
        s.close()
    assert out["f32"] < -5e-5, out          # the force accelerates the core (stored w < 0)
    assert abs(out["f16"] - out["f32"]) <= 0.05 * abs(out["f32"]), out


def test_fp16_config1_200_steps(built, ctx):
    dom, m2, f, prm = config1(built)
    ref, _ = O.run_core(m2, 64, f, prm, 200, monitor_every=50, radius=15.0)
    got, log = run_gpu(built, ctx, dom, prm, built.F16, f, 200)
    ep, eu, eps = errors(got, ref, m2)
    print(f"FP16 small 64x32x32 pipe, 200 steps: rel L2 u {eu:.3e}, p (scaled) {eps:.3e}")
    assert eu <= 1e-4 and eps <= 1e-4, (ep, eu, eps)
    assert [r["step"] for r in log] == [50, 100, 150, 200]


def test_fp16_set_get_round_trip(built, ctx):
    fb = built
    dom, m2, f, prm = config1(fb, L=16)
    s = fb.Solve(ctx, dom, to_params(fb, prm), fb.F16)
    s.set_fields(f)
    got = s.get_fields()
    want = f.astype(np.float16).astype(np.float64)
    want[:, :, m2 != 0] = 0.0
    assert np.array_equal(got[:3], want[:3])
    # w: the base is the column's streamwise mean, the stored deviation an FP16 value
    base = np.where(m2 == 0, f[3].mean(axis=0), 0.0).astype(np.float32)
    dev = f[3].astype(np.float32) - base[None]
    assert np.all(np.abs(got[3] - f[3]) <= 0.5 * f16_ulp(dev) + 1e-7)
    assert np.all(got[3][:, m2 != 0] == 0.0)
    # the profile itself is not rounded: the error stays far below raw FP16 storage of w
    assert np.max(np.abs(got[3] - f[3])) < 0.01 * 0.5 * np.max(f16_ulp(f[3][:, m2 == 0]))
    assert s.info()["dtype"] == fb.F16
    s.close()
