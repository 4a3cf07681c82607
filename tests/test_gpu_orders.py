"""Higher corrector orders on the GPU against the oracle (one-column kernel, 50 steps of a small
pipe). Tolerances as for the reference order: FP64 1e-12, FP32 1e-5 relative L2 (p scaled as in
the parity tests). d1 = 1 runs at nu = 0.12: with a stride of one cell the corrector
anti-diffuses the grid's finest modes and every order (the reference's too) diverges at small
nu."""
import numpy as np
import pytest

import oracle_lib as O
from test_gpu_parity import circle_mask, errors, run_gpu

pytestmark = pytest.mark.gpu

CASES = [  # dtype, d1, order, blend
    ("f32", 1, 6, 0.4), ("f32", 1, 8, 0.5), ("f32", 1, 10, 0.0), ("f32", 1, 12, 0.0),
    ("f32", 1, 14, 0.0), ("f32", 2, 6, 0.4), ("f32", 2, 8, 1.0), ("f64", 1, 6, 1.0),
    ("f64", 1, 8, 0.5),
]


def case(d1, order, blend):
    lx = ly = 32
    L, R, c = 24, 14.0, 15.5
    m2 = circle_mask(lx, ly, R, c, c)
    rng = np.random.default_rng(5)
    f = np.zeros((4, L, ly, lx))
    f[0] = 1e-3 * rng.uniform(-1, 1, f[0].shape)
    f[1:] = 0.02 * rng.uniform(-1, 1, f[1:].shape)
    f[3] -= 0.1
    f[:, :, m2 != 0] = 0
    prm = dict(tblend=0.8, pin=0.001, nu=0.12 if d1 == 1 else 0.03, d1=d1, blend=blend,
               fd_order=order, force=(0.0, 0.0, -1e-5))
    return m2, L, R, f, prm


@pytest.mark.parametrize("dt,d1,order,blend", CASES)
def test_order_parity(built, ctx, dt, d1, order, blend):
    fb = built
    m2, L, R, f, prm = case(d1, order, blend)
    dom = fb.make_domain(32, 32, L, radius=R, cx=15.5, cy=15.5)
    ref, mon = O.run_core(m2, L, f, prm, 50, monitor_every=25, radius=R)
    got, log = run_gpu(fb, ctx, dom, prm, fb.F64 if dt == "f64" else fb.F32, f, 50, monitor_every=25)
    _, eu, eps = errors(got, ref, m2)
    tol = 1e-12 if dt == "f64" else 1e-5
    assert eu <= tol and eps <= tol, (eu, eps)
    assert [r["step"] for r in log] == [25, 50]


@pytest.mark.parametrize("dt,d1,order", [("f32", 2, 10), ("f64", 2, 6), ("f16", 2, 6), ("f32", 1, 7)])
def test_unsupported_orders_rejected(built, ctx, dt, d1, order):
    fb = built
    dom = fb.make_domain(32, 32, 24, radius=14.0, cx=15.5, cy=15.5)
    prm = fb.Params.make(tblend=0.8, pin=0.001, nu=0.03, d1=d1, blend=0.0, fd_order=order)
    with pytest.raises(fb.FslbmError) as e:
        fb.Solve(ctx, dom, prm, {"f32": fb.F32, "f64": fb.F64, "f16": fb.F16}[dt])
    assert e.value.code == -1


def test_order_change_by_set_params(built, ctx):
    """A live parameter change of the order (as a param.txt reload would) switches kernels."""
    fb = built
    m2, L, R, f, prm = case(2, 6, 0.4)
    dom = fb.make_domain(32, 32, L, radius=R, cx=15.5, cy=15.5)
    p4 = dict(prm, fd_order=0, blend=1.0)
    mid, _ = O.run_core(m2, L, f, p4, 20, monitor_every=0, radius=R)
    ref, _ = O.run_core(m2, L, mid, prm, 20, monitor_every=0, radius=R)
    s = fb.Solve(ctx, dom, fb.Params.make(tblend=0.8, pin=0.001, nu=0.03, d1=2, blend=1.0,
                                          monitor_every=0, force=(0.0, 0.0, -1e-5)), fb.F32)
    s.set_fields(f)
    s.step(20)
    s.set_params(fb.Params.make(tblend=0.8, pin=0.001, nu=0.03, d1=2, blend=0.4, monitor_every=0,
                                force=(0.0, 0.0, -1e-5), fd_order=6))
    s.step(20)
    s.sync()
    _, eu, eps = errors(s.get_fields(), ref, m2)
    assert eu <= 1e-5 and eps <= 1e-5, (eu, eps)
    s.close()
