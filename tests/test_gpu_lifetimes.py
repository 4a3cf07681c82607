"""Handle lifetimes: a context is released only after its last solve and batch, so handles may
be destroyed in any order (error paths, or objects finalised in arbitrary order at interpreter
exit) without touching freed memory."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_solve(fb, ctx, L=24, n=28):
    c = (n - 1) / 2
    dom = fb.make_domain(n, n, L, radius=n / 2 - 1.5, cx=c, cy=c)
    s = fb.Solve(ctx, dom, fb.Params.make(nu=0.05, force=(0.0, 0.0, -1e-5)), fb.F32)
    s.set_fields(fb.init_poiseuille(dom, 0.05, noise=1e-3, seed=3))
    return s


def test_context_destroyed_before_its_solves(built):
    fb = built
    ref_ctx = fb.Context(0)
    ref = small_solve(fb, ref_ctx)
    ref.step(20)
    want = ref.get_fields(np.float32)
    ref.close()
    ref_ctx.close()

    ctx = fb.Context(0)
    a, b = small_solve(fb, ctx), small_solve(fb, ctx)
    batch = fb.Batch(ctx, [a, b])
    ctx.close()                      # the creator's reference only
    batch.step(10)
    batch.sync()
    a.close()                        # a member freed before its batch
    b.step(10)                       # the context's stream and pool are still alive
    b.sync()
    assert np.array_equal(b.get_fields(np.float32), want)
    batch.close()
    b.close()                        # the last reference: the context is released here


def test_bounded_device_waits_give_up_and_report(built, ctx):
    """The kernels' bounded waits (a gpu-scope counter wait of the chained batched launch, an
    mbarrier phase wait of the march) run against conditions nothing satisfies: both give up
    after the limit, the kernel returns, the host reads FSLBM_ERR_TIMEOUT, and the context keeps
    working (a solve afterwards steps normally)."""
    import time
    fb = built
    t0 = time.perf_counter()
    rc, bits = ctx.selftest_waits(limit_ms=5.0)
    dt = time.perf_counter() - t0
    assert rc == -6 and bits == 3, (rc, bits)
    assert dt < 5.0
    s = small_solve(fb, ctx)
    s.step(4)
    s.sync()
    assert np.isfinite(s.get_fields(np.float32)).all()
    s.close()
    with pytest.raises(fb.FslbmError):
        fb._check(fb.lib().fslbm_selftest_waits(ctx.handle, -1.0, None))
