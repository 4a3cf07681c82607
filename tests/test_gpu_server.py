"""Served solves (fslbm_server_*): continuous batching must not change any result.

Each request's final fields must equal, bit for bit, the same request run alone on a plain
solve (same start, same steps): the step's arithmetic per cell does not depend on the batch a
solve shares, and FP16 rounding noise is seeded by cell and step only. Requests arrive while
others run, with FP32 and FP16 storage mixed, and admission keeps the resident footprint
under the budget.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def pipe(fb, n, L):
    R = n / 2 - 1
    c = (n - 1) / 2
    return fb.make_domain(n, n, L, radius=R, cx=c, cy=c), R


def params(fb, R, re, monitor_every=50):
    ub = 0.1
    nu = 2 * R * ub / re
    return fb.Params.make(tblend=0.02, pin=0.0, nu=nu, d1=2, delta=1, blend=1.0,
                          monitor_every=monitor_every, force=(0.0, 0.0, -8 * nu * ub / R ** 2))


SPECS = [  # n, L, Re, steps, dtype, seed
    (24, 40, 80.0, 37, 1, 11), (40, 96, 900.0, 120, 2, 12), (33, 64, 300.0, 75, 1, 13),
    (56, 48, 2000.0, 150, 1, 14), (28, 128, 60.0, 53, 2, 15), (48, 32, 1500.0, 101, 1, 16),
    (36, 72, 500.0, 64, 2, 17), (64, 40, 2500.0, 88, 1, 18),
]


def alone(fb, ctx, n, L, re, steps, dtype, seed, init=None):
    dom, R = pipe(fb, n, L)
    s = fb.Solve(ctx, dom, params(fb, R, re), dtype)
    if init is None:
        s.init_poiseuille(0.2, noise=1e-3, modes=2, mode_amp=0.05, seed=seed)
    else:
        s.set_fields(init)
    s.step(steps)
    s.sync()
    out = s.get_fields(np.float32)
    last = s.monitor() if steps >= 50 else None
    s.close()
    return out, last


def test_served_equals_alone(built, ctx):
    fb = built
    with fb.Server(0, quantum=25) as srv:
        ids = []
        for k, (n, L, re, steps, dt, seed) in enumerate(SPECS):
            dom, R = pipe(fb, n, L)
            ids.append(srv.submit(dom, params(fb, R, re), dt, steps,
                                  init_spec=dict(umax=0.2, noise=1e-3, modes=2, mode_amp=0.05,
                                                 seed=seed)))
            if k % 3 == 2:
                time.sleep(0.02)          # later arrivals join rounds already running
        srv.drain(120)
        st = srv.stats()
        assert st["completed"] == len(SPECS) and st["failed"] == 0
        assert st["rounds"] >= 1 and st["bytes_resident"] == 0
        for rid, (n, L, re, steps, dt, seed) in zip(ids, SPECS):
            res = srv.poll(rid)
            assert res["status"] == fb.REQ_DONE and res["steps_done"] == steps
            assert res["t_submit"] <= res["t_admit"] <= res["t_done"]
            want, last = alone(fb, ctx, n, L, re, steps, dt, seed)
            got = srv.release(rid)
            assert np.array_equal(got, want), (n, L, dt, float(np.abs(got - want).max()))
            if last is not None:
                assert res["last"]["step"] == last["step"]
                assert res["last"]["q1"] == last["q1"]


def test_served_host_start(built, ctx):
    fb = built
    n, L, re, steps = 30, 48, 400.0, 60
    dom, R = pipe(fb, n, L)
    f0 = fb.init_poiseuille(dom, 0.2, noise=1e-3, modes=1, mode_amp=0.05, seed=5).astype(np.float32)
    with fb.Server(0) as srv:
        rid = srv.submit(dom, params(fb, R, re), fb.F32, steps, init=f0)
        res = srv.wait(rid, 60)
        assert res["status"] == fb.REQ_DONE
        want, _ = alone(fb, ctx, n, L, re, steps, fb.F32, 0, init=f0)
        assert np.array_equal(srv.fields(rid), want)


def test_served_budget_admission(built):
    fb = built
    dom, R = pipe(fb, 48, 96)
    foot = built.lib()
    import ctypes
    b = ctypes.c_int64()
    fb._check(foot.fslbm_solve_footprint(ctypes.byref(dom), fb.F32, ctypes.byref(b)))
    budget = int(2.5 * b.value)                     # two resident at a time
    with fb.Server(0, hbm_budget=budget, quantum=20) as srv:
        ids = [srv.submit(dom, params(fb, R, 300.0), fb.F32, 60, want_fields=False,
                          init_spec=dict(umax=0.2, seed=k)) for k in range(5)]
        peak_seen = 0
        while srv.stats()["completed"] < 5:
            st = srv.stats()
            assert st["bytes_resident"] <= budget
            peak_seen = max(peak_seen, st["resident"])
            time.sleep(0.002)
        st = srv.stats()
        assert st["bytes_peak"] <= budget and st["bytes_peak"] >= 2 * b.value
        res = [srv.poll(i) for i in ids]
        assert all(r["status"] == fb.REQ_DONE for r in res)
        # arrival order admission: the last two waited for earlier ones to leave
        assert res[4]["t_admit"] >= min(r["t_done"] for r in res[:2])


def test_served_rejects_and_fails(built):
    fb = built
    dom, R = pipe(fb, 48, 64)
    with fb.Server(0, hbm_budget=1 << 20) as srv:             # 1 MiB: nothing fits
        with pytest.raises(fb.FslbmError) as e:
            srv.submit(dom, params(fb, R, 300.0), fb.F32, 10)
        assert e.value.code == -7
    with fb.Server(0) as srv:
        bad = fb.Params.make(tblend=0.02, pin=0.0, nu=0.01, d1=3, blend=1.0)   # no FP16 kernel for d1 3
        rid = srv.submit(dom, bad, fb.F16, 10)
        ok = srv.submit(dom, params(fb, R, 300.0), fb.F32, 10)
        assert srv.wait(rid, 60)["status"] == fb.REQ_FAILED
        assert srv.wait(ok, 60)["status"] == fb.REQ_DONE


def test_many_admissions_after_retirements(built, ctx):
    """Requests retire and new ones are admitted round after round (short step budgets, small
    quantum, three waves). A new request's solve may land at the address of one that just
    retired; the server must still build its batch for the new request (its own work items and
    stop step): every request completes, and a spread of them equal the same request alone."""
    fb = built
    rng = np.random.default_rng(123)
    waves = []
    with fb.Server(0, quantum=7) as srv:
        for wave in range(3):
            ids = []
            for k in range(8):
                n = int(rng.integers(24, 60))
                L = int(rng.integers(24, 80))
                spec = (n, L, float(rng.uniform(60, 1500)), int(rng.integers(5, 40)),
                        1 if k % 3 else 2, 1000 * wave + k)
                dom, R = pipe(fb, n, L)
                ids.append((srv.submit(dom, params(fb, R, spec[2]), spec[4], spec[3],
                                       init_spec=dict(umax=0.2, noise=1e-3, modes=2,
                                                      mode_amp=0.05, seed=spec[5])), spec))
                time.sleep(0.003)
            waves.append(ids)
            time.sleep(0.01)
        srv.drain(120)
        st = srv.stats()
        assert (st["completed"], st["failed"]) == (24, 0), (st["completed"], st["failed"])
        for ids in waves:
            for j, (rid, (n, L, re, steps, dt, seed)) in enumerate(ids):
                res = srv.poll(rid)
                assert res["status"] == fb.REQ_DONE and res["steps_done"] == steps
                got = srv.release(rid)
                if j % 3 == 0:
                    want, _ = alone(fb, ctx, n, L, re, steps, dt, seed)
                    assert np.array_equal(got, want), (n, L, dt, steps)


@pytest.mark.parametrize("policy", ["all", "least_work"])
def test_round_policy_order(built, ctx, policy):
    """Request A has more steps but far less work (box cells x steps) than request B. When every
    round advances every resident request (SERVE_ALL), B, with fewer steps, finishes first; when
    rounds take the least work first, one request at a time (SERVE_LEAST_WORK, round_cells = 1),
    A finishes first. Either way both equal the same requests run alone."""
    fb = built
    a = (24, 32, 300.0, 120, 1, 41)           # n, L, Re, steps, dtype, seed: 18 Ki cells
    b = (56, 64, 900.0, 40, 1, 42)            # 196 Ki cells
    pol = fb.SERVE_ALL if policy == "all" else fb.SERVE_LEAST_WORK
    with fb.Server(0, quantum=10, policy=pol, round_cells=1) as srv:
        ids = []
        for n, L, re, steps, dt, seed in (b, a):
            dom, R = pipe(fb, n, L)
            ids.append(srv.submit(dom, params(fb, R, re), dt, steps,
                                  init_spec=dict(umax=0.2, noise=1e-3, modes=2, mode_amp=0.05,
                                                 seed=seed)))
        srv.drain(120)
        rb, ra = srv.poll(ids[0]), srv.poll(ids[1])
        assert ra["status"] == rb["status"] == fb.REQ_DONE
        if policy == "all":
            assert rb["t_done"] < ra["t_done"]
        else:
            assert ra["t_done"] < rb["t_done"]
        for rid, spec in zip(ids, (b, a)):
            want, _ = alone(fb, ctx, *spec)
            assert np.array_equal(srv.release(rid), want)

