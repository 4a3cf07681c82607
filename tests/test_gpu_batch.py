"""Batched ensemble: members of uneven size advanced together (one persistent launch per time
step, CUDA graph replay) must give each member's own plain-path result. The batched launch
chooses its own streamwise chunking; the step's per-cell arithmetic does not depend on it, so
fields and monitor records must agree exactly (FP32 and FP16 storage)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def member_specs(n=6, seed=4):
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        ny = int(rng.integers(24, 70))
        L = int(rng.integers(32, 140))
        R = ny / 2 - 1
        re = float(np.exp(rng.uniform(np.log(50), np.log(3000))))
        ub = 0.1
        nu = 2 * R * ub / re
        g = 8 * nu * ub / R ** 2
        specs.append(dict(lx=ny, ly=ny, L=L, R=R, nu=nu, g=g, ub=ub, seed=100 + i))
    return specs


def make_member(fb, ctx, sp, monitor_every=25, dtype=None):
    c = (sp["lx"] - 1) / 2
    dom = fb.make_domain(sp["lx"], sp["ly"], sp["L"], radius=sp["R"], cx=c, cy=c)
    prm = fb.Params.make(tblend=0.5, pin=0.0, nu=sp["nu"], d1=2, delta=1, blend=1.0,
                         monitor_every=monitor_every, force=(0.0, 0.0, -sp["g"]))
    s = fb.Solve(ctx, dom, prm, fb.F32 if dtype is None else dtype)
    f = fb.init_poiseuille(dom, 2 * sp["ub"], noise=0.02, modes=2, mode_amp=0.05, seed=sp["seed"])
    s.set_fields(f)
    return s


@pytest.mark.parametrize("use_graph,dtype", [(True, 1), (False, 1), (True, 2)])
def test_batch_matches_members_alone(built, ctx, use_graph, dtype):
    """dtype 1 = FP32, 2 = FP16 storage. The step's arithmetic per cell does not depend on the
    streamwise chunking and the FP16 rounding noise is seeded by cell and step only, so the
    batched result equals the member's own result exactly."""
    fb = built
    specs = member_specs()
    steps = 61   # odd: graph pairs plus one direct step
    alone = []
    for sp in specs:
        s = make_member(fb, ctx, sp, dtype=dtype)
        s.step(steps)
        s.sync()
        alone.append((s.get_fields(np.float32), s.monitor_log()))
        s.close()
    members = [make_member(fb, ctx, sp, dtype=dtype) for sp in specs]
    b = fb.Batch(ctx, members)
    b.step(steps, use_graph=use_graph)
    b.sync()
    assert b.elapsed_ms() > 0
    for s, (want, wlog) in zip(members, alone):
        got = s.get_fields(np.float32)
        err = np.linalg.norm((got - want).astype(np.float64)) / np.linalg.norm(want.astype(np.float64))
        assert err == 0.0, err
        assert s.info()["steps"] == steps
        glog = s.monitor_log()
        assert [r["step"] for r in glog] == [r["step"] for r in wlog] == [25, 50]
        # means of pressure cancel to ~1e-5; compare them on the scale of u_b^2 = 1e-2
        for r, w in zip(glog, wlog):
            for key, scale in (("q1", 0.0), ("p1", 1e-2), ("p2", 1e-2), ("sample", 0.0)):
                t = 1e-12 * max(abs(w[key]), scale, 1e-6)
                assert abs(r[key] - w[key]) <= t, (key, r[key], w[key])
    # members stay usable on their own after batched steps
    members[0].step(3)
    members[0].sync()
    assert members[0].info()["steps"] == steps + 3
    b.close()
    for s in members:
        s.close()


@pytest.mark.parametrize("tile_y,shape", [(16, 0), (16, 2), (32, 1), (32, 2)])
def test_batch_tile_heights_and_warp_shapes(built, ctx, monkeypatch, tile_y, shape):
    """The batch's own tile height (32 x 16 tiles, two CTAs per SM, or 32 x 32) and warp shape
    (32 x 2, 16 x 4 or 8 x 8 cells) place the threads differently but change no cell's
    arithmetic, and the batched monitor sums in the same order at either block size: fields and
    monitor records equal the members stepped alone, bit for bit."""
    monkeypatch.setenv("FSLBM_BATCH_TILE_Y", str(tile_y))
    fb = built
    specs = member_specs(n=4, seed=7)
    steps = 30
    alone = []
    for sp in specs:
        s = make_member(fb, ctx, sp)
        s.step(steps)
        s.sync()
        alone.append((s.get_fields(np.float32), s.monitor_log()))
        s.close()
    members = [make_member(fb, ctx, sp) for sp in specs]
    b = fb.Batch(ctx, members)
    for i in range(len(members)):
        b.set_tiling(i, 48, shape)
    b.step(steps)
    b.sync()
    for s, (want, wlog) in zip(members, alone):
        assert np.array_equal(s.get_fields(np.float32), want)
        glog = s.monitor_log()
        assert len(glog) == len(wlog) == 1
        for key in ("q1", "p1", "p2", "sample"):
            assert glog[0][key] == wlog[0][key], key
    b.close()
    for s in members:
        s.close()


def test_batch_fp64_members_step_alone(built, ctx):
    """FP64 members do not enter the persistent launch (FP32 / FP16 storage only): the batch steps
    them one after another through the FP64 column kernel, with each member's own result."""
    fb = built
    specs = member_specs(n=3, seed=11)
    steps = 20
    alone = []
    for sp in specs:
        s = make_member(fb, ctx, sp, dtype=fb.F64)
        s.step(steps)
        s.sync()
        alone.append(s.get_fields(np.float64))
        s.close()
    members = [make_member(fb, ctx, sp, dtype=fb.F64) for sp in specs]
    b = fb.Batch(ctx, members)
    b.step(steps)
    b.sync()
    for s, want in zip(members, alone):
        assert np.array_equal(s.get_fields(np.float64), want)
        assert s.info()["steps"] == steps
    b.close()
    for s in members:
        s.close()


def test_batch_member_stops(built, ctx):
    """Members with different step budgets share launches; each stops at its own budget and
    equals the member stepped alone for that many steps."""
    fb = built
    specs = member_specs(n=4, seed=9)
    budgets = [17, 40, 3, 33]
    alone = []
    for sp, n in zip(specs, budgets):
        s = make_member(fb, ctx, sp)
        s.step(n)
        s.sync()
        alone.append(s.get_fields(np.float32))
        s.close()
    members = [make_member(fb, ctx, sp) for sp in specs]
    b = fb.Batch(ctx, members)
    for i, n in enumerate(budgets):
        b.set_stop(i, n)
    b.step(25)
    b.step(25)
    b.sync()
    for s, n, want in zip(members, budgets, alone):
        assert s.info()["steps"] == n
        assert np.array_equal(s.get_fields(np.float32), want)
    b.close()
    for s in members:
        s.close()


def test_autotune_restores_state_and_keeps_results(built, ctx, tmp_path):
    """The autotuner times tilings on the batch itself and restores every member; tiling never
    changes results, so the tuned batch still equals each member stepped alone, and a saved
    table loads into another batch."""
    import json
    fb = built
    specs = member_specs(n=5, seed=21)
    steps = 30
    alone = []
    for sp in specs:
        s = make_member(fb, ctx, sp)
        s.step(steps)
        s.sync()
        alone.append((s.get_fields(np.float32), s.monitor_log()))
        s.close()
    members = [make_member(fb, ctx, sp) for sp in specs]
    b = fb.Batch(ctx, members)
    path = str(tmp_path / "tiling.json")
    table = b.autotune(trial_steps=4, path=path)
    assert table and all(set(v) >= {"chunk", "warp_shape"} for v in table.values())
    assert all(v["warp_shape"] in (0, 1, 2) for v in table.values())
    assert json.load(open(path))["format"] == "fslbm batch tiling 1"
    for s in members:
        assert s.info()["steps"] == 0 and s.monitor_log() == []
    b.step(steps)
    b.sync()
    for s, (want, wlog) in zip(members, alone):
        assert np.array_equal(s.get_fields(np.float32), want)
        assert [r["q1"] for r in s.monitor_log()] == [r["q1"] for r in wlog]
    b.close()
    again = [make_member(fb, ctx, sp) for sp in specs]
    b2 = fb.Batch(ctx, again)
    b2.load_tiling(path)
    b2.step(steps)
    b2.sync()
    for s, (want, _) in zip(again, alone):
        assert np.array_equal(s.get_fields(np.float32), want)
    b2.close()
    # a table in the earlier form ("warp16x4": 0 or 1, the same meaning as warp_shape 0 or 1) loads
    old_form = str(tmp_path / "tiling_old.json")
    with open(old_form, "w") as f:
        f.write('{"format": "fslbm batch tiling 1", "classes": {' + ", ".join(
            f'"{k}": {{"chunk": {v["chunk"]}, "warp16x4": {min(v["warp_shape"], 1)}, "trial_ms": 1.0}}'
            for k, v in table.items()) + "}}")
    third = [make_member(fb, ctx, sp) for sp in specs]
    b3 = fb.Batch(ctx, third)
    b3.load_tiling(old_form)
    b3.step(steps)
    b3.sync()
    for s, (want, _) in zip(third, alone):
        assert np.array_equal(s.get_fields(np.float32), want)
    b3.close()
    for s in members + again + third:
        s.close()


def test_reconfigured_member_is_refused(built, ctx):
    """The batched kernel counts a member's step complete after the member's own number of work
    items; a member reconfigured after the batch was made (here to the order-6 corrector, which
    the batched kernel does not run) is refused with FSLBM_ERR_STATE instead of being stepped
    from a stale item table."""
    fb = built
    specs = member_specs(n=3, seed=31)
    members = [make_member(fb, ctx, sp) for sp in specs]
    b = fb.Batch(ctx, members)
    b.step(4)
    b.sync()
    sp = specs[0]
    members[0].set_params(fb.Params.make(tblend=0.5, pin=0.0, nu=sp["nu"], d1=2, delta=1,
                                         blend=1.0, monitor_every=25,
                                         force=(0.0, 0.0, -sp["g"]), fd_order=6))
    with pytest.raises(fb.FslbmError) as e:
        b.step(2)
    assert e.value.code == -3
    b.close()
    for s in members:
        s.close()


@pytest.mark.parametrize("chain", ["1", "5"])
def test_chain_length_does_not_change_results(built, ctx, monkeypatch, chain):
    """Steps per chained launch (FSLBM_BATCH_CHAIN; odd values run as the next even count) only
    decide where launches end: 2 or 6 steps per launch, graph replays plus a remainder launch,
    give each member's own plain-path result bit for bit, monitors included."""
    fb = built
    monkeypatch.setenv("FSLBM_BATCH_CHAIN", chain)
    specs = member_specs(n=4, seed=57)
    steps = 53
    alone = []
    for sp in specs:
        s = make_member(fb, ctx, sp)
        s.step(steps)
        s.sync()
        alone.append((s.get_fields(np.float32), [r["q1"] for r in s.monitor_log()]))
        s.close()
    members = [make_member(fb, ctx, sp) for sp in specs]
    b = fb.Batch(ctx, members)
    b.step(steps)
    b.sync()
    for s, (want, q1) in zip(members, alone):
        assert np.array_equal(s.get_fields(np.float32), want)
        assert [r["q1"] for r in s.monitor_log()] == q1
        assert s.info()["steps"] == steps
    b.close()
    for s in members:
        s.close()
