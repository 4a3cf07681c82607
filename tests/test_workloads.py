"""The seeded benchmark workloads: deterministic, and within the ranges and distributions the
ensemble and served benchmarks state (no GPU needed)."""
import math

import numpy as np

from flowcontrast_b200 import workloads as wl


def test_ensemble_is_seeded_and_in_range():
    a, b = wl.ensemble(64), wl.ensemble(64)
    assert [s.as_dict() for s in a] == [s.as_dict() for s in b]
    assert len(a) == 64 and len({s.seed for s in a}) == 64
    for s in a:
        assert 32 <= s.L <= 256 and 24 <= s.n <= 96
        assert 50.0 <= s.re <= 3000.0 and s.steps == 2000 and s.dtype == 1
        assert s.radius == s.n / 2 - 1
        # Re = 2 R u_b / nu and the Poiseuille body force g = 8 nu u_b / R^2
        assert math.isclose(2 * s.radius * wl.U_BULK / s.nu, s.re, rel_tol=1e-12)
        assert math.isclose(-s.force_z, 8 * s.nu * wl.U_BULK / s.radius ** 2, rel_tol=1e-12)
    assert wl.ensemble(64, seed=1)[0].as_dict() != a[0].as_dict()


def test_request_stream_distribution():
    reqs = wl.request_stream(4000, rate=200.0)
    assert [r.as_dict() for r in reqs[:50]] == [r.as_dict() for r in wl.request_stream(50)]
    arrivals = np.array([r.arrival for r in reqs])
    gaps = np.diff(np.concatenate([[0.0], arrivals]))
    assert (gaps > 0).all()
    assert abs(gaps.mean() - 1 / 200.0) < 0.1 / 200.0          # Poisson at 200 per second
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.1           # exponential gaps: CV = 1
    steps = np.array([r.steps for r in reqs])
    assert steps.min() >= 200 and steps.max() <= 5000
    assert abs(steps.mean() - 2600) < 100
    re = np.array([r.re for r in reqs])
    assert re.min() >= 50 and re.max() <= 5000
    assert abs(np.log(re).mean() - 0.5 * (math.log(50) + math.log(5000))) < 0.1
    n = np.array([r.n for r in reqs])
    L = np.array([r.L for r in reqs])
    assert n.min() >= 24 and n.max() <= 96 and L.min() >= 32 and L.max() <= 256
    fp16 = np.mean([r.dtype == 2 for r in reqs])
    assert abs(fp16 - 0.5) < 0.05
