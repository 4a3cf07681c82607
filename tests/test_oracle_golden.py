"""Pins the oracle to the reference: the FP32 and FP64 instantiations of the oracle's step are
compared with golden fields produced by the reference's own kernels (FSLBMcalc, shiftback,
bcond of PipeDemoStandalone/FSLBM.cu, run on a B200 by tests/golden/make_ref_fixtures.py).

Cases with a monitor apply the reference's gauge: after step 50 the mean p of the first outlet
buffer plane (FSLBM.cu:630-647) is subtracted from p in step 51 (FSLBM.cu:628, 295-303); the
oracle's monitor forms that p2 in FP64, the reference's harness in FP32 as the reference does.

Tolerance: relative L2 over non-wall cells of the reference layout, separately for u=(u,v,w)
and for p scaled by |p| + 1.5|u|^2: 2e-6 up to 40 steps, growing in proportion beyond (both
sides compute in FP32 with different operation order, and their rounding differences grow with
the step count: FP32-vs-FP64 drift of the method itself is ~1e-6 over 40 steps). The
gauges agree to 1e-4 relative: the reference forms the cell count l1 by adding 1/(2 d2) in FP32
once per buffer cell (FSLBM.cu:589-591), about 2300 additions of an inexact 0.05 here, which
leaves it about 2e-5 off the exact count the oracle and the solver use. A gauge shifts p by
the same amount on every non-wall cell, and later steps keep a uniform shift of p uniform (the
weights sum to one and the wall rule copies the centre's p) without touching u, so p is
compared after removing the difference of the applied gauges (gauge_offset).
"""
import ctypes
import os

import numpy as np
import pytest

import oracle_lib as O
import ref_cases as RC

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 2e-6
GAUGE_TOL = 1e-4


def tol(n):
    """FP32-against-FP32 tolerance after n steps."""
    return TOL * max(1.0, n / 40.0)


def load(name):
    path = os.path.join(GOLDEN, f"ref_{name}.npz")
    if not os.path.exists(path):
        pytest.fail(f"golden fixture {path} is missing; generate it with "
                    "tests/golden/make_ref_fixtures.py on a GPU")
    return np.load(path)


def gauge_offset(g, case, n, ours):
    """Uniform p offset (ours - reference) after step n from the gauges applied before it: the
    p2 of the monitor at step k*monitor is subtracted in step k*monitor + 1."""
    monitor = case.get("monitor", 0)
    if not monitor:
        return 0.0
    ref_p2 = g[f"p2_step{max(case['steps'])}"].astype(np.float64)
    applied = [j for j in range(len(ours)) if (j + 1) * monitor < n]
    return float(sum(ref_p2[j] - ours[j] for j in applied))


def rel(a, b):
    eu = np.linalg.norm(a[1:] - b[1:]) / np.linalg.norm(b[1:])
    scale = np.linalg.norm(np.abs(b[0]) + 1.5 * (b[1:] ** 2).sum(0))
    return np.linalg.norm(a[0] - b[0]) / scale, eu


@pytest.mark.parametrize("name", list(RC.CASES))
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_oracle_matches_reference_kernels(name, dtype):
    g = load(name)
    c = RC.CASES[name]
    io, ref, prm = RC.inputs(name)
    keep = RC.nonwall_index(io)
    monitor = c.get("monitor", 0)
    f = ref.astype(dtype)
    done, gauge, gauges = 0, 0.0, []
    for n in c["steps"]:
        while done < n:
            f = O.step_ref(io, f, dict(prm, gauge=gauge), dtype=dtype)
            done += 1
            gauge = 0.0                                   # FSLBM.cu:628
            if monitor and done % monitor == 0:
                gauge = O.monitor_ref(io, f, prm["nu"], c["lx0"] / 2, d2=RC.D)[3]
                gauges.append(gauge)
        got = f.reshape(4, -1)[:, keep].astype(np.float64)
        got[0] -= gauge_offset(g, c, n, gauges)
        want = g[f"step{n}"].astype(np.float64)
        ep, eu = rel(got, want)
        assert ep < tol(n) and eu < tol(n), (name, n, ep, eu)
        if f"p2_step{n}" in g:
            want_p2 = g[f"p2_step{n}"].astype(np.float64)
            assert len(want_p2) == len(gauges) and np.all(np.abs(want_p2) > 0)
            assert np.allclose(gauges, want_p2, rtol=GAUGE_TOL, atol=0), (gauges, want_p2)


def test_gauge_cases_reach_a_nonzero_gauge():
    cases = [n for n, c in RC.CASES.items() if c.get("monitor")]
    assert cases
    for name in cases:
        c = RC.CASES[name]
        assert max(c["steps"]) > c["monitor"] and c["prm"]["blend"] != 0


def _ref_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libfslbm_ref.so")
    if not os.path.exists(path):
        pytest.skip("oracle/_ref is built only where the reference source is present")
    return ctypes.CDLL(path)


def test_reference_statistics_abs_is_floating_point():
    """The reference accumulates abs(dd) of doubles (FSLBM.cu:741-744) with only <cstdlib>
    among its includes (FSLBM.cu:28-34). Compiled by nvcc in its own translation unit, the
    unqualified abs resolves to a floating-point overload, not abs(int): the "RMS" statistics
    are mean absolute deviations, as the oracle (fabs) and the device kernel compute them."""
    L = _ref_lib()
    L.ref_abs_probe.restype = ctypes.c_double
    L.ref_abs_probe.argtypes = [ctypes.c_double]
    for x in (-0.25, -2.75, 3e-7, -1e-300, 0.5):
        assert L.ref_abs_probe(x) == abs(x)
