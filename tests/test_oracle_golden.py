"""Pins the oracle to the reference: the FP32 and FP64 instantiations of the oracle's step are
compared with golden fields produced by the reference's own kernels (FSLBMcalc, shiftback,
bcond of PipeDemoStandalone/FSLBM.cu, run on a B200 by tests/golden/make_ref_fixtures.py).

Tolerance: relative L2 over non-wall cells of the reference layout, separately for u=(u,v,w)
and for p scaled by |p| + 1.5|u|^2: 2e-6 (both sides compute in FP32 with different operation
order; FP32-vs-FP64 drift of the method itself is ~1e-6 over 40 steps on these cases).
"""
import os

import numpy as np
import pytest

import oracle_lib as O
import ref_cases as RC

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 2e-6


def load(name):
    path = os.path.join(GOLDEN, f"ref_{name}.npz")
    if not os.path.exists(path):
        pytest.fail(f"golden fixture {path} is missing; generate it with "
                    "tests/golden/make_ref_fixtures.py on a GPU")
    return np.load(path)


def rel(a, b):
    eu = np.linalg.norm(a[1:] - b[1:]) / np.linalg.norm(b[1:])
    scale = np.linalg.norm(np.abs(b[0]) + 1.5 * (b[1:] ** 2).sum(0))
    return np.linalg.norm(a[0] - b[0]) / scale, eu


@pytest.mark.parametrize("name", list(RC.CASES))
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_oracle_matches_reference_kernels(name, dtype):
    g = load(name)
    io, ref, prm = RC.inputs(name)
    keep = RC.nonwall_index(io)
    f = ref.astype(dtype)
    done = 0
    for n in RC.CASES[name]["steps"]:
        while done < n:
            f = O.step_ref(io, f, prm, dtype=dtype)
            done += 1
        got = f.reshape(4, -1)[:, keep].astype(np.float64)
        want = g[f"step{n}"].astype(np.float64)
        ep, eu = rel(got, want)
        assert ep < TOL and eu < TOL, (name, n, ep, eu)
