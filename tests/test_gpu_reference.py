"""The CUDA path, driven through the reference-layout entry points of the C ABI
(fslbm_solve_set_fields_ref / get_fields_ref), against the reference's own kernels' output on
the golden cases. The periodic core with the +-pin seam must reproduce the reference's buffer
planes and bcond copies; cases with a monitor also the gauge p2 of step 50, applied in step 51.
Tolerance as in test_oracle_golden.py (FP32 against FP32)."""
import numpy as np
import pytest

import ref_cases as RC
from test_oracle_golden import GAUGE_TOL, gauge_offset, load, rel, tol

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(RC.CASES))
def test_gpu_matches_reference_kernels(built, ctx, name):
    g = load(name)
    c = RC.CASES[name]
    io, ref, prm = RC.inputs(name)
    keep = RC.nonwall_index(io)
    core = built.ref_mask_to_core(io, RC.D)
    lz, ly, lx = io.shape
    dom = built.make_domain(lx, ly, lz - 2 * RC.D, mask=core, radius=c["lx0"] / 2,
                            buffer_depth=RC.D)
    monitor = c.get("monitor", 0)
    params = built.Params.make(tblend=prm["tblend"], pin=prm["pin"], nu=prm["nu"],
                               d1=prm["d1"], delta=1, blend=prm["blend"], monitor_every=monitor)
    for dt in (built.F32, built.F64):
        for n in c["steps"]:
            s = built.Solve(ctx, dom, params, dt)
            s.set_fields_ref(ref)
            s.step(n)
            out = s.get_fields_ref()
            mons = s.monitor_log() if monitor else []
            s.close()
            got = out.reshape(4, -1)[:, keep].astype(np.float64)
            got[0] -= gauge_offset(g, c, n, [m["p2"] for m in mons])
            ep, eu = rel(got, g[f"step{n}"].astype(np.float64))
            assert ep < tol(n) and eu < tol(n), (name, dt, n, ep, eu)
            if f"p2_step{n}" in g:
                want = g[f"p2_step{n}"].astype(np.float64)
                p2 = np.array([m["p2"] for m in mons])
                assert len(p2) == len(want) and np.allclose(p2, want, rtol=GAUGE_TOL, atol=0)
