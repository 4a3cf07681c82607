"""bench.py helpers that need no GPU.

The CPU legs of the benchmark (the timed CPU baseline and the reference arm) must start from
the same seeded state as the GPU arm without loading the solver library: their generator is
the oracle's, which must equal the library's fslbm_init_poiseuille bit for bit. A bench
subprocess of the reference arm's set-up must not map libfslbm.so.
"""
import os
import json
import subprocess
import sys

import numpy as np

import bench
import oracle_lib as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_oracle_start_equals_library_start(built):
    fb = built
    for (lx, ly, L, R, cx, cy, modes, seed) in [(24, 20, 9, 8.5, 11.5, 9.0, 4, 5),
                                                 (16, 16, 5, 7.0, 7.5, 7.5, 0, 1),
                                                 (33, 29, 7, 13.0, 16.0, 14.0, 16, 99)]:
        dom = fb.make_domain(lx, ly, L, radius=R, cx=cx, cy=cy)
        want = fb.init_poiseuille(dom, 0.07, noise=1e-3, modes=modes, mode_amp=0.2, seed=seed)
        got = O.init_poiseuille(lx, ly, L, R, cx, cy, 0.07, noise=1e-3, modes=modes,
                                mode_amp=0.2, seed=seed)
        assert np.array_equal(got, want)


def test_bench_seeded_start_is_the_workload_start(built):
    fb = built
    ub, umax, g = bench.physics()
    W = bench.W
    dom = fb.make_domain(W["lx"], W["ly"], 6, radius=W["R"], cx=W["cx"], cy=W["cy"])
    want = fb.init_poiseuille(dom, umax, noise=1e-3, modes=4, mode_amp=0.1 * ub / umax,
                              seed=W["seed"])
    assert np.array_equal(bench.seeded_start(O, 6), want)


def test_reference_arm_inputs_do_not_load_the_library():
    code = ("import sys; sys.path.insert(0, %r); import bench; "
            "O = bench._oracle(); f = bench.seeded_start(O, 4); "
            "print(open('/proc/self/maps').read())" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "liboracle.so" in r.stdout
    assert "libfslbm.so" not in r.stdout


def test_reference_arm_runs_and_prints_its_line():
    """`bench.py --impl reference` end to end on the host cores (no GPU needed for its timed
    part): one JSON line with the reference arm's keys, and the solver library never loaded."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "3"], capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("port", "reference")
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["config"] == bench.workload_config()


def test_fluid_fraction_of_the_bench_pipe():
    # R = 63 centred at (63.5, 63.5) in 128 x 128: 12 492 fluid cells per cross-section
    assert abs(bench.fluid_fraction() * 128 * 128 - 12492) < 0.5
