"""bench.py end to end on the GPU, as the driver runs it: one JSON line with the contract's keys,
the roofline and end-to-end objects, the measurements after the timed region (ensemble with its
bitwise check, precision per storage type), and the FP64 line's kernel and bytes per cell."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bench(*argv):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *argv], capture_output=True,
                       text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_default_line_contract():
    d = bench("--steps", "20", "--warmup", "3", "--cpu-seconds", "1", "--e2e-reps", "1")
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "roofline",
                "cpu_baseline", "e2e", "gpu_launches", "clocks"):
        assert key in d, key
    assert d["n_gpus"] == 1 and d["steps"] == 20 and d["value"] > 0 and d["dtype"] == "f32"
    rf = d["roofline"]
    assert rf["bound"] == "hbm" and rf["unit"] == "GB/s" and 0 < rf["frac"] < 1.5
    assert rf["algorithmic_bytes"] == 32.0 * d["config"]["cells"]
    assert d["e2e"]["h2d_bytes_per_step"] > 0 and d["e2e"]["d2h_bytes_per_step"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["gpu_launches"] >= d["steps"]
    ens = d["ensemble"]
    assert ens["batch_equals_plain_bitwise"] is True and ens["members"] == 64
    assert ens["value"] > ens["plain_one_at_a_time_mlups"] > 0
    err = d["precision"]["errors_200_steps_vs_f64"]
    assert set(err) == {"re500", "re2000", "re5300"}
    assert all(e["f32"]["rel_l2_u"] <= 1e-4 for e in err.values())


def test_fp64_line():
    d = bench("--dtype", "f64", "--steps", "20", "--warmup", "3", "--cpu-seconds", "0",
              "--e2e-reps", "0")
    assert d["dtype"] == "f64" and d["vs_baseline"] is None
    assert d["roofline"]["kernel"] == "fslbm_col_kernel<2,16>"
    assert d["roofline"]["algorithmic_bytes"] == 64.0 * d["config"]["cells"]
    assert "ensemble" not in d
