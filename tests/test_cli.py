"""fslbm_pipe input handling (no GPU needed): every input file is validated before the device
is used, and errors end the run with a message and a non-zero status."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

CLI = os.path.join(ROOT, "flowcontrast_b200", "fslbm_pipe")
SMALL = ["--lx", "40", "--ly", "40", "--lz", "60", "--radius", "10"]


def run(args, cwd):
    return subprocess.run([CLI, *args], cwd=cwd, capture_output=True, text=True, timeout=120)


def write_inputs(fb, d, mask=None):
    fb.write_param_txt(os.path.join(d, "param.txt"),
                       fb.Params.make(tblend=1.0, pin=0.003, nu=0.02, d1=2, delta=1, blend=0.0))
    m = fb.pipe_m_mask(20, 40, 10) if mask is None else mask
    fb.write_pipe_txt(os.path.join(d, "pipe.txt"), m)
    return m


@pytest.fixture
def cli(built):
    assert os.path.exists(CLI), "fslbm_pipe was not built"
    return built


def test_missing_param_txt(cli, tmp_path):
    r = run(SMALL + ["--steps", "10"], tmp_path)
    assert r.returncode == 1 and "param.txt" in r.stderr


def test_bad_option_prints_usage(cli, tmp_path):
    r = run(["--frobnicate", "1"], tmp_path)
    assert r.returncode == 2 and "usage" in r.stderr


def test_pipe_txt_wrong_size(cli, tmp_path):
    write_inputs(cli, tmp_path)
    r = run(["--lx", "40", "--ly", "40", "--lz", "61", "--radius", "10", "--steps", "10"], tmp_path)
    assert r.returncode == 1 and "pipe.txt" in r.stderr


def test_geometry_rejected(cli, tmp_path):
    m = cli.pipe_m_mask(20, 40, 10).copy()
    m[30, 0, 5] = 0                     # fluid on the box rim
    write_inputs(cli, tmp_path, m)
    r = run(SMALL + ["--steps", "10"], tmp_path)
    assert r.returncode == 1 and "geometry" in r.stderr


def test_restart_requested_but_missing(cli, tmp_path):
    write_inputs(cli, tmp_path)
    r = run(SMALL + ["--steps", "10", "--init", "restart"], tmp_path)
    assert r.returncode == 1 and "p3Dii" in r.stderr


def test_truncated_restart_file(cli, tmp_path):
    write_inputs(cli, tmp_path)
    for name in ("p3Dii", "ux3Dii", "uy3Dii", "uz3Dii"):
        np.zeros(40 * 40 * 60 - 1, np.float32).tofile(os.path.join(tmp_path, name))
    r = run(SMALL + ["--steps", "10"], tmp_path)
    assert r.returncode == 1 and "p3Dii" in r.stderr


def test_valid_inputs_reach_the_device(cli, tmp_path):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    write_inputs(cli, tmp_path)
    r = run(SMALL + ["--steps", "10"], tmp_path)
    assert r.returncode == 1 and "device" in r.stderr
