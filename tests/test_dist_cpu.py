"""bench.py's one-process-per-GPU path with two ranks on the CPU (gloo): process-group set-up
from the torchrun environment, barriers, and the max-over-ranks job time."""
import json
import os
import socket
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_gloo(tmp_path):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           os.path.join(HERE, "dist_helper.py"), str(tmp_path)]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    got = [json.load(open(tmp_path / f"rank{k}.json")) for k in range(2)]
    assert sorted(g["rank"] for g in got) == [0, 1]
    assert all(g["world"] == 2 and g["max"] == 1.5 for g in got)
