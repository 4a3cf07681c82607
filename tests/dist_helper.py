"""Run under torchrun by test_dist_cpu.py: bench.py's multi-rank helpers on two CPU ranks."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def main():
    out = sys.argv[1]
    rank, world, local = bench.dist_setup(world_n := int(os.environ["WORLD_SIZE"]))
    bench.barrier(world, local)
    slowest = bench.max_over_ranks(0.5 + rank, world, local)
    bench.barrier(world, local)
    with open(os.path.join(out, f"rank{rank}.json"), "w") as f:
        json.dump({"rank": rank, "world": world, "local": local, "max": slowest,
                   "requested": world_n}, f)
    import torch.distributed as dist
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
