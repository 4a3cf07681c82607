#!/usr/bin/env python3
"""Benchmark of the plain FSLBM step on one B200 (replicas on N GPUs).

Workload (FP32): periodic pipe of 512 streamwise planes with a 128x128
cross-section, circle R = 63 centred at (63.5, 63.5), paper regime (tblend 0.02, nu 0.0111,
d1 2, order-4 corrector blend), body force from Re_tau = 180, seeded Poiseuille flow at bulk
Re ~ 5300 plus random-phase streamwise/azimuthal modes at 10 % of u_bulk. A "step" is one
FSLBM time step over the whole pipe. MLUPS counts every box cell (the paper's convention).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one process per GPU (torchrun); each rank advances its own replica of the pipe:
the solve does not shard (single-GPU by design), so there is no data-path collective; `value`
sums the replicas' cells over the slowest rank's time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W = dict(lx=128, ly=128, lz=512, R=63.0, cx=63.5, cy=63.5, nu=0.0111, tblend=0.02, d1=2,
         blend=1.0, re_bulk=5300.0, re_tau=180.0, seed=20261203)
PUBLISHED_MLUPS = 3790.0          # the reference's published FP32 D3Q27 FSLBM throughput
E2E_INNER = 200                   # time steps per end-to-end solve request
METRIC = "MLUPS (plain FSLBM step, all box cells)"


def physics():
    ub = W["re_bulk"] * W["nu"] / (2 * W["R"])
    ut = W["re_tau"] * W["nu"] / W["R"]
    return ub, 2 * ub, 2 * ut * ut / W["R"]


def workload_config(extra=None):
    ub, umax, g = physics()
    c = {"workload": "plain FSLBM FP32, periodic pipe 512 (z, streamwise) x 128 x 128, R=63, "
                     "bulk Re 5300 body force, order-4 corrector, tblend 0.02",
         "grid": [W["lz"], W["ly"], W["lx"]], "cells": W["lx"] * W["ly"] * W["lz"],
         "params": {"tblend": W["tblend"], "nu": W["nu"], "d1": W["d1"], "blend": W["blend"],
                    "force_z": -g, "monitor_every": 50},
         "l2": "inputs larger than L2: 2 x 134 MB FP32 state ping-pong vs 126 MB L2",
         "parallelism": "replicas (one independent pipe per GPU)"}
    if extra:
        c.update(extra)
    return c


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def barrier(world, local):
    if world > 1:
        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            dist.barrier(device_ids=[local])
        else:
            dist.barrier()


def max_over_ranks(x, world, local):
    """Max of a float over ranks (the slowest replica sets the job time)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = f"cuda:{local}" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.lines, self.proc = device, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self, t0, t1):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [(ts, l.split(", ")) for ts, l in self.lines]
        rows = [(ts, r) for ts, r in rows if len(r) >= 9]
        inside = [r for ts, r in rows if t0 - 0.1 <= ts <= t1 + 0.1] or [r for _, r in rows]
        sm = [float(r[1]) for r in inside if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in inside if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in inside for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(inside)}


def read_traffic():
    """DRAM bytes per step-kernel launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "fslbm_step2_f32_512x128x128.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("dram_bytes_per_launch_full_size:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def cpu_port_sample(seconds=10.0, planes=64, nthreads=0):
    """The oracle's FP32 restatement of the reference step on the host cores, on a bounded
    streamwise slice of the workload (same cross-section and parameters)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    import flowcontrast_b200 as fb
    ub, umax, g = physics()
    dom = fb.make_domain(W["lx"], W["ly"], planes, radius=W["R"], cx=W["cx"], cy=W["cy"])
    f = fb.init_poiseuille(dom, umax, noise=1e-3, modes=4, mode_amp=0.1 * ub / umax, seed=W["seed"])
    y, x = np.mgrid[0:W["ly"], 0:W["lx"]]
    m2 = np.where((x - W["cx"]) ** 2 + (y - W["cy"]) ** 2 <= W["R"] ** 2, 0, 125).astype(np.uint8)
    prm = dict(tblend=W["tblend"], pin=0.0, nu=W["nu"], d1=W["d1"], blend=W["blend"],
               force=(0.0, 0.0, -g))
    threads = nthreads or O.threads()
    f = f.astype(np.float32)
    f, _ = O.run_core(m2, planes, f, prm, 1, monitor_every=50, radius=W["R"], dtype=np.float32,
                      nthreads=threads)                      # warm-up
    steps, t0 = 0, time.perf_counter()
    while True:
        f, _ = O.run_core(m2, planes, f, prm, 1, monitor_every=50, radius=W["R"],
                          dtype=np.float32, nthreads=threads)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds and steps >= 3:
            break
    cells = W["lx"] * W["ly"] * planes
    return {"value": cells * steps / el / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port",
            "sample": f"{steps} FP32 steps of a {planes}-plane slice (128x128 cross-section) of "
                      f"the workload, oracle restatement of FSLBM.cu with OpenMP"}, el / steps


def run_reference_arm(args, rank, world, local):
    """--impl reference: the reference method's CPU implementation (the oracle port) on the
    host cores, rank 0 only, on a bounded slice per step."""
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    import flowcontrast_b200 as fb
    ub, umax, g = physics()
    threads = O.threads()
    # size the per-step slice so the whole run stays within about two minutes
    _, t_step64 = cpu_port_sample(seconds=0.0, planes=64, nthreads=threads)
    budget = 100.0 / max(1, args.steps + args.warmup)
    planes = int(max(6, min(W["lz"], 64 * budget / max(t_step64, 1e-6))))
    dom = fb.make_domain(W["lx"], W["ly"], planes, radius=W["R"], cx=W["cx"], cy=W["cy"])
    f = fb.init_poiseuille(dom, umax, noise=1e-3, modes=4, mode_amp=0.1 * ub / umax,
                           seed=W["seed"]).astype(np.float32)
    y, x = np.mgrid[0:W["ly"], 0:W["lx"]]
    m2 = np.where((x - W["cx"]) ** 2 + (y - W["cy"]) ** 2 <= W["R"] ** 2, 0, 125).astype(np.uint8)
    prm = dict(tblend=W["tblend"], pin=0.0, nu=W["nu"], d1=W["d1"], blend=W["blend"],
               force=(0.0, 0.0, -g))
    for _ in range(args.warmup):
        f, _ = O.run_core(m2, planes, f, prm, 1, monitor_every=50, radius=W["R"],
                          dtype=np.float32, nthreads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        f, _ = O.run_core(m2, planes, f, prm, 1, monitor_every=50, radius=W["R"],
                          dtype=np.float32, nthreads=threads)
    el = time.perf_counter() - t0
    cells = W["lx"] * W["ly"] * planes
    mlups = cells * args.steps / el / 1e6
    sample = (f"each step: one FP32 time step of a {planes}-plane slice (128x128 cross-section) "
              f"of the workload on {threads} host threads (oracle restatement of FSLBM.cu; the "
              "reference has no CPU implementation and its CUDA source predates CUDA 12)")
    line = {"metric": METRIC, "value": mlups, "unit": "MLUPS", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config({"sample_planes": planes}),
            "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local):
    import flowcontrast_b200 as fb
    from flowcontrast_b200 import build
    build.build()
    ub, umax, g = physics()
    ctx = fb.Context(local)
    dom = fb.make_domain(W["lx"], W["ly"], W["lz"], radius=W["R"], cx=W["cx"], cy=W["cy"],
                         buffer_depth=10)
    prm = fb.Params.make(tblend=W["tblend"], pin=0.0, nu=W["nu"], d1=W["d1"], delta=1,
                         blend=W["blend"], monitor_every=50, force=(0.0, 0.0, -g))
    s = fb.Solve(ctx, dom, prm, fb.F32)
    f0 = fb.init_poiseuille(dom, umax, noise=1e-3, modes=4, mode_amp=0.1 * ub / umax,
                            seed=W["seed"] + rank)
    s.set_fields(f0)
    cells = W["lx"] * W["ly"] * W["lz"]

    # warm-up, then exactly K timed steps between barriers and device syncs
    s.step(args.warmup)
    s.sync()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    s.set_timing(True)
    s.kernel_time()
    launches0 = s.info()["kernel_launches"]
    barrier(world, local)
    s.sync()
    t_wall0 = time.time()
    s.step(args.steps)
    s.sync()
    t_wall1 = time.time()
    ms_local = s.info()["last_step_ms"]        # CUDA events around the K steps, solve stream
    kern_ms, kern_n = s.kernel_time()
    s.set_timing(False)
    launches = s.info()["kernel_launches"] - launches0
    barrier(world, local)
    clocks = sampler.stop(t_wall0, t_wall1)
    ms = max_over_ranks(ms_local, world, local)
    umax_now = s.check()

    # end to end through the C ABI with pinned host buffers: upload the state, run a
    # 200-step solve request with its monitor read-back, download the state
    import torch
    shape = (W["lz"], W["ly"], W["lx"])
    host_in = [torch.from_numpy(np.ascontiguousarray(f0[k], np.float32)).pin_memory()
               for k in range(4)]
    host_out = [torch.empty(shape, dtype=torch.float32).pin_memory() for _ in range(4)]
    ptr_in = [t.data_ptr() for t in host_in]
    ptr_out = [t.data_ptr() for t in host_out]

    def request():
        s.set_fields_host(fb.F32, *ptr_in)
        s.step(E2E_INNER)
        s.monitor()
        s.get_fields_host(fb.F32, *ptr_out)

    reps = args.e2e_reps
    e2e = None
    if reps > 0:
        request()
    barrier(world, local)
    t0 = time.perf_counter()
    for _ in range(reps):
        request()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, local)
    state_bytes = 4 * cells * 4
    if reps > 0:
      e2e = {"value": world * cells * E2E_INNER * reps / e2e_s / 1e6, "unit": "MLUPS",
             "h2d_bytes_per_step": state_bytes / E2E_INNER,
             "d2h_bytes_per_step": (state_bytes + (E2E_INNER // 50) * 64) / E2E_INNER,
             "request": f"H2D of the FP32 state from pinned memory + {E2E_INNER} steps + "
                        "monitor read-back + D2H of the state, via fslbm_solve_set_fields/step/"
                        "monitor/get_fields"}

    if rank == 0:
        peak, peak_kind = hbm_peak()
        kern_avg_ms = kern_ms / max(kern_n, 1)
        alg_bytes = 32.0 * cells                  # read p,u,v,w + write p,u,v,w, FP32
        achieved = alg_bytes / (kern_avg_ms * 1e-3) / 1e9
        traffic = read_traffic()
        cpu, _ = cpu_port_sample(seconds=args.cpu_seconds) if args.cpu_seconds > 0 else (None, 0)
        value = world * cells * args.steps / (ms * 1e-3) / 1e6
        line = {"metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak",
                "vs_baseline": value / PUBLISHED_MLUPS, "dtype": "f32",
                "data": "synthetic (seeded Poiseuille + random-phase modes)",
                "config": workload_config({"e2e_request_steps": E2E_INNER}),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic,
                             "peak_source": f"{peak_kind} hbm_gbs",
                             "kernel": "fslbm_step2_kernel<2,32,packed>",
                             "kernel_ms_avg": kern_avg_ms, "algorithmic_bytes": alg_bytes},
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clocks, "max_abs_u": umax_now}
        print(json.dumps(line), flush=True)
    s.close()
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--e2e-reps", type=int, default=3)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            return run_reference_arm(args, rank, world, local)
        return run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
