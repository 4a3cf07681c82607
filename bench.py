#!/usr/bin/env python3
"""Benchmark of the plain FSLBM step on one B200 (replicas on N GPUs).

Workload (the production pipe, FP32): periodic pipe of 512 streamwise planes with a 128x128
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
# plain workload's storage types (--dtype): library type, bytes per value, step kernel, the
# line's dtype (the arithmetic type; FP16 storage computes in FP32)
STORAGE = {"f32": ("F32", 4, "fslbm_step2_kernel<2,32,packed>", "f32"),
           "f64": ("F64", 8, "fslbm_col_kernel<2,16>", "f64"),
           "f16": ("F16", 2, "fslbm_step2_kernel<2,32,packed,__half>", "f16 storage, f32 arithmetic")}


def physics():
    ub = W["re_bulk"] * W["nu"] / (2 * W["R"])
    ut = W["re_tau"] * W["nu"] / W["R"]
    return ub, 2 * ub, 2 * ut * ut / W["R"]


def fluid_fraction():
    """Share of the box cells that are fluid (the circle of radius R in the cross-section)."""
    y, x = np.mgrid[0:W["ly"], 0:W["lx"]]
    return float(np.count_nonzero((x - W["cx"]) ** 2 + (y - W["cy"]) ** 2 <= W["R"] ** 2)) / (W["lx"] * W["ly"])


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


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def _oracle():
    """The test-only oracle library (the CPU restatement of the reference step); the CPU legs
    of the benchmark use it and never load the solver library."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    return O


def seeded_start(O, planes, seed_offset=0):
    """The workload's seeded start on `planes` streamwise planes, (4, planes, ly, lx) float64,
    from the oracle's generator (bitwise equal to the library's fslbm_init_poiseuille)."""
    ub, umax, g = physics()
    return O.init_poiseuille(W["lx"], W["ly"], planes, W["R"], W["cx"], W["cy"], umax,
                             noise=1e-3, modes=4, mode_amp=0.1 * ub / umax,
                             seed=W["seed"] + seed_offset)


def cpu_port_sample(seconds=10.0, planes=64, nthreads=0, dtype=np.float32):
    """The oracle's restatement of the reference step (FP32, or FP64 for an FP64 line) on the
    host cores, on a bounded streamwise slice of the workload (same cross-section and
    parameters)."""
    O = _oracle()
    ub, umax, g = physics()
    f = seeded_start(O, planes)
    y, x = np.mgrid[0:W["ly"], 0:W["lx"]]
    m2 = np.where((x - W["cx"]) ** 2 + (y - W["cy"]) ** 2 <= W["R"] ** 2, 0, 125).astype(np.uint8)
    prm = dict(tblend=W["tblend"], pin=0.0, nu=W["nu"], d1=W["d1"], blend=W["blend"],
               force=(0.0, 0.0, -g))
    threads = nthreads or O.threads()
    f = f.astype(dtype)
    f, _ = O.run_core(m2, planes, f, prm, 1, monitor_every=50, radius=W["R"], dtype=dtype,
                      nthreads=threads)                      # warm-up
    steps, t0 = 0, time.perf_counter()
    while True:
        f, _ = O.run_core(m2, planes, f, prm, 1, monitor_every=50, radius=W["R"],
                          dtype=dtype, nthreads=threads)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds and steps >= 3:
            break
    cells = W["lx"] * W["ly"] * planes
    return {"value": cells * steps / el / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port",
            "sample": f"{steps} {'FP64' if dtype == np.float64 else 'FP32'} steps of a {planes}-plane "
                      f"slice (128x128 cross-section) of "
                      f"the workload, oracle restatement of FSLBM.cu with OpenMP"}, el / steps


def reference_gpu_sample(steps=20):
    """The reference's own step kernels (FSLBMcalc, shiftback, bcond of FSLBM.cu) on this GPU,
    built from the reference source with a texture-object compatibility header into
    oracle/_ref (present only where the reference source was available at build time), on the
    same pipe in the reference layout (10 buffer planes each end). MLUPS over the 512 core
    planes, as the main metric counts. None when the library or a GPU is missing."""
    import ctypes
    path = os.path.join(ROOT, "oracle", "_ref", "libfslbm_ref.so")
    try:
        import torch
        if not (os.path.exists(path) and torch.cuda.is_available()):
            return None
    except ImportError:
        return None
    lib = ctypes.CDLL(path)
    u8 = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
    f32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    i = ctypes.c_int
    lib.ref_run.argtypes = [u8, i, i, i, i, f32, f32, f32, i, ctypes.POINTER(ctypes.c_float),
                            ctypes.POINTER(ctypes.c_uint)]
    d2, L = 10, W["lz"]
    core = seeded_start(_oracle(), L).astype(np.float32)
    f = np.concatenate([core[:, -d2:], core, core[:, :d2]], axis=1)
    y, x = np.mgrid[0:W["ly"], 0:W["lx"]]
    fluid = (x - W["cx"]) ** 2 + (y - W["cy"]) ** 2 <= W["R"] ** 2
    io = np.where(fluid, 0, 125).astype(np.uint8)[None].repeat(L + 2 * d2, axis=0)
    io[:d2][:, fluid] = 1
    io[-d2:][:, fluid] = 1
    prm = np.array([W["tblend"], 0.0, W["nu"], W["d1"], W["blend"]], np.float32)
    out = np.empty_like(f)
    ms, oob = ctypes.c_float(0), ctypes.c_uint(0)
    rc = lib.ref_run(io, W["lx"], W["ly"], L + 2 * d2, d2, prm, np.ascontiguousarray(f).ravel(),
                     out.ravel(), steps, ctypes.byref(ms), ctypes.byref(oob))
    if rc != 0:
        return {"unavailable": f"ref_run returned {rc}"}
    cells = W["lx"] * W["ly"] * L
    return {"value": cells * steps / (ms.value * 1e-3) / 1e6, "unit": "MLUPS", "steps": steps,
            "kind": "the reference's FSLBMcalc/shiftback/bcond kernels on this GPU (CUDA-12 "
                    "texture-object compatibility header), 512+2x10 planes, core cells counted"}


def run_reference_arm(args, rank, world, local):
    """--impl reference: the reference method's CPU implementation (the oracle port) on the
    host cores, rank 0 only, on a bounded slice per step."""
    if rank != 0:
        return 0
    O = _oracle()
    ub, umax, g = physics()
    threads = O.threads()
    # size the per-step slice so the whole run stays within about two minutes
    _, t_step64 = cpu_port_sample(seconds=0.0, planes=64, nthreads=threads)
    budget = 100.0 / max(1, args.steps + args.warmup)
    planes = int(max(6, min(W["lz"], 64 * budget / max(t_step64, 1e-6))))
    f = seeded_start(O, planes).astype(np.float32)
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
            "fluid_mlups": mlups * fluid_fraction(),
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(), "sample_planes": planes,
            "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "reference_gpu": reference_gpu_sample()}
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
    st_name, es, kernel_name, dtype_name = STORAGE[args.dtype]
    s = fb.Solve(ctx, dom, prm, getattr(fb, st_name))
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
             "request_steps": E2E_INNER,
             "request": f"H2D of the FP32 state from pinned memory + {E2E_INNER} steps + "
                        "monitor read-back + D2H of the state, via fslbm_solve_set_fields/step/"
                        "monitor/get_fields"}

    if rank == 0:
        peak, peak_kind = hbm_peak()
        kern_avg_ms = kern_ms / max(kern_n, 1)
        alg_bytes = 8.0 * es * cells              # read p,u,v,w + write p,u,v,w
        achieved = alg_bytes / (kern_avg_ms * 1e-3) / 1e9
        cpu, _ = (cpu_port_sample(seconds=args.cpu_seconds,
                                  dtype=np.float64 if args.dtype == "f64" else np.float32)
                  if args.cpu_seconds > 0 else (None, 0))
        value = world * cells * args.steps / (ms * 1e-3) / 1e6
        line = {"metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world,
                "fluid_mlups": value * fluid_fraction(),
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak",
                "vs_baseline": value / PUBLISHED_MLUPS if args.dtype == "f32" else None,
                "dtype": dtype_name,
                "data": "synthetic (seeded Poiseuille + random-phase modes)",
                "config": workload_config() if args.dtype == "f32" else workload_config({
                    "workload": f"plain FSLBM, {args.dtype.upper()} storage, periodic pipe 512 (z, "
                                "streamwise) x 128 x 128, R=63, bulk Re 5300 body force, order-4 "
                                "corrector, tblend 0.02",
                    "l2": f"inputs larger than L2: 2 x {8 * es * cells / 2 / 1e6:.0f} MB state "
                          "ping-pong vs 126 MB L2"}),
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": None,
                             "traffic_note": "DRAM counters need a profiler, so the run does not "
                                             "measure them; per-launch DRAM bytes of ncu captures "
                                             "are in profiles/",
                             "peak_source": f"{peak_kind} hbm_gbs",
                             "kernel": kernel_name,
                             "kernel_ms_avg": kern_avg_ms, "algorithmic_bytes": alg_bytes},
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clocks, "max_abs_u": umax_now}
        if world == 1 and args.dtype == "f32" and not args.no_extras:
            line.update(extra_measurements(args))
        print(json.dumps(line), flush=True)
    s.close()
    ctx.close()
    return 0


def extra_measurements(args):
    """Measured after the timed region of the single-GPU default line, on the same GPU: the
    batched ensemble against the same pipes one at a time (500 steps each way), and the error of
    each storage form against FP64 after 200 steps on the production pipe."""
    import copy
    a = copy.copy(args)
    a.steps, a.warmup, a.ensemble_dtype, a.tuning_out = 500, 20, "f32", None
    ens = ensemble_line(a)
    mix = mixed_line(a)
    return {
        "ensemble": {"workload": ens["config"]["workload"], "members": ens["config"]["members"],
                     "cells": ens["config"]["cells"], "steps": ens["steps"],
                     "value": ens["value"], "unit": "MLUPS",
                     "plain_one_at_a_time_mlups": ens["plain_one_at_a_time_mlups"],
                     "speedup_vs_plain": ens["speedup_vs_plain"],
                     "batch_equals_plain_bitwise": ens["batch_equals_plain_bitwise"],
                     "kernel": ens["roofline"]["kernel"], "clocks": ens["clocks"]},
        "precision": {"workload": mix["config"]["workload"],
                      "errors_200_steps_vs_f64": mix["errors_200_steps"], "mlups": mix["mlups"]},
    }


# ------------------------------------------------------------------------------------------
# other workloads (one JSON line each; the default line above is the plain step)
# ------------------------------------------------------------------------------------------
def _member_start(fb, s, sp):
    from flowcontrast_b200 import workloads as wl
    s.init_poiseuille(2 * wl.U_BULK, noise=1e-3, modes=4, mode_amp=0.05, seed=sp.seed)


def batch_kernel_name(storage):
    """The batched kernel the library launches: 32 x 16 tiles unless FSLBM_BATCH_TILE_Y=32,
    packed pair arithmetic unless FSLBM_BATCH_PACKED=0."""
    ty = 32 if os.environ.get("FSLBM_BATCH_TILE_Y") == "32" else 16
    form = "scalar" if os.environ.get("FSLBM_BATCH_PACKED") == "0" else "packed"
    te = "__half" if storage == "f16" else "float"
    return f"fslbm_step2_batch_kernel<2,{ty},{form},{te}> (chained steps)"


def ensemble_line(args):
    """Mixed-size ensemble (64 seeded pipes, L in [32,256], n in [24,96], Re in [50,3000]):
    the batched persistent launch (FP32 storage, or FP16 storage with --ensemble-dtype f16)
    against the same pipes stepped one at a time by the plain FP32 method. Returns its line."""
    import flowcontrast_b200 as fb
    from flowcontrast_b200 import build, workloads as wl
    build.build()
    ctx = fb.Context(0)
    specs = wl.ensemble(64, steps=args.steps)
    cells = sum(sp.cells for sp in specs)
    dt = fb.F16 if args.ensemble_dtype == "f16" else fb.F32

    def fresh(dtype=dt):
        out = [fb.Solve(ctx, sp.domain(fb), sp.params(fb), dtype) for sp in specs]
        for sp, s in zip(specs, out):
            _member_start(fb, s, sp)
        for s in out:
            s.sync()
        return out

    def one_at_a_time(dtype):
        """Device time of each member's K steps on the plain path, summed; final fields."""
        solves = fresh(dtype)
        for s in solves:
            s.step(args.warmup)
        ms = 0.0
        for s in solves:
            s.sync()
            s.step(args.steps)
            s.sync()
            ms += s.info()["last_step_ms"]
        fields = [s.get_fields(np.float32) for s in solves]
        for s in solves:
            s.close()
        return ms, fields

    # the plain method (FP32) one at a time, and the same storage type alone for the bitwise check
    plain_ms, plain_fields = one_at_a_time(fb.F32)
    alone_ms = plain_ms
    if dt != fb.F32:
        alone_ms, plain_fields = one_at_a_time(dt)

    # batched, default tiling (the shipped table): the same starts, chained steps (one
    # persistent launch per 16 steps, replayed from a CUDA graph)
    solves = fresh()
    b = fb.Batch(ctx, solves)
    b.step(args.warmup)
    b.sync()
    b.step(args.steps)
    b.sync()
    default_ms = b.elapsed_ms()
    same = all(np.array_equal(s.get_fields(np.float32), want) for s, want in zip(solves, plain_fields))
    b.close()
    for s in solves:
        s.close()

    # batched after the autotuner (tiling per size class timed on this batch, state restored)
    import tempfile
    solves = fresh()
    b = fb.Batch(ctx, solves)
    t_tune = time.perf_counter()
    tune_path = args.tuning_out or os.path.join(tempfile.mkdtemp(), "batch_tiling.json")
    table = b.autotune(trial_steps=20, path=tune_path)
    t_tune = time.perf_counter() - t_tune
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    b.step(args.warmup)
    b.sync()
    launches0 = solves[0].info()["kernel_launches"]
    t_w0 = time.time()
    b.step(args.steps)
    b.sync()
    t_w1 = time.time()
    batch_ms = b.elapsed_ms()
    launches = solves[0].info()["kernel_launches"] - launches0   # batched launches (all members)
    clocks = sampler.stop(t_w0, t_w1)
    same = same and all(np.array_equal(s.get_fields(np.float32), want)
                        for s, want in zip(solves, plain_fields))

    # end to end: host starts in (pinned), K batched steps, fields out
    import torch
    host = [[torch.empty((sp.L, sp.n, sp.n), dtype=torch.float32).pin_memory() for _ in range(4)]
            for sp in specs]
    for f, h in zip(plain_fields, host):          # any host state of the right shape
        for k in range(4):
            h[k].copy_(torch.from_numpy(f[k]))
    t0 = time.perf_counter()
    for s, h in zip(solves, host):
        s.set_fields_host(fb.F32, *[t.data_ptr() for t in h])
    b.step(args.steps)
    for s, h in zip(solves, host):
        s.get_fields_host(fb.F32, *[t.data_ptr() for t in h])
    for s in solves:
        s.sync()
    e2e_s = time.perf_counter() - t0
    peak, peak_kind = hbm_peak()
    value = cells * args.steps / (batch_ms * 1e-3) / 1e6
    plain = cells * args.steps / (plain_ms * 1e-3) / 1e6
    achieved = 32.0 * cells * args.steps / (batch_ms * 1e-3) / 1e9
    line = {"metric": "aggregate MLUPS, batched ensemble (all box cells)", "value": value,
            "unit": "MLUPS", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": batch_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.ensemble_dtype, "data": "synthetic (seeded ensemble)",
            "config": {"workload": "64 seeded pipes, L~U[32,256] streamwise, n~U[24,96] square "
                                   "cross-section, R=n/2-1, Re log-uniform [50,3000] (u_b 0.1), "
                                   "tblend 0.02, d1 2, order-4 blend, "
                                   + ("FP16 storage (FP32 arithmetic)" if dt == fb.F16 else "FP32")
                                   + "; baseline: the plain FP32 method one pipe at a time",
                       "cells": cells, "members": len(specs),
                       "l2": f"inputs larger than L2: {2 * 16 * cells / 1e9:.2f} GB of state"},
            "plain_one_at_a_time_mlups": plain, "speedup_vs_plain": value / plain,
            "same_storage_one_at_a_time_mlups": cells * args.steps / (alone_ms * 1e-3) / 1e6,
            "default_tiling_mlups": cells * args.steps / (default_ms * 1e-3) / 1e6,
            "autotune": {"seconds": t_tune, "classes": len(table), "trial_steps": 20},
            "batch_equals_plain_bitwise": bool(same),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": None,
                         "peak_source": f"{peak_kind} hbm_gbs",
                         "kernel": batch_kernel_name(args.ensemble_dtype)},
            "e2e": {"value": cells * args.steps / e2e_s / 1e6, "unit": "MLUPS",
                    "h2d_bytes_per_step": 16.0 * cells / args.steps,
                    "d2h_bytes_per_step": 16.0 * cells / args.steps},
            "gpu_launches": launches, "clocks": clocks}
    b.close()
    for s in solves:
        s.close()
    ctx.close()
    return line


def run_ensemble(args):
    print(json.dumps(ensemble_line(args)), flush=True)
    return 0


def _pct(xs, q):
    return float(np.percentile(np.asarray(xs), q)) if xs else None


def serve_stream(fb, wl, reqs, policy, round_cells=0):
    """The seeded request stream submitted in real time to a fresh server with `policy`;
    returns its aggregate MLUPS, latency percentiles and makespan (no fields read back)."""
    srv = fb.Server(0, hbm_budget=int(150e9), quantum=50, policy=policy, round_cells=round_cells)
    for sp in reqs[:4]:                       # warm-up, not counted
        srv.submit(sp.domain(fb), sp.params(fb), sp.dtype, 20, want_fields=False,
                   init_spec=dict(umax=0.2, seed=1))
    srv.drain(600)
    ids = []
    t0 = time.perf_counter()
    for sp in reqs:
        dt = t0 + sp.arrival - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        ids.append(srv.submit(sp.domain(fb), sp.params(fb), sp.dtype, sp.steps, want_fields=False,
                              init_spec=dict(umax=2 * wl.U_BULK, noise=1e-3, modes=4,
                                             mode_amp=0.05, seed=sp.seed)))
    srv.drain(3600)
    res = [srv.poll(i) for i in ids]
    srv.close()
    done = [r for r in res if r["status"] == fb.REQ_DONE]
    lat = [r["t_done"] - r["t_submit"] for r in done]
    span = max(r["t_done"] for r in res) - min(r["t_submit"] for r in res)
    work = sum(r["cells"] * sp.steps for r, sp in zip(res, reqs) if r["status"] == fb.REQ_DONE)
    return {"value": work / span / 1e6, "unit": "MLUPS", "makespan_s": span,
            "latency_s": {"p50": _pct(lat, 50), "p95": _pct(lat, 95), "p99": _pct(lat, 99),
                          "max": max(lat) if lat else None},
            "completed": len(done), "failed": len(res) - len(done)}


def run_served(args):
    """Served solves: a seeded Poisson stream (--rate, 200 requests/s by default) of pipe solves
    (32^3 .. 256x96x96 cells, 200..5000 steps, Re 50..5000, FP32 or FP16 storage) submitted in
    real time to the continuous-batching server under a 150 GB budget."""
    import flowcontrast_b200 as fb
    from flowcontrast_b200 import build, workloads as wl
    build.build()
    f32_only = args.served_dtype == "f32"
    reqs = wl.request_stream(args.requests, rate=args.rate, mixed_fraction=0.0 if f32_only else 0.5)
    check = set(range(0, len(reqs), max(1, len(reqs) // 4)))     # requests checked afterwards
    srv = fb.Server(0, hbm_budget=int(150e9), quantum=50)
    # warm-up (kernel set-up and graph capture paths), not counted
    for sp in reqs[:4]:
        srv.submit(sp.domain(fb), sp.params(fb), sp.dtype, 20, want_fields=False,
                   init_spec=dict(umax=0.2, seed=1))
    srv.drain(600)
    base = srv.stats()
    sampler = ClockSampler(0)
    sampler.start()
    time.sleep(0.3)
    ids = []
    t0 = time.perf_counter()
    tw0 = time.time()
    for k, sp in enumerate(reqs):
        dt = t0 + sp.arrival - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        ids.append(srv.submit(sp.domain(fb), sp.params(fb), sp.dtype, sp.steps,
                              want_fields=k in check,
                              init_spec=dict(umax=2 * wl.U_BULK, noise=1e-3, modes=4,
                                             mode_amp=0.05, seed=sp.seed)))
    srv.drain(3600)
    tw1 = time.time()
    clocks = sampler.stop(tw0, tw1)
    res = [srv.poll(i) for i in ids]
    st = srv.stats()
    lat = [r["t_done"] - r["t_submit"] for r in res if r["status"] == fb.REQ_DONE]
    span = max(r["t_done"] for r in res) - min(r["t_submit"] for r in res)
    work = sum(r["cells"] * sp.steps for r, sp in zip(res, reqs) if r["status"] == fb.REQ_DONE)
    # per-request checks: the same request alone (same dtype) must match bit for bit; the
    # error against the FP64 solve of the same request is reported
    ctx = fb.Context(0)
    checks = []
    for k in sorted(check):
        sp, rid = reqs[k], ids[k]
        got = srv.release(rid)
        out = {}
        for name, dt in (("same", sp.dtype), ("f64", fb.F64)):
            s = fb.Solve(ctx, sp.domain(fb), sp.params(fb), dt)
            s.init_poiseuille(2 * wl.U_BULK, noise=1e-3, modes=4, mode_amp=0.05, seed=sp.seed)
            s.step(sp.steps)
            s.sync()
            out[name] = s.get_fields(np.float64)
            s.close()
        g = got.astype(np.float64)
        checks.append({"request": k, "cells": sp.cells, "steps": sp.steps, "re": round(sp.re, 1),
                       "dtype": "f16" if sp.dtype == fb.F16 else "f32",
                       "equals_alone": bool(np.array_equal(g, out["same"])),
                       "rel_l2_u_vs_f64": float(np.linalg.norm(g[1:] - out["f64"][1:]) /
                                                np.linalg.norm(out["f64"][1:]))})
    # the plain method on the same stream: a seeded sample of the requests run one at a time
    # (each its full step count), aggregate MLUPS = sample work / sample device time
    rng = np.random.default_rng(7)
    sample = sorted(rng.choice(len(reqs), size=min(32, len(reqs)), replace=False).tolist())
    alone_work = alone_ms = 0.0
    for k in sample:
        sp = reqs[k]
        s = fb.Solve(ctx, sp.domain(fb), sp.params(fb), sp.dtype)
        s.init_poiseuille(2 * wl.U_BULK, noise=1e-3, modes=4, mode_amp=0.05, seed=sp.seed)
        s.set_timing(True)
        s.step(sp.steps)
        s.sync()
        alone_ms += s.info()["last_step_ms"]
        alone_work += sp.cells * sp.steps
        s.close()
    plain_alone = alone_work / (alone_ms * 1e-3) / 1e6
    ctx.close()
    srv.close()
    # the same stream with rounds that take the requests with the least work left first
    least_work = serve_stream(fb, wl, reqs, fb.SERVE_LEAST_WORK)
    least_work["policy"] = "least work left first, 48 Mi box cells per round"
    line = {"metric": "aggregate MLUPS and p50/p95/p99 latency, served solves", "value": work / span / 1e6,
            "unit": "MLUPS", "n_gpus": 1, "steps": len(reqs), "warmup": 4,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if f32_only else "f32+f16", "data": "synthetic (seeded Poisson request stream)",
            "config": {"workload": f"{len(reqs)} requests, Poisson {args.rate:g}/s, cells log-uniform "
                                   "32^3..256x96x96, steps U[200,5000], Re log-uniform [50,5000], "
                                   + ("FP32 storage only" if f32_only else "FP32 or FP16 storage 50/50")
                                   + ", budget 150 GB, quantum 50",
                       "requests": len(reqs), "policy": "every resident request each round"},
            "latency_s": {"p50": _pct(lat, 50), "p95": _pct(lat, 95), "p99": _pct(lat, 99),
                          "max": max(lat) if lat else None},
            "completed": st["completed"] - base["completed"], "failed": st["failed"] - base["failed"],
            "makespan_s": span, "busy_s": st["busy_seconds"] - base["busy_seconds"],
            "rounds": st["rounds"] - base["rounds"], "peak_device_bytes": st["bytes_peak"],
            "worker_seconds": {k: st[k] - base[k] for k in
                               ("t_admit", "t_regroup", "t_launch", "t_wait", "t_retire")},
            "checks": checks, "clocks": clocks,
            "plain_one_at_a_time_mlups": plain_alone,
            "plain_sample": f"{len(sample)} requests of the stream (seeded), each stepped alone on "
                            "the plain path for its full step count, device time",
            "speedup_vs_plain": work / span / 1e6 / plain_alone,
            "least_work_first": least_work}
    print(json.dumps(line), flush=True)
    return 0


def mixed_line(args):
    """Storage precision on the production pipe (512x128x128, Re 500/2000/5300): error of the
    FP32 and FP16-storage forms against the FP64 solve after 200 steps, and their step rates.
    Returns its line."""
    import flowcontrast_b200 as fb
    from flowcontrast_b200 import build
    build.build()
    ctx = fb.Context(0)
    dom = fb.make_domain(W["lx"], W["ly"], W["lz"], radius=W["R"], cx=W["cx"], cy=W["cy"])
    cells = W["lx"] * W["ly"] * W["lz"]
    out = {}
    for re in (500.0, 2000.0, 5300.0):
        ub = re * W["nu"] / (2 * W["R"])
        g = (2 * (W["re_tau"] * W["nu"] / W["R"]) ** 2 / W["R"]) if re >= 5000 else 8 * W["nu"] * ub / W["R"] ** 2
        prm = fb.Params.make(tblend=W["tblend"], pin=0.0, nu=W["nu"], d1=W["d1"], delta=1,
                             blend=W["blend"], monitor_every=50, force=(0.0, 0.0, -g))
        f = {}
        for name, dt in (("f64", fb.F64), ("f32", fb.F32), ("f16", fb.F16)):
            s = fb.Solve(ctx, dom, prm, dt)
            s.init_poiseuille(2 * ub, noise=1e-3, modes=4, mode_amp=0.05, seed=W["seed"])
            s.step(200)
            s.sync()
            f[name] = s.get_fields(np.float64)
            s.close()
        ref = f["f64"]
        row = {}
        for name in ("f32", "f16"):
            row[name] = {"rel_l2_u": float(np.linalg.norm(f[name][1:] - ref[1:]) / np.linalg.norm(ref[1:])),
                         "rel_l2_p": float(np.linalg.norm(f[name][0] - ref[0]) / np.linalg.norm(ref[0])),
                         "rel_l2_rho": float(np.linalg.norm(f[name][0] - ref[0]) / np.linalg.norm(1.0 + ref[0]))}
        out[f"re{int(re)}"] = row
    rates = {}
    for name, dt in (("f64", fb.F64), ("f32", fb.F32), ("f16", fb.F16)):
        s = fb.Solve(ctx, dom, fb.Params.make(tblend=W["tblend"], pin=0.0, nu=W["nu"], d1=W["d1"],
                                              blend=W["blend"], monitor_every=50,
                                              force=(0.0, 0.0, -physics()[2])), dt)
        s.init_poiseuille(physics()[1], noise=1e-3, modes=4, mode_amp=0.05, seed=W["seed"])
        s.step(args.warmup)
        s.sync()
        s.set_timing(True)
        s.kernel_time()
        s.step(args.steps)
        s.sync()
        ms, n = s.kernel_time()
        rates[name] = cells / (ms / n * 1e-3) / 1e6
        s.close()
    ctx.close()
    line = {"metric": "error vs FP64 after 200 steps and MLUPS per storage type", "value": rates["f16"],
            "unit": "MLUPS", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cells / rates["f16"] / 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f16 storage, f32 arithmetic", "data": "synthetic",
            "config": {"workload": "512x128x128 pipe, R=63, tblend 0.02, d1 2, order 4, Re 500/2000/5300"},
            "errors_200_steps": out, "mlups": rates, "f16_gain_vs_f32": rates["f16"] / rates["f32"]}
    return line


def run_mixed(args):
    print(json.dumps(mixed_line(args)), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--e2e-reps", type=int, default=3)
    ap.add_argument("--workload", default="plain", choices=["plain", "ensemble", "served", "mixed"])
    ap.add_argument("--no-extras", action="store_true",
                    help="default line: skip the ensemble and precision measurements after it")
    ap.add_argument("--dtype", default="f32", choices=["f32", "f64", "f16"],
                    help="plain workload: storage type of the solve (the default line is FP32)")
    ap.add_argument("--requests", type=int, default=1000, help="served workload: request count")
    ap.add_argument("--rate", type=float, default=200.0,
                    help="served workload: Poisson arrival rate (requests per second)")
    ap.add_argument("--ensemble-dtype", default="f32", choices=["f32", "f16"],
                    help="ensemble workload: storage type of the batched members")
    ap.add_argument("--served-dtype", default="mixed", choices=["mixed", "f32"],
                    help="served workload: storage types of the requests (FP32/FP16 50/50, or FP32)")
    ap.add_argument("--tuning-out", default=None, help="ensemble workload: write the tuned tiling table here")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.workload != "plain":
            if args.impl == "reference":
                if rank == 0:
                    print(json.dumps({"impl": "reference", "unavailable":
                                      "the reference runs one pipe per process; it has no "
                                      "batched, served or reduced-precision form"}), flush=True)
                return 0
            if world > 1:
                raise SystemExit("--workload other than plain runs on one GPU")
            return {"ensemble": run_ensemble, "served": run_served, "mixed": run_mixed}[args.workload](args)
        if args.impl == "reference":
            return run_reference_arm(args, rank, world, local)
        return run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
