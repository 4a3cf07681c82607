"""Generate the golden fixtures by running the reference's own kernels on a GPU.

Runs on a machine with a GPU, after `make -C oracle ref` has built oracle/_ref/libfslbm_ref.so
(the reference's FSLBMcalc/shiftback/bcond compiled for sm_100a from its own source). For each
case in ref_cases.CASES and each step count, it advances the seeded initial state and stores
the non-wall cells of the resulting reference-layout fields as float32:

    python tests/golden/make_ref_fixtures.py --out tests/golden [--only name,name]

Cases with `race_free` run the kernels on snapshot reads and cases with `monitor` apply the
reference's gauge (see ref_cases.py).

With --time it also times the reference's step loop on the demo grid (pipe.m, 120x120x320)
and on a 128x128x(512+20) pipe, and writes ref_kernel_timing.json (context numbers only).
"""
import argparse
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ref_cases  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(HERE))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libfslbm_ref.so")


def load():
    lib = ctypes.CDLL(REF_LIB)
    u8 = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
    f32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    i = ctypes.c_int
    lib.ref_run2.argtypes = [u8, i, i, i, i, f32, f32, f32, i, i, i,
                             ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_uint), f32]
    return lib


def run(lib, io, fields, prm, nsteps, monitor=0, race_free=0):
    """Returns (fields, device ms, p2 of each monitor)."""
    lz, ly, lx = io.shape
    p = np.array([prm["tblend"], prm["pin"], prm["nu"], prm["d1"], prm["blend"]], np.float32)
    src = np.ascontiguousarray(fields, np.float32)
    out = np.empty_like(src)
    p2 = np.zeros(max(1, nsteps // monitor if monitor else 0), np.float32)
    ms, oob = ctypes.c_float(0), ctypes.c_uint(0)
    rc = lib.ref_run2(np.ascontiguousarray(io), lx, ly, lz, prm["d2"], p, src.ravel(), out.ravel(),
                      nsteps, monitor, race_free, ctypes.byref(ms), ctypes.byref(oob), p2)
    if rc != 0:
        raise RuntimeError(f"ref_run2 failed: {rc}")
    if oob.value:
        raise RuntimeError(f"reference kernels wrote {oob.value} cells outside the box")
    return out, ms.value, p2[:nsteps // monitor if monitor else 0]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--time", action="store_true")
    ap.add_argument("--only", default="", help="comma-separated case names (default: all)")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    lib = load()
    only = [x for x in a.only.split(",") if x]
    for name, c in ref_cases.CASES.items():
        if only and name not in only:
            continue
        io, ref, prm = ref_cases.inputs(name)
        keep = ref_cases.nonwall_index(io)
        arrays = {}
        for n in c["steps"]:
            out, _, p2 = run(lib, io, ref, prm, n, c.get("monitor", 0), c.get("race_free", 0))
            arrays[f"step{n}"] = out.reshape(4, -1)[:, keep]
            if len(p2):
                arrays[f"p2_step{n}"] = p2
        np.savez_compressed(os.path.join(a.out, f"ref_{name}.npz"), **arrays)
        print(name, {k: v.shape for k, v in arrays.items()})
    if a.time:
        res = {}
        for label, (lx0, l0) in {"pipe_m_demo_120x120x320": (100, 300),
                                 "pipe_128x128x532": (108, 512)}.items():
            io = ref_cases.pipe_m_mask(lx0, l0)
            mask2d = np.where(io[ref_cases.D] == 125, 125, 0).astype(np.uint8)
            core = ref_cases.core_state(mask2d, l0, 5, 0.05, 0.005, 1e-3)
            f = ref_cases.pad_reference(core, mask2d, np.float32(0.003))
            prm = dict(tblend=1.0, pin=0.003, nu=0.004006, d1=2, blend=0.0, d2=ref_cases.D)
            run(lib, io, f, prm, 3)                      # warm-up
            steps = 40
            _, ms, _ = run(lib, io, f, prm, steps)
            cells = io.size
            res[label] = dict(cells=int(cells), steps=steps, ms=ms,
                              mlups=cells * steps / (ms * 1e-3) / 1e6)
            print(label, res[label])
        with open(os.path.join(a.out, "ref_kernel_timing.json"), "w") as fh:
            json.dump(res, fh, indent=1)


if __name__ == "__main__":
    main()
