"""Builds the native library libfslbm.so (sm_100a) and the drop-in executable fslbm_pipe in
place, next to this file. Rebuilds only when a source is newer than its output."""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfslbm.so")
CLI = os.path.join(HERE, "fslbm_pipe")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xptxas", "-warn-spills", "-I" + os.path.join(ROOT, "include")]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + [
        p for p in glob.glob(os.path.join(CSRC, "*.cpp")) if not p.endswith("pipe_main.cpp")])


def _deps():
    return (glob.glob(os.path.join(CSRC, "*")) + [os.path.join(ROOT, "include", "fslbm.h"),
                                                 os.path.abspath(__file__)])


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError(f"build failed: {' '.join(cmd[:3])} ...")
    if verbose and r.stdout.strip():
        print(r.stdout)


def build(verbose=False, force=False):
    deps = _deps()
    if force or _stale(LIB, deps):
        _run(["nvcc", *NVCC_FLAGS, "-shared", "-o", LIB, *_sources()], verbose)
    main = os.path.join(CSRC, "pipe_main.cpp")
    if os.path.exists(main) and (force or _stale(CLI, deps + [LIB])):
        _run(["nvcc", *NVCC_FLAGS, "-o", CLI, main, "-L" + HERE, "-lfslbm",
              "-Xlinker", "-rpath=$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
