"""fslbm_pipe on the GPU: the reference's file set, equality with the library run, restart.

A pipe.m geometry (20-cell diameter, 40 core planes, 10 buffer planes each end: a 40x40x60
reference box) runs 1000 steps from the initphys start with the reference's intervals (monitor
every 50, dumps every 500) and a backup at step 1000:
  - every output file exists with the reference's line count and format;
  - the backup state equals the same solve run through the library (bit for bit);
  - qp.txt holds the library's monitor records as "%e" text;
  - a run restarted from a step-500 backup continues it: after 500 more steps u, v, w agree
    with the uninterrupted run to 1e-5 relative (the restart does not carry the gauge p2 of
    the step-500 monitor, as in the reference, so p differs by a near-uniform offset).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from test_cli import CLI, SMALL, write_inputs

pytestmark = pytest.mark.gpu


def run(args, cwd):
    r = subprocess.run([CLI, *args], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r


def lines(d, name):
    with open(os.path.join(d, name)) as f:
        return f.read().splitlines()


def library_run(fb, ctx, d, mask3d, steps):
    lz, ly, lx = mask3d.shape
    core = fb.ref_mask_to_core(mask3d, 10)
    dom = fb.make_domain(lx, ly, lz - 20, mask=core, radius=10.0, buffer_depth=10)
    prm = fb.read_param_txt(os.path.join(d, "param.txt"))     # FP32-rounded as the CLI reads it
    prm.monitor_every = 50
    s = fb.Solve(ctx, dom, prm, fb.F32)
    f = np.zeros((4, lz, ly, lx), np.float32)
    z = np.arange(lz, dtype=np.float32)
    f[0] = (np.float32(np.float32(0.003) * (np.float32(lz - 10) - z)) / np.float32(lz - 20))[:, None, None]
    s.set_fields_ref(f)
    s.step(steps)
    s.sync()
    out = s.get_fields_ref()
    log = s.monitor_log()
    s.close()
    return out, log


def test_cli_files_and_library_equality(built, ctx, tmp_path):
    fb = built
    d = str(tmp_path)
    mask = write_inputs(fb, d)
    run(SMALL + ["--steps", "1000", "--backup", "1000", "--quiet"], d)
    nyz, nxy = 40 * 60, 40 * 40
    qp = lines(d, "qp.txt")
    assert len(qp) == 20 and all(len(l.split()) == 6 for l in qp)
    for name in ("p.txt", "ux.txt", "uy.txt", "uz.txt", "IO.txt", "_p.txt", "_ux.txt", "_uy.txt",
                 "_uz.txt", "_p2.txt", "_ux2.txt", "_uy2.txt", "_uz2.txt", "_uxy2.txt",
                 "_uxz2.txt", "_uyz2.txt", "_pii.txt", "_uyz2ii.txt"):
        assert len(lines(d, name)) == nyz, name
    for name in ("p1.txt", "ux1.txt", "uy1.txt", "uz1.txt"):
        assert len(lines(d, name)) == nxy, name
    assert lines(d, "_av.txt") == ["2 1"]            # delta 1: the fluctuation sums restart
    assert lines(d, "_avii.txt") == ["2 1"]
    assert lines(d, "qpii.txt") == qp
    io = np.array([int(v) for v in lines(d, "IO.txt")]).reshape(60, 40)
    assert np.array_equal(io, mask[:, :, 20])
    raw = [np.fromfile(os.path.join(d, n), np.float32).reshape(60, 40, 40)
           for n in ("p3Dii", "ux3Dii", "uy3Dii", "uz3Dii")]
    want, log = library_run(fb, ctx, d, mask, 1000)
    for k in range(4):
        assert np.array_equal(raw[k], want[k]), k
    assert [float(v) for v in qp[-1].split()] == [float(f"{log[-1][k]:e}") for k in
                                                  ("q1", "q2", "p1", "p2", "f", "sample")]
    uz = np.array([float(v) for v in lines(d, "uz.txt")])
    assert np.allclose(uz, want[3][:, :, 20].ravel(), rtol=1e-5, atol=1e-12)


def test_cli_restart_continues(built, tmp_path):
    fb = built
    a, b = str(tmp_path / "a"), str(tmp_path / "b")
    os.makedirs(a)
    write_inputs(fb, a)
    shutil.copytree(a, b)
    run(SMALL + ["--steps", "1000", "--backup", "1000", "--quiet"], a)
    run(SMALL + ["--steps", "500", "--backup", "500", "--quiet"], b)
    run(SMALL + ["--steps", "500", "--backup", "500", "--quiet", "--init", "restart"], b)
    qa, qb = lines(a, "qp.txt"), lines(b, "qp.txt")
    assert len(qb) == 20 and qb[:10] == qa[:10]
    fa = [np.fromfile(os.path.join(a, n), np.float32) for n in ("ux3Dii", "uy3Dii", "uz3Dii")]
    fbk = [np.fromfile(os.path.join(b, n), np.float32) for n in ("ux3Dii", "uy3Dii", "uz3Dii")]
    u_a, u_b = np.concatenate(fa).astype(np.float64), np.concatenate(fbk).astype(np.float64)
    assert np.linalg.norm(u_a - u_b) <= 1e-5 * np.linalg.norm(u_a)
    # statistics continue from the backup: the same sample counts as the straight run
    assert lines(b, "_av.txt") == lines(a, "_av.txt")


STAT_FILES = ("_p.txt", "_ux.txt", "_uy.txt", "_uz.txt", "_p2.txt", "_ux2.txt", "_uy2.txt",
              "_uz2.txt", "_uxy2.txt", "_uxz2.txt", "_uyz2.txt")


def test_cli_live_param_reload_and_statistics(built, ctx, tmp_path):
    """Live param.txt reload (FSLBM.cu:667-690) with the delta reset policy, end to end.

    param.txt is a named pipe, so each of the CLI's reads (at start-up and before the
    statistics of every 500-step dump) blocks until this test hands it the next parameter set:
    start delta 2, nu 0.02; dump 500: nu 0.03 (delta 2); dump 1000: delta 1 (the fluctuation
    sums restart); dump 1500: delta 0 (everything restarts); dump 2000: delta 2, tblend 0.8.
    After each dump the statistics files and _av.txt are captured and compared with the same
    schedule run through the library (fslbm_solve_set_params, then fslbm_stats_sample), whose
    statistics the device-statistics tests pin to the oracle: the counts follow the policy
    and every value equals the library's "%e" text. The printed dtddy follows the new nu.
    """
    import threading

    fb = built
    d = str(tmp_path)
    mask = write_inputs(fb, d)
    base = fb.read_param_txt(os.path.join(d, "param.txt"))
    os.remove(os.path.join(d, "param.txt"))
    sched = [dict(nu=0.02, delta=2), dict(nu=0.03, delta=2), dict(nu=0.03, delta=1),
             dict(nu=0.03, delta=0), dict(nu=0.03, delta=2, tblend=0.8)]
    texts = []
    for k, upd in enumerate(sched):
        p = fb.Params.from_buffer_copy(base)
        for key, val in upd.items():
            setattr(p, key, val)
        path = os.path.join(d, f"param{k}.tmp")
        fb.write_param_txt(path, p)
        texts.append(open(path).read())
    fifo = os.path.join(d, "param.txt")
    os.mkfifo(fifo)
    proc = subprocess.Popen([CLI, *SMALL, "--steps", "2000"], cwd=d, stdout=subprocess.PIPE,
                            stderr=subprocess.PIPE, text=True)
    snaps = []

    def snapshot():
        snaps.append({n: lines(d, n) for n in STAT_FILES + ("_av.txt",)})

    def qp_lines():
        try:
            with open(os.path.join(d, "qp.txt")) as fh:
                return fh.read().count("\n")
        except OSError:
            return 0

    def feeder():
        # Hands texts[k] to the k-th read (start-up, then the dumps at steps 500k). The next
        # open waits until qp.txt holds the monitor record of step 500k + 50, which the CLI
        # writes after it closed param.txt, so two parameter sets never share one read.
        import errno
        import time
        for k, text in enumerate(texts):
            fd = None
            t0 = time.time()
            while fd is None and proc.poll() is None and time.time() - t0 < 300:
                try:
                    fd = os.open(fifo, os.O_WRONLY | os.O_NONBLOCK)
                except OSError as e:
                    if e.errno != errno.ENXIO:
                        raise
                    time.sleep(0.001)
            if fd is None:
                return
            if k >= 2:
                snapshot()                # the previous dump's files are complete
            os.set_blocking(fd, True)
            os.write(fd, text.encode())
            os.close(fd)
            if k + 1 < len(texts):
                while qp_lines() < 10 * k + 1 and proc.poll() is None and time.time() - t0 < 300:
                    time.sleep(0.001)

    th = threading.Thread(target=feeder, daemon=True)
    th.start()
    try:
        out, err = proc.communicate(timeout=600)
    finally:
        if proc.poll() is None:
            proc.kill()
    th.join(timeout=10)
    assert proc.returncode == 0, err
    snapshot()
    assert len(snaps) == 4
    assert [s["_av.txt"] for s in snaps] == [["1 1"], ["2 1"], ["1 1"], ["2 2"]]
    dtddy = [float(l.split("dtddy: ")[1].split(",")[0]) for l in out.splitlines()
             if l.startswith("time step:")]
    assert len(dtddy) == 40
    assert abs(dtddy[9] - (0.02 - 0.16666666)) < 1e-6 and abs(dtddy[10] - (0.03 - 0.16666666)) < 1e-6

    # the same schedule through the library
    core = fb.ref_mask_to_core(mask, 10)
    lz, ly, lx = mask.shape
    dom = fb.make_domain(lx, ly, lz - 20, mask=core, radius=10.0, buffer_depth=10)
    prms = []
    for k in range(len(texts)):
        p = fb.read_param_txt(os.path.join(d, f"param{k}.tmp"))
        p.monitor_every = 50
        prms.append(p)
    s = fb.Solve(ctx, dom, prms[0], fb.F32)
    f = np.zeros((4, lz, ly, lx), np.float32)
    z = np.arange(lz, dtype=np.float32)
    f[0] = (np.float32(np.float32(0.003) * (np.float32(lz - 10) - z)) / np.float32(lz - 20))[:, None, None]
    s.set_fields_ref(f)
    try:
        for k in range(4):
            s.step(500)
            s.set_params(prms[k + 1])
            s.stats_sample()
            means, cnt, cnt2 = s.stats_get()
            assert snaps[k]["_av.txt"] == [f"{cnt} {cnt2}"]
            for j, name in enumerate(STAT_FILES):
                got = [float(v) for v in snaps[k][name]]
                assert got == [float(f"{v:e}") for v in means[j]], (k, name)
        # the fluctuation statistics are not trivially zero
        assert np.abs(means[4:8]).max() > 0
    finally:
        s.close()
