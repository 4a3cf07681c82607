"""Golden cases: small pipes in the reference layout, run by the reference's own kernels.

Each case is the pipe.m geometry (pipe.m:36-60) scaled down: a circle of diameter `lx0`
cells padded by `d` wall cells in x and y, `l0` fluid planes between `d` buffer planes at
each streamwise end. Inputs are regenerated from the seed by `inputs()` (numpy PCG64, stable
across machines), so the fixture files hold only the reference's outputs.

Initial state: stored streamwise velocity w = -u0 (1 - r^2/R^2) plus uniform noise on all
velocity components and on p; wall cells are zero; buffer planes hold the bcond copies of
the wrapped core planes with the +-pin pressure jump (FSLBM.cu:291-301).

`monitor` is the monitor period of the run (0: none, so the gauge p2 stays 0; 50: the
reference's, so step 51 subtracts the p2 of step 50, FSLBM.cu:628-647). `race_free` runs the
reference's kernels on snapshot reads (each slab loop and bcond sample the field as it was
before them), which removes their intra-launch read/write races when blend != 0 or p2 != 0
and leaves the arithmetic as compiled; cases with blend 0 and no gauge run as shipped.
"""
import numpy as np

D = 10  # buffer depth and wall padding of pipe.m (pipe.m:38), and d2 of FSLBM.cu:514

CASES = {
    # pipe.m's own parameters (pipe.m:68): tblend 1, pin 0.003, nu 0.004006, d1 2, blend 0
    "pipe_m_r6": dict(lx0=12, l0=16, seed=11, u0=0.05, noise=0.005, pnoise=1e-3,
                      prm=dict(tblend=1.0, pin=0.003, nu=0.004006, d1=2, blend=0.0),
                      steps=(1, 30)),
    # the paper's smooth-pipe regime: small time-step blend, nu about 0.011 (PDF Table 1)
    "paper_tb002": dict(lx0=12, l0=24, seed=12, u0=0.3, noise=0.03, pnoise=2e-3,
                        prm=dict(tblend=0.02, pin=0.0193, nu=0.0111, d1=2, blend=0.0),
                        steps=(1, 40)),
    # unit corrective stride
    "d1_one": dict(lx0=12, l0=16, seed=13, u0=0.04, noise=0.004, pnoise=1e-3,
                   prm=dict(tblend=0.5, pin=0.002, nu=0.12, d1=1, blend=0.0),
                   steps=(1, 25)),
    # the benchmark's setting: order-4 corrector (blend 1) in the paper's regime
    "paper_blend1": dict(lx0=12, l0=24, seed=14, u0=0.3, noise=0.03, pnoise=2e-3,
                         prm=dict(tblend=0.02, pin=0.0193, nu=0.0111, d1=2, blend=1.0),
                         steps=(1, 40), race_free=1),
    # order-4 corrector across the first monitor: step 51 applies the gauge p2 of step 50
    "gauge_blend1": dict(lx0=12, l0=16, seed=15, u0=0.05, noise=0.005, pnoise=1e-3,
                         prm=dict(tblend=0.6, pin=0.003, nu=0.02, d1=2, blend=1.0),
                         steps=(50, 51, 56), monitor=50, race_free=1),
}


def pipe_m_mask(lx0, l0, d=D):
    """pipe.m:36-60 in numpy: shape (lz, ly, lx), 0 fluid / 1 buffer / 125 wall."""
    lx, lz = lx0 + 2 * d, l0 + 2 * d
    o = lx0 / 2.0
    i = np.arange(1, lx0 + 1, dtype=np.float64)
    inside = ((i[None, :] - o) ** 2 + (i[:, None] - o) ** 2) <= o * o   # [j, i]
    plane = np.full((lx, lx), 125, np.uint8)
    plane[d:d + lx0, d:d + lx0] = np.where(inside, 0, 125)
    io = np.repeat(plane[None], lz, axis=0)
    buf = np.where(plane == 0, 1, 125).astype(np.uint8)
    io[:d] = buf
    io[lz - d:] = buf
    return io


def core_state(mask2d, L, seed, u0, noise, pnoise, dtype=np.float32):
    """Seeded core fields (4, L, ly, lx) on a cross-section mask (0 fluid / 125 wall)."""
    ly, lx = mask2d.shape
    rng = np.random.default_rng(seed)
    fluid = mask2d == 0
    ys, xs = np.nonzero(fluid)
    cy, cx = ys.mean(), xs.mean()
    r2 = ((np.arange(ly)[:, None] - cy) ** 2 + (np.arange(lx)[None, :] - cx) ** 2)
    R2 = r2[fluid].max() + 1.0
    prof = np.where(fluid, 1.0 - r2 / R2, 0.0)
    f = np.zeros((4, L, ly, lx), np.float64)
    f[0] = pnoise * rng.uniform(-1, 1, (L, ly, lx))
    f[1] = noise * rng.uniform(-1, 1, (L, ly, lx))
    f[2] = noise * rng.uniform(-1, 1, (L, ly, lx))
    f[3] = -u0 * prof[None] + noise * rng.uniform(-1, 1, (L, ly, lx))
    f *= fluid[None, None]
    return f.astype(dtype)


def pad_reference(core, mask2d, pin, d=D):
    """Core (4,L,ly,lx) -> reference layout (4,L+2d,ly,lx) with bcond-consistent buffers."""
    _, L, ly, lx = core.shape
    out = np.zeros((4, L + 2 * d, ly, lx), core.dtype)
    out[:, d:d + L] = core
    out[:, :d] = core[:, L - d:]
    out[:, d + L:] = core[:, :d]
    nonwall = (mask2d != 125)
    out[0, :d] += (core.dtype.type(pin) * nonwall)
    out[0, d + L:] -= (core.dtype.type(pin) * nonwall)
    return out


def inputs(name):
    """(io, reference-layout float32 fields, params) of a golden case."""
    c = CASES[name]
    io = pipe_m_mask(c["lx0"], c["l0"])
    mask2d = np.where(io[D] == 125, 125, 0).astype(np.uint8)
    core = core_state(mask2d, c["l0"], c["seed"], c["u0"], c["noise"], c["pnoise"])
    ref = pad_reference(core, mask2d, np.float32(c["prm"]["pin"]))
    return io, ref, dict(c["prm"], d2=D)


def nonwall_index(io):
    return np.flatnonzero(io.ravel() != 125)
