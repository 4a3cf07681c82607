"""Seeded pipe-solve workloads: the mixed-size ensemble and the served request stream.

Both are sets of independent periodic pipes (streamwise length ``L`` = the reference's x
extent, square cross-section ``n x n`` with a centred circular wall of radius ``n/2 - 1``),
driven by the constant body force of laminar Poiseuille flow at the member's Reynolds number
(``g = 8 nu u_b / R^2``, bulk velocity ``u_b``) and started from Poiseuille flow plus seeded
noise and random-phase streamwise/azimuthal modes. The solver parameters are the reference's
paper regime (tblend 0.02, d1 2, order-4 corrector blend, FSLBM.cu:499-510 param.txt
values), with the viscosity set by ``Re = 2 R u_b / nu``.
"""
import math
from dataclasses import dataclass

import numpy as np

U_BULK = 0.1          # lattice bulk velocity of every member
TBLEND = 0.02
D1 = 2


@dataclass
class PipeSpec:
    L: int            # streamwise planes (periodic)
    n: int            # cross-section width = height
    re: float         # bulk Reynolds number 2 R u_b / nu
    seed: int
    steps: int = 0
    dtype: int = 1    # FSLBM_F32
    arrival: float = 0.0

    @property
    def radius(self):
        return self.n / 2.0 - 1.0

    @property
    def nu(self):
        return 2.0 * self.radius * U_BULK / self.re

    @property
    def force_z(self):
        return -8.0 * self.nu * U_BULK / self.radius ** 2

    @property
    def cells(self):
        return self.L * self.n * self.n

    def domain(self, fb):
        c = (self.n - 1) / 2.0
        return fb.make_domain(self.n, self.n, self.L, radius=self.radius, cx=c, cy=c)

    def params(self, fb, monitor_every=50):
        return fb.Params.make(tblend=TBLEND, pin=0.0, nu=self.nu, d1=D1, delta=1, blend=1.0,
                              monitor_every=monitor_every, force=(0.0, 0.0, self.force_z))

    def initial_fields(self, fb):
        """(4, L, n, n) float64: Poiseuille (u_max = 2 u_b), noise 1e-3 u_max, 4 modes at 5 %
        of u_max (10 % of u_bulk)."""
        return fb.init_poiseuille(self.domain(fb), 2 * U_BULK, noise=1e-3, modes=4,
                                  mode_amp=0.05, seed=self.seed)

    def as_dict(self):
        return {"L": self.L, "n": self.n, "re": round(self.re, 3), "seed": self.seed,
                "steps": self.steps, "dtype": self.dtype, "arrival": self.arrival}


def ensemble(count=64, seed=20261203, steps=2000):
    """Mixed-size ensemble: L uniform in [32, 256], n uniform in [24, 96], Re log-uniform in
    [50, 3000], FP32, the same step count for all members."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        L = int(rng.integers(32, 257))
        n = int(rng.integers(24, 97))
        re = float(math.exp(rng.uniform(math.log(50.0), math.log(3000.0))))
        out.append(PipeSpec(L=L, n=n, re=re, seed=seed * 1000 + i, steps=steps))
    return out


def request_stream(count, rate=200.0, seed=20261204, mixed_fraction=0.5):
    """Served solves: Poisson arrivals at ``rate`` per second; grid cells log-uniform between
    32^3 and 256 x 96 x 96 (the cross-section n in [24, 96] log-uniform, L from the cell
    count, clamped to [32, 256]); step counts uniform in [200, 5000]; Re log-uniform in
    [50, 5000]; dtype FP32 or mixed (FP16 storage) with probability ``mixed_fraction``."""
    rng = np.random.default_rng(seed)
    t = 0.0
    lo, hi = math.log(32.0 ** 3), math.log(256.0 * 96 * 96)
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        cells = math.exp(rng.uniform(lo, hi))
        n = int(round(math.exp(rng.uniform(math.log(24.0), math.log(96.0)))))
        L = int(min(256, max(32, round(cells / (n * n)))))
        steps = int(rng.integers(200, 5001))
        re = float(math.exp(rng.uniform(math.log(50.0), math.log(5000.0))))
        dtype = 2 if rng.uniform() < mixed_fraction else 1
        out.append(PipeSpec(L=L, n=n, re=re, seed=seed * 1000 + i, steps=steps, dtype=dtype,
                            arrival=t))
    return out


def rough_pipe_mask(n, L, radius, amplitude=1.5, modes=3, seed=1):
    """Seeded rough pipe (masks varying along z, one cross-section per plane), shape (L, n, n),
    0 fluid / 125 wall: a cell is fluid where its distance from the axis is below
    R(theta, z) = radius + amplitude * mean of `modes` sinusoids in theta (orders 3..) and z
    (periodic over L, wavenumbers 1..), with seeded phases. The box rim stays wall."""
    rng = np.random.default_rng(seed)
    c = (n - 1) / 2.0
    y, x = np.mgrid[0:n, 0:n]
    r = np.hypot(x - c, y - c)
    th = np.arctan2(y - c, x - c)
    out = np.empty((L, n, n), np.uint8)
    ph = rng.uniform(0, 2 * np.pi, size=(modes, 2))
    for z in range(L):
        bump = np.zeros_like(r)
        for m in range(modes):
            bump += np.sin((3 + m) * th + ph[m, 0]) * np.cos(2 * np.pi * (1 + m) * z / L + ph[m, 1])
        rw = radius + amplitude * bump / modes
        fluid = r <= rw
        fluid[0, :] = fluid[-1, :] = fluid[:, 0] = fluid[:, -1] = False
        out[z] = np.where(fluid, 0, 125)
    return out
