"""Radial profiles of the full-volume pipe statistics (the post-processing the reference does in
MATLAB with avgFields.m and avgRstress.m, here on the FP64 sums of fslbm_profile_sample).

profile_get() returns, per cross-section column, sums over the streamwise planes and over the
samples of p, u, v, w, uu, vv, ww, uv, uw, vw. Column means over z and time give the mean
fields and, with the column means removed, the Reynolds stresses; these are rotated to
cylindrical components about the pipe axis and averaged in radial bins of the fluid columns.
Velocities are returned in the physical sign (the stored velocity is the negated one).
"""
import numpy as np


def radial_profiles(sums, nsamples, L, cx, cy, R, mask=None, nbins=16):
    """sums: (10, ly, lx) from Solve.profile_get(); L streamwise planes; centre (cx, cy),
    radius R; mask (ly, lx) 0 = fluid (default: the circle). Returns a dict of arrays over the
    radial bins: r (bin centre / R), w (mean axial velocity), p, and the stresses uu_r, uu_t,
    ww, uw_r (<u_r' w'>), plus counts (columns per bin)."""
    s = np.asarray(sums, np.float64) / float(nsamples * L)
    p, u, v, w, uu, vv, ww, uv, uw, vw = s
    ly, lx = p.shape
    y, x = np.mgrid[0:ly, 0:lx]
    dx, dy = x - cx, y - cy
    r = np.hypot(dx, dy)
    fluid = (r <= R) if mask is None else (np.asarray(mask) == 0)
    # fluctuations about the column means (over z and time)
    cuu = uu - u * u
    cvv = vv - v * v
    cww = ww - w * w
    cuv = uv - u * v
    cuw = uw - u * w
    cvw = vw - v * w
    with np.errstate(invalid="ignore", divide="ignore"):
        c = np.where(r > 0, dx / r, 1.0)
        sn = np.where(r > 0, dy / r, 0.0)
    # second moments keep their sign under the stored (negated) velocity convention
    urr = c * c * cuu + 2 * c * sn * cuv + sn * sn * cvv
    utt = sn * sn * cuu - 2 * c * sn * cuv + c * c * cvv
    urw = c * cuw + sn * cvw
    edges = np.linspace(0.0, R, nbins + 1)
    idx = np.clip(np.digitize(r, edges) - 1, 0, nbins - 1)
    out = {k: np.zeros(nbins) for k in ("w", "p", "uu_r", "uu_t", "ww", "uw_r")}
    counts = np.zeros(nbins)
    for b in range(nbins):
        sel = fluid & (idx == b)
        counts[b] = sel.sum()
        if counts[b] == 0:
            continue
        out["w"][b] = -w[sel].mean()
        out["p"][b] = p[sel].mean()
        out["uu_r"][b] = urr[sel].mean()
        out["uu_t"][b] = utt[sel].mean()
        out["ww"][b] = cww[sel].mean()
        out["uw_r"][b] = urw[sel].mean()
    out["r"] = 0.5 * (edges[:-1] + edges[1:]) / R
    out["counts"] = counts
    return out


def profile_error(a, b, key, counts=None):
    """Relative L2 difference of profile `key` (a against reference b), weighted by the
    columns per bin."""
    wgt = np.ones_like(b[key]) if counts is None else counts
    num = np.sqrt(np.sum(wgt * (a[key] - b[key]) ** 2))
    den = np.sqrt(np.sum(wgt * b[key] ** 2))
    return float(num / den) if den > 0 else float(num)
