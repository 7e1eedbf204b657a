"""Host-side FP64 post-processing of swarm and committor runs.

* ``fit_nucleation_rate``: the fit of the nucleated fraction to
  1 - exp(-k (t - t0)) used by the reference workflow
  (Jupyter/GASP_rates.ipynb:162-193: fit from the last zero entry of the
  fraction curve, p0 = (8e-5, 1000), rate per site = k / L^2).
* ``bootstrap_rate``: bootstrap standard errors of (k, t0) obtained by
  resampling replicas (or blocks of replicas) from their first-passage
  sweeps.
* ``committor_errbar``: the reference's bootstrap error bar on pB
  (src/bootstrap.c:6-65) through the C ABI.
"""
from __future__ import annotations

import numpy as np


def _fitfunc(t, rate, t_ind):
    return 1.0 - np.exp(-rate * (t - t_ind))


def fit_nucleation_rate(frac, mag_output_int, L=None, p0=(8e-5, 1000.0)):
    """Returns (k, t0, k_per_site) from a nucleated-fraction curve sampled every
    mag_output_int sweeps.  k is 0 when nothing nucleated (frac[-1] < 1/n is
    the reference's test; here: no non-zero entry)."""
    from scipy.optimize import curve_fit

    frac = np.asarray(frac, np.float64)
    xdata = np.arange(frac.size, dtype=np.float64) * mag_output_int
    nz = np.argwhere(frac)
    if nz.size == 0:
        return 0.0, float("nan"), 0.0
    si = max(int(nz[0][0]) - 1, 0)
    popt, _ = curve_fit(_fitfunc, xdata[si:], frac[si:], p0=list(p0), maxfev=20000)
    k, t0 = float(popt[0]), float(popt[1])
    return k, t0, (k / (L * L) if L else float("nan"))


def fraction_from_first_passage(first_passage, tot_nsweeps, mag_output_int):
    """Nucleated fraction at each check from per-replica first-passage sweeps
    (-1: never crossed)."""
    fp = np.asarray(first_passage)
    t = np.arange(tot_nsweeps // mag_output_int) * mag_output_int
    crossed = np.sort(fp[fp >= 0])
    return np.searchsorted(crossed, t, side="right") / max(fp.size, 1)


def bootstrap_rate(first_passage, tot_nsweeps, mag_output_int, nboot=200, block=1, seed=0,
                   L=None):
    """Bootstrap (k, t0) by resampling replicas in blocks of ``block``
    consecutive replicas (use 32 for modes whose 32 replicas of a warp share
    their site sequence).  Returns dict(k, t0, k_se, t0_se, samples)."""
    fp = np.asarray(first_passage)
    n = fp.size // block
    fpb = fp[:n * block].reshape(n, block)
    k, t0, _ = fit_nucleation_rate(
        fraction_from_first_passage(fp, tot_nsweeps, mag_output_int), mag_output_int)
    rng = np.random.default_rng(seed)
    ks, ts = [], []
    for _ in range(nboot):
        idx = rng.integers(0, n, n)
        f = fraction_from_first_passage(fpb[idx].reshape(-1), tot_nsweeps, mag_output_int)
        try:
            kk, tt, _ = fit_nucleation_rate(f, mag_output_int)
        except RuntimeError:
            continue
        ks.append(kk)
        ts.append(tt)
    ks, ts = np.array(ks), np.array(ts)
    return {"k": k, "t0": t0, "k_se": float(ks.std(ddof=1)), "t0_se": float(ts.std(ddof=1)),
            "k_per_site": (k / (L * L) if L else float("nan")), "samples": int(ks.size)}


def committor_errbar(fates_block):
    """The reference's bootstrap error bar (libc rand(), m = n resamples,
    population standard deviation) for one input block of fates."""
    from ._native import lib

    f = np.ascontiguousarray(fates_block, np.int32)
    return float(lib().gasp_bootstrap_errbar(f.size, f.size, f))
