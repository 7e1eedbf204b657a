"""Production RNG mode (MWC64X) against the reference stream at the system's
own configurations, on a B200.

* The plain production swarm: L=64, 32768 replicas, beta=0.54, h=0.07,
  all-down start, magnetisation checked every 100 sweeps, up threshold 0.9
  -- 20 000 of its 50 000 sweeps (94 % of the replicas nucleate by then).
  The nucleated fraction is fitted to 1 - exp(-k (t - t0)) as the
  reference's notebook fits it (Jupyter/GASP_rates.ipynb:162-193), with
  bootstrap errors over replicas.
* Committor shooting of the seeded droplet grids (all -1, a centred +1
  disc of radius r ~ U[4, 12], 2 % random flips), 4096 shots per grid,
  dn -0.93, up 0.9, cap 20 000 sweeps.

The reference stream is bit-identical to the reference kernels
(test_parity_gpu.py), so it is the reference sample here.  Tolerances are 4
combined standard errors."""
import os
import sys

import numpy as np
import pytest

from conftest import REPO
from gpu_2dising_b200 import analysis, engine

pytestmark = pytest.mark.gpu

L, R, BETA, H, MAG, UP = 64, 32768, 0.54, 0.07, 100, 0.9
TOT = 20000
# Jupyter/GASP_rates.ipynb:178: one unseeded run of 1024 replicas on the
# reference's GPU path.  With ~600 nucleation events behind it, its own
# relative error is ~4 %; the band below is 15 % (about 4 of those errors).
PUBLISHED_K = 1.5032e-4


@pytest.fixture(scope="module", autouse=True)
def device():
    return engine.init_device(0)


def _swarm(kind, seed):
    dg = engine.DeviceGrids(L, R)
    rng = engine.RngStates(R, seed, kind=kind)
    fu = np.full(R, -1, np.int32)
    res, _, _, _ = engine.run_driver(dg, rng, BETA, H, TOT, MAG, TOT, itask=0, dn_thr=-0.9,
                                     up_thr=UP, first_up=fu)
    dg.close()
    rng.close()
    return res, fu


@pytest.fixture(scope="module")
def swarm_fits():
    out = {}
    for kind, seed in (("xorwow", 20240501), ("mwc64x", 20240502)):
        res, fu = _swarm(kind, seed)
        out[kind] = {"res": res, "fu": fu,
                     "fit": analysis.bootstrap_rate(fu, TOT, MAG, nboot=100, L=L)}
    return out


def test_swarm_rate_and_lag_agree_between_streams(swarm_fits):
    a, b = swarm_fits["xorwow"]["fit"], swarm_fits["mwc64x"]["fit"]
    assert a["samples"] >= 90 and b["samples"] >= 90
    assert abs(a["k"] - b["k"]) < 4 * np.hypot(a["k_se"], b["k_se"]), (a, b)
    assert abs(a["t0"] - b["t0"]) < 4 * np.hypot(a["t0_se"], b["t0_se"]), (a, b)


def test_swarm_rate_near_published_value(swarm_fits):
    for kind in ("xorwow", "mwc64x"):
        k = swarm_fits[kind]["fit"]["k"]
        assert abs(k - PUBLISHED_K) < 0.15 * PUBLISHED_K, (kind, k)


def test_swarm_fraction_curves_agree(swarm_fits):
    """At every check the two nucleated fractions differ by less than 4
    binomial errors (plus one replica)."""
    fa = np.asarray(swarm_fits["xorwow"]["res"], np.float64)
    fb = np.asarray(swarm_fits["mwc64x"]["res"], np.float64)
    se = np.sqrt(fa * (1 - fa) / R + fb * (1 - fb) / R)
    assert np.all(np.abs(fa - fb) < 4 * se + 1.0 / R)
    assert fa[-1] > 0.9 and fb[-1] > 0.9


@pytest.fixture(scope="module")
def committor_pb():
    sys.path.insert(0, REPO)
    import bench
    inputs, radii = bench.committor_inputs(16)
    shots = 4096
    out = {}
    for kind, seed in (("xorwow", 71), ("mwc64x", 72)):
        dg = engine.DeviceGrids(L, inputs.shape[0] * shots)
        dg.upload_inputs(inputs)
        rng = engine.RngStates(inputs.shape[0] * shots, seed, kind=kind)
        res, fates, _, _ = engine.run_driver(dg, rng, BETA, H, 20000, 10, 20000, itask=1,
                                             dn_thr=-0.93, up_thr=UP, ninputs=inputs.shape[0],
                                             compact=True)
        dg.close()
        rng.close()
        resolved = (fates >= 0).reshape(inputs.shape[0], shots).sum(axis=1)
        out[kind] = (np.asarray(res, np.float64), resolved)
    return out, radii


def test_committor_droplets_agree_between_streams(committor_pb):
    out, radii = committor_pb
    (pa, na), (pb, nb) = out["xorwow"], out["mwc64x"]
    assert np.all(na == 4096) and np.all(nb == 4096)  # every trajectory committed
    se = np.sqrt(pa * (1 - pa) / na + pb * (1 - pb) / nb)
    informative = (pa > 0.02) & (pa < 0.98)
    assert informative.sum() >= 4, (pa, radii)
    z = np.abs(pa - pb)[informative] / se[informative]
    assert np.all(z < 4), (pa, pb, radii)
    # jointly: the mean squared z is near 1 for agreeing estimates
    assert np.mean(z ** 2) < 3.0, z
    # where shooting is not informative, both agree on the basin
    sure = ~informative
    assert np.all(np.abs(pa - pb)[sure] < 0.05)
