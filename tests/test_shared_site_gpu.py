"""The multispin shared-site sweep (variant 7: a tile of 32 replicas shares
each attempt's site, transposed bit planes, bitwise full-adder neighbour
counts, per-lane acceptance draws, ballot flip mask) on a B200, bit for bit
against its serial statement in the oracle, including a partial last tile."""
import numpy as np
import pytest

from gpu_2dising_b200 import _native as nat
from gpu_2dising_b200 import engine

import oracle

pytestmark = pytest.mark.gpu

BETA, H = 0.54, 0.07


@pytest.fixture(scope="module", autouse=True)
def device():
    return engine.init_device(0)


@pytest.mark.parametrize("L,nsweeps,n", [(64, 2, 70), (32, 3, 70), (128, 1, 70), (48, 2, 70),
                                         (20, 3, 70), (5, 6, 70), (3, 4, 1)])
def test_shared_site_kernel_matches_serial_oracle(L, nsweeps, n):
    # n = 70: two full tiles and one of six; n = 1: a tile of one replica
    rs = np.random.default_rng(L)
    frac = rs.uniform(0.1, 0.9, size=(n, 1, 1))
    g0 = np.where(rs.random((n, L, L)) < frac, 1, -1).astype(np.int32)
    dg = engine.DeviceGrids(L, n, g0)
    dg.set_option(nat.OPT_SWEEP_VARIANT, 7)
    rng = engine.RngStates(n, 1000 + L, kind="mwc64x")
    st0 = rng.read_states()
    thr, fc = dg.thresholds(BETA, H)
    assert not fc
    dg.sweep(rng, BETA, H, nsweeps)
    g1, st1, mag = dg.download(), rng.read_states(), dg.magnetisation()
    for t0 in range(0, n, 32):
        t1 = min(n, t0 + 32)
        g = g0[t0:t1].copy()
        xs, cs = oracle.sweep_shared(L, g, nsweeps, st0[0, t0:t1], st0[1, t0:t1], thr)
        assert np.array_equal(g, g1[t0:t1]), t0
        assert np.array_equal(xs, st1[0, t0:t1]) and np.array_equal(cs, st1[1, t0:t1]), t0
        assert np.array_equal(mag[t0:t1], oracle.magnetisation_gpu(L, g))


def test_shared_site_kernel_needs_the_production_stream():
    dg = engine.DeviceGrids(64, 32)
    dg.set_option(nat.OPT_SWEEP_VARIANT, 7)
    rng = engine.RngStates(32, 1, kind="xorwow")
    with pytest.raises(nat.GaspError) as e:
        dg.sweep(rng, BETA, H, 1)
    assert e.value.status == nat.GASP_ERR_UNSUPPORTED


def test_shared_site_swarm_agrees_with_per_lane_sites():
    """Nucleated fraction of an L=32 swarm after 1500 sweeps: shared sites
    (tiles of 32 correlated replicas) vs per-lane sites, within 4.5 standard
    errors computed over blocks of 32 replicas."""
    L, R, tot, mag, up = 32, 8192, 1500, 50, 0.9
    out = {}
    for v, seed in ((0, 5), (7, 6)):
        dg = engine.DeviceGrids(L, R, -np.ones((R, L, L), np.int32))
        dg.set_option(nat.OPT_SWEEP_VARIANT, v)
        rng = engine.RngStates(R, seed, kind="mwc64x")
        fu = np.full(R, -1, np.int32)
        engine.run_driver(dg, rng, BETA, 0.10, tot, mag, tot, itask=0, dn_thr=-0.95, up_thr=up,
                          first_up=fu)
        blocks = (fu >= 0).reshape(-1, 32).mean(axis=1)
        out[v] = (blocks.mean(), blocks.std(ddof=1) / np.sqrt(blocks.size))
    (a, sa), (b, sb) = out[0], out[7]
    assert 0.05 < a < 0.95, out
    assert abs(a - b) < 4.5 * np.hypot(sa, sb), out
