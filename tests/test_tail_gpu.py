"""The production (MWC64X) sweeps on a B200 against the oracle, bit for bit:
the row and generic kernels against the serial one-stream sweep, and the
one-warp-per-replica kernel (variant 6) against its serial statement -- which
applies attempts one at a time, so equality also shows that the kernel's
parallel rounds change nothing.  On the reference (XORWOW) stream variant 6
draws in the replica's own order and equals the row kernel bit for bit.  Then
committor shooting that switches to variant 6 for its last undecided
replicas against shooting that never does."""
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


def _lane_tables():
    mul = np.zeros(32, np.uint64)
    inv = np.zeros(32, np.uint64)
    assert nat.lib().gasp_mwc64x_lane_multipliers(mul, inv) == 0
    return mul, inv


def _start(L, n, seed):
    rs = np.random.default_rng(seed)
    frac = rs.uniform(0.1, 0.9, size=(n, 1, 1))
    return np.where(rs.random((n, L, L)) < frac, 1, -1).astype(np.int32)


def _run(L, n, variant, nsweeps, seed):
    g0 = _start(L, n, seed)
    dg = engine.DeviceGrids(L, n, g0)
    dg.set_option(nat.OPT_SWEEP_VARIANT, variant)
    rng = engine.RngStates(n, seed, kind="mwc64x")
    st0 = rng.read_states()
    thr, fc = dg.thresholds(BETA, H)
    assert not fc
    dg.sweep(rng, BETA, H, nsweeps)
    return g0, st0, thr, dg.download(), rng.read_states(), dg.magnetisation()


@pytest.mark.parametrize("L,variant", [(64, 0), (32, 0), (128, 0), (64, 2), (48, 2), (48, 1),
                                       (20, 1)])
def test_production_kernels_match_serial_oracle(L, variant):
    n, nsweeps = 40, 2
    g0, st0, thr, g1, st1, mag = _run(L, n, variant, nsweeps, seed=L + variant)
    for r in range(n):
        g = g0[r].copy().reshape(-1)
        x, c = oracle.sweep_mwc(L, g, nsweeps * L * L, st0[0, r], st0[1, r], thr)
        assert np.array_equal(g.reshape(L, L), g1[r]), r
        assert (x, c) == (int(st1[0, r]), int(st1[1, r])), r
        assert mag[r] == oracle.magnetisation_gpu(L, g.reshape(1, L, L))[0]


@pytest.mark.parametrize("L,nsweeps,n", [(64, 2, 37), (48, 2, 37), (20, 3, 37), (128, 1, 37),
                                         (5, 4, 37), (3, 5, 3), (64, 1, 1)])
def test_warp_per_replica_kernel_matches_serial_oracle(L, nsweeps, n):
    g0, st0, thr, g1, st1, mag = _run(L, n, 6, nsweeps, seed=100 + L)
    mul, inv = _lane_tables()
    for r in range(n):
        g = g0[r].copy().reshape(-1)
        x, c = oracle.sweep_tail(L, g, nsweeps, st0[0, r], st0[1, r], thr, mul, inv)
        assert np.array_equal(g.reshape(L, L), g1[r]), r
        assert (x, c) == (int(st1[0, r]), int(st1[1, r])), r
        assert mag[r] == oracle.magnetisation_gpu(L, g.reshape(1, L, L))[0]


@pytest.mark.parametrize("L,nsweeps,n,beta", [(64, 2, 37, BETA), (48, 2, 37, BETA),
                                              (20, 3, 37, BETA), (128, 1, 37, BETA),
                                              (5, 4, 37, BETA), (3, 5, 3, BETA),
                                              (64, 1, 1, BETA), (64, 2, 33, 3.0)])
def test_warp_per_replica_kernel_on_reference_stream_equals_row_kernel(L, nsweeps, n, beta):
    """On the XORWOW stream variant 6 draws each replica's attempts in the
    replica's own order, so its grids, magnetisation and RNG states equal the
    row kernel's (and so the reference kernels'), the float-comparison path
    (beta = 3) included."""
    g0 = _start(L, n, 300 + L)
    outs = []
    for variant in (0, 6):
        dg = engine.DeviceGrids(L, n, g0)
        dg.set_option(nat.OPT_SWEEP_VARIANT, variant)
        rng = engine.RngStates(n, 17 + L, kind="xorwow")
        dg.sweep(rng, beta, H, nsweeps)
        dg.sweep(rng, beta, H, 1)
        outs.append((dg.download(), dg.magnetisation(), rng.read_states()[:, :n]))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert np.array_equal(outs[0][2], outs[1][2])
    assert not np.array_equal(outs[0][0], g0)


@pytest.mark.parametrize("tail", [1 << 30, 700])
def test_committor_tail_on_reference_stream_changes_nothing(tail):
    """Committor shooting on the XORWOW stream: fates, pB, attempt counts and
    final grids are the same whether the last undecided replicas (or all of
    them from the start) sweep with one warp each or stay on the row kernel."""
    yy, xx = np.mgrid[0:64, 0:64]
    inputs = np.stack([np.where((yy - 32) ** 2 + (xx - 32) ** 2 <= r * r, 1, -1)
                       for r in (6.0, 7.0, 8.0)]).astype(np.int32)
    outs = []
    for t in (0, tail):
        dg = engine.DeviceGrids(64, 3 * 256)
        dg.upload_inputs(inputs)
        dg.set_option(nat.OPT_TAIL_REPLICAS, t)
        rng = engine.RngStates(3 * 256, 29, kind="xorwow")
        res, fates, _, att = engine.run_driver(dg, rng, BETA, H, 20000, 10, 20000, itask=1,
                                               dn_thr=-0.93, up_thr=0.9, ninputs=3,
                                               compact=True)
        assert np.count_nonzero(fates == -1) == 0
        outs.append((np.asarray(res).copy(), fates.copy(), att, dg.download()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2]
    assert np.array_equal(outs[0][3], outs[1][3])


def _droplets(L, radii):
    yy, xx = np.mgrid[0:L, 0:L]
    return np.stack([np.where((yy - L / 2) ** 2 + (xx - L / 2) ** 2 <= r * r, 1, -1)
                     for r in radii]).astype(np.int32)


def _shoot(inputs, shots, seed, tail):
    L, k = inputs.shape[1], inputs.shape[0]
    dg = engine.DeviceGrids(L, k * shots)
    dg.upload_inputs(inputs)
    dg.set_option(nat.OPT_TAIL_REPLICAS, tail)
    rng = engine.RngStates(k * shots, seed, kind="mwc64x")
    res, fates, _, att = engine.run_driver(dg, rng, BETA, H, 20000, 10, 20000, itask=1,
                                           dn_thr=-0.93, up_thr=0.9, ninputs=k, compact=True)
    assert np.count_nonzero(fates == -1) == 0
    return np.asarray(res, np.float64), att


def test_committor_with_warp_per_replica_tail_agrees():
    """pB of droplets around the critical size: never switching, switching at
    the default threshold, and sweeping every replica with variant 6 from the
    start agree within binomial errors; the switched runs are deterministic."""
    inputs = _droplets(64, (5.5, 6.5, 7.0, 7.5, 8.0, 9.0))
    shots = 2048
    base, _ = _shoot(inputs, shots, 7, 0)
    informative = (base > 0.05) & (base < 0.95)
    assert informative.sum() >= 2, base
    for tail, seed in ((4096, 8), (1 << 30, 9)):
        pb, att = _shoot(inputs, shots, seed, tail)
        se = np.sqrt(base * (1 - base) / shots + pb * (1 - pb) / shots) + 1e-12
        assert np.all(np.abs(pb - base) < 4.5 * se), (tail, base, pb)
        pb2, att2 = _shoot(inputs, shots, seed, tail)
        assert np.array_equal(pb, pb2) and att == att2
