"""Bit-exact parity of the CUDA path with the reference, on a B200.

Oracles: the reference's GPU kernels and driver compiled unmodified for
sm_100a (oracle/_ref/libref_gpu.so), the reference CPU driver's committed
golden runs (tests/golden/ref_cpu_driver.npz) and the CPU restatement fed the
device-recorded cuRAND stream.  Every comparison is exact (integer spins and
bit-identical float magnetisation)."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN
from gpu_2dising_b200 import engine
from gpu_2dising_b200._native import GaspError

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def device():
    return engine.init_device(0)


def _grids(L, ng, kind, seed):
    rng = np.random.default_rng(seed)
    if kind == "down":
        return -np.ones((ng, L, L), np.int32)
    if kind == "random":
        return np.where(rng.random((ng, L, L)) < 0.5, 1, -1).astype(np.int32)
    # sparse random up-spins in a down background
    return np.where(rng.random((ng, L, L)) < 0.1, 1, -1).astype(np.int32)


def _ours_kernels(L, ng, method, seed, beta, h, nsw, ncalls, g0):
    dg = engine.DeviceGrids(L, ng, g0)
    r = engine.RngStates(ng, seed)
    mags = [dg.magnetisation()]
    for _ in range(ncalls):
        dg.sweep(r, beta, h, nsw, gpu_method=method)
        mags.append(dg.magnetisation())
    return dg.download(), np.stack(mags)


CASES = [  # L, ngrids, method, init, beta, h, nsweeps, ncalls
    (16, 1, 2, "random", 0.54, 0.07, 3, 2),
    (16, 33, 2, "random", 0.45, 0.10, 2, 3),
    (32, 64, 0, "sparse", 0.54, 0.07, 2, 2),
    (48, 40, 1, "random", 0.60, 0.12, 1, 2),
    (64, 96, 2, "down", 0.54, 0.07, 2, 2),
    (64, 70, 0, "random", 0.30, 0.50, 1, 2),
    (64, 33, 1, "sparse", 0.54, 0.07, 1, 2),
    (20, 35, 2, "random", 0.50, -0.20, 2, 2),
    (96, 32, 2, "random", 0.44, 0.00, 1, 1),
    (128, 40, 2, "sparse", 0.55, 0.05, 1, 1),
    (8, 33, 2, "random", 0.54, 0.07, 4, 2),
    (8, 1, 1, "random", 0.40, 0.10, 3, 2),
    (64, 1, 2, "random", 0.54, 0.07, 2, 2),
    (96, 65, 0, "sparse", 0.54, -0.07, 1, 2),
    (96, 1, 1, "random", 0.60, 0.10, 1, 1),
    # beta = 3: the most costly class can never accept (P below the smallest
    # uniform), so the kernels compare in float instead of by threshold
    (64, 40, 2, "random", 3.0, 0.10, 2, 2),
    (48, 33, 0, "random", 3.0, -0.20, 2, 1),
    (128, 32, 1, "sparse", 3.0, 0.05, 1, 1),
]


@pytest.mark.parametrize("L,ng,method,init,beta,h,nsw,ncalls", CASES)
def test_exact_sweep_matches_reference_kernels(ref_gpu, L, ng, method, init, beta, h, nsw, ncalls):
    seed = 1000 + 7 * L + ng
    g0 = _grids(L, ng, init, seed)
    gref = g0.reshape(-1).copy()
    mref = np.zeros((ncalls + 1) * ng, np.float32)
    assert ref_gpu.refgpu_run_kernels(L, ng, 32, method, seed, beta, h, nsw, ncalls, gref, mref) == 0
    gour, mour = _ours_kernels(L, ng, method, seed, beta, h, nsw, ncalls, g0)
    assert np.array_equal(gour.reshape(-1), gref)
    assert np.array_equal(mour.reshape(-1), mref)
    assert not np.array_equal(gour, g0)  # the sweep did something


def test_exact_sweep_matches_cpu_oracle_on_recorded_stream(ref_gpu):
    """The restated GPU arithmetic, fed the reference's own device stream."""
    L, ng, nsw, seed, beta, h = 16, 5, 4, 4242, 0.5, 0.1
    g0 = _grids(L, ng, "random", seed)
    n = 2 * L * L * nsw
    u = np.zeros(ng * n, np.float32)
    assert ref_gpu.refgpu_uniform_stream(seed, ng, n, u) == 0
    P = oracle.probs_gpu(beta, h)
    exp = g0.copy()
    for i in range(ng):
        x = np.ascontiguousarray(exp[i]).reshape(-1)
        oracle.sweep_gpu_stream(L, x, u[i * n:(i + 1) * n], P)
        exp[i] = x.reshape(L, L)
    gour, mour = _ours_kernels(L, ng, 2, seed, beta, h, nsw, 1, g0)
    assert np.array_equal(gour, exp)
    assert np.array_equal(mour[-1], oracle.magnetisation_gpu(L, exp))


def _golden_names():
    return list(np.load(os.path.join(GOLDEN, "ref_cpu_driver.npz"))["names"])


@pytest.mark.parametrize("name", _golden_names())
def test_trace_cpu_mode_matches_reference_cpu_driver(name):
    """mc_driver_cpu (golden, MT19937 seeded) vs the CUDA kernel in CPU-trace
    mode consuming the same genrand_real3 stream."""
    d = np.load(os.path.join(GOLDEN, "ref_cpu_driver.npz"))
    c = {k.split("__", 1)[1]: d[k] for k in d.files if k.startswith(name + "__")}
    L, ng = int(c["L"]), int(c["ngrids"])
    beta, h = float(c["beta"]), float(c["h"])
    mt = oracle.MTReal3(int(c["seed"]))
    dg = engine.DeviceGrids(L, ng, c["initial"].astype(np.int32))

    def sweep_batch(g, batch, spc):
        dg.upload(g)
        dg.sweep_trace_cpu(mt.batch(ng, L, spc), beta, h, spc)
        g[...] = dg.download()

    grids = c["initial"].astype(np.int32).copy()
    tr = oracle.driver_cpu_semantics(grids, sweep_batch, lambda g: (dg.upload(g), dg.magnetisation())[1],
                                     int(c["tot"]), int(c["mag"]), int(c["grid"]),
                                     itask=int(c["itask"]), up=float(c["up"]), dn=float(c["dn"]),
                                     ninputs=int(c["ninputs"]))
    assert np.array_equal(grids, c["final"].astype(np.int32))
    assert np.array_equal(tr.result, c["result"])
    for (isw, g, m), fg, fm in zip(tr.dumps, c["frame_grids"], c["frame_mag"]):
        assert np.array_equal(g, fg.astype(np.int32))
        assert np.array_equal(m, fm)
    if int(c["itask"]) == 1:
        assert np.array_equal(tr.fates, c["fates"])


def _ref_driver(ref_gpu, L, ng, seed, beta, h, tot, mag, grid, itask, dn, up, ninputs, g0):
    g = g0.reshape(-1).copy()
    fates = np.full(ng, -1, np.int32)
    nres = tot // mag if itask == 0 else ninputs
    result = np.zeros(max(nres, 1) + 1, np.float32)  # +1: the reference may write result[tot/mag]
    maxf = tot // min(mag, grid) + 2
    fg = np.zeros(maxf * ng * L * L, np.int32)
    fi = np.zeros(maxf, np.int32)
    fm = np.zeros(maxf * ng, np.float32)
    n = ref_gpu.refgpu_run_driver(L, ng, 32, 2, seed, beta, h, tot, mag, grid, itask, dn, up,
                                  ninputs, g, fates.ctypes.data, result, maxf, fg.ctypes.data,
                                  fi.ctypes.data, fm.ctypes.data)
    n = min(n, maxf)
    return (result[:nres], fates, fi[:n], fg[:n * ng * L * L].reshape(n, ng, L, L),
            g.reshape(ng, L, L))


DRIVER_CASES = [  # L, ng, seed, beta, h, tot, mag, grid, itask, dn, up, ninputs, init
    (32, 64, 11, 0.50, 0.30, 300, 20, 50, 0, -0.9, 0.2, 1, "down"),
    (16, 40, 12, 0.54, 0.07, 31, 10, 20, 0, -0.9, 0.9, 1, "random"),   # isweep == tot-1, stale dump
    (16, 33, 13, 0.45, 0.10, 31, 20, 10, 0, -0.9, -0.3, 1, "sparse"),  # stale check, result[tot/mag]
    (24, 64, 14, 0.45, 0.10, 400, 10, 40, 1, -0.7, 0.2, 2, "sparse"),
    (16, 96, 15, 0.40, 0.20, 300, 5, 25, 1, -0.8, 0.5, 3, "random"),
]


@pytest.mark.parametrize("case", DRIVER_CASES)
@pytest.mark.parametrize("compact", [False, True])
def test_driver_matches_reference_driver(ref_gpu, case, compact):
    (L, ng, seed, beta, h, tot, mag, grid, itask, dn, up, ninputs, init) = case
    if compact and itask == 0:
        pytest.skip("compaction applies to committor runs")
    g0 = _grids(L, ng, init, seed)
    r_res, r_fates, r_fi, r_fg, r_final = _ref_driver(ref_gpu, L, ng, seed, beta, h, tot, mag,
                                                      grid, itask, dn, up, ninputs, g0)
    dg = engine.DeviceGrids(L, ng, g0)
    rng = engine.RngStates(ng, seed)
    frames = []

    def out(L_, ng_, g, isweep, m):
        frames.append((isweep, g.copy()))
        return 0

    res, fates, _, _ = engine.run_driver(dg, rng, beta, h, tot, mag, grid, itask=itask, dn_thr=dn,
                                         up_thr=up, ninputs=ninputs, outfunc=out,
                                         compact=compact)
    assert np.array_equal(res, r_res)
    assert [f[0] for f in frames] == list(r_fi)
    # With compaction a resolved replica is no longer simulated, so dumped
    # grids can differ from the reference after its fate is decided; the
    # first frame and every fate/result are still identical.
    for (isw, g), rg in zip(frames[:1] if compact else frames, r_fg):
        assert np.array_equal(g, rg)
    if itask == 1:
        assert np.array_equal(fates, r_fates)
    else:
        assert np.array_equal(dg.download(), r_final)


@pytest.mark.parametrize("case", [c for c in DRIVER_CASES if c[8] == 1])
@pytest.mark.parametrize("mag_grid", [None, (10, 7)])
def test_committor_on_device_matches_reference_driver(ref_gpu, case, mag_grid):
    """Compaction without callbacks runs the checks on the device; fates and
    pB must equal the reference driver's (and so the host loop's)."""
    (L, ng, seed, beta, h, tot, mag, grid, itask, dn, up, ninputs, init) = case
    if mag_grid is not None:  # checks every 10 sweeps, launches of 7 sweeps
        mag, grid = mag_grid
    g0 = _grids(L, ng, init, seed)
    r_res, r_fates, _, _, _ = _ref_driver(ref_gpu, L, ng, seed, beta, h, tot, mag, grid, itask,
                                          dn, up, ninputs, g0)
    dg = engine.DeviceGrids(L, ng, g0)
    rng = engine.RngStates(ng, seed)
    res, fates, _, att = engine.run_driver(dg, rng, beta, h, tot, mag, grid, itask=1, dn_thr=dn,
                                           up_thr=up, ninputs=ninputs, compact=True)
    assert np.array_equal(fates, r_fates)
    assert np.array_equal(res, r_res)
    # the host loop (a no-op packed callback keeps the driver on the host)
    dg2 = engine.DeviceGrids(L, ng, g0)
    rng2 = engine.RngStates(ng, seed)
    res2, fates2, _, att2 = engine.run_driver(dg2, rng2, beta, h, tot, mag, grid, itask=1,
                                              dn_thr=dn, up_thr=up, ninputs=ninputs,
                                              compact=True, packed_out=lambda *a: 0)
    assert np.array_equal(fates2, fates) and np.array_equal(res2, res)
    assert att == att2
    assert np.array_equal(dg.download(), dg2.download())


@pytest.mark.parametrize("L,ng", [(5, 7), (16, 33), (64, 64), (30, 65), (48, 70), (32, 1),
                                  (64, 32768)])
def test_pack_unpack_frame_and_magnetisation(L, ng):
    g = _grids(L, ng, "random", L + ng)
    dg = engine.DeviceGrids(L, ng, g)
    assert np.array_equal(dg.download(), g)
    assert np.array_equal(dg.pack_frame(), oracle.pack_frame(L, g))
    assert np.array_equal(dg.magnetisation(), oracle.magnetisation_gpu(L, g))


def test_full_size_swarm_step_bit_exact(ref_gpu):
    """The bench workload's shape (L=64, 32768 replicas, all down) for one
    sweep batch, against the reference bitmap32 kernel."""
    L, ng, seed, beta, h = 64, 32768, 20240501, 0.54, 0.07
    g0 = -np.ones((ng, L, L), np.int32)
    gref = g0.reshape(-1).copy()
    mref = np.zeros(2 * ng, np.float32)
    assert ref_gpu.refgpu_run_kernels(L, ng, 32, 2, seed, beta, h, 2, 1, gref, mref) == 0
    gour, mour = _ours_kernels(L, ng, 2, seed, beta, h, 2, 1, g0)
    assert np.array_equal(mour.reshape(-1), mref)
    assert np.array_equal(gour.reshape(-1), gref)


@pytest.mark.parametrize("L,nin,per", [(64, 3, 5), (30, 4, 16), (7, 1, 9)])
def test_upload_inputs_replicates_like_init_grids_from_array(L, nin, per):
    inputs = _grids(L, nin, "random", L * nin)
    dg = engine.DeviceGrids(L, nin * per)
    dg.upload_inputs(inputs)
    assert np.array_equal(dg.download(), np.repeat(inputs, per, axis=0))
    with pytest.raises(GaspError):
        engine.DeviceGrids(L, 10).upload_inputs(np.repeat(inputs[:1], 3, axis=0))


def test_large_lattice_hbm_path_matches_reference_method0(ref_gpu):
    """L beyond the shared-memory limit runs in place in HBM, bit-exact with
    the reference's global-memory kernel."""
    L = engine.max_shared_L(0) + 6
    ng, seed, beta, h = 40, 77, 0.5, 0.1
    g0 = _grids(L, ng, "random", seed)
    gref = g0.reshape(-1).copy()
    mref = np.zeros(2 * ng, np.float32)
    assert ref_gpu.refgpu_run_kernels(L, ng, 32, 0, seed, beta, h, 1, 1, gref, mref) == 0
    gour, mour = _ours_kernels(L, ng, 0, seed, beta, h, 1, 1, g0)
    assert np.array_equal(gour.reshape(-1), gref)
    assert np.array_equal(mour.reshape(-1), mref)


def test_errors_are_raised_not_hidden():
    with pytest.raises(GaspError):
        engine.DeviceGrids(8193, 32)
    dg = engine.DeviceGrids(16, 64)
    r = engine.RngStates(32, 1)
    with pytest.raises(GaspError):
        dg.sweep(r, 0.5, 0.1, 1)  # fewer RNG states than replicas
    with pytest.raises(GaspError):
        dg.sweep(engine.RngStates(64, 1), 0.5, 0.1, 1, gpu_method=3)


def test_float_comparison_switch_is_reported():
    """At beta = 3 some class can never accept and the set reports the float
    comparison; at beta = 0.54 the integer thresholds are exact."""
    dg = engine.DeviceGrids(64, 32)
    assert dg.thresholds(3.0, 0.10)[1] is True
    assert dg.thresholds(0.54, 0.07)[1] is False
