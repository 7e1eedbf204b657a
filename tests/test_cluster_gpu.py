"""Largest-cluster collective variable on a B200: gasp_largest_cluster against
the committed golden sizes (reference CPU code), the oracle and the
reference's own cluster kernel; the driver with cv='largest_cluster' against
the reference driver.  All comparisons are exact."""
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN
from gpu_2dising_b200 import engine

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def device():
    return engine.init_device(0)


def _random(L, ng, p, seed):
    rng = np.random.default_rng(seed)
    return np.where(rng.random((ng, L, L)) < p, 1, -1).astype(np.int32)


def test_device_matches_golden():
    d = np.load(os.path.join(GOLDEN, "ref_cluster.npz"))
    for L in d["Ls"]:
        L = int(L)
        g = d[f"L{L}_grids"].astype(np.int32)
        dg = engine.DeviceGrids(L, g.shape[0], g)
        for k, spin in enumerate((1, -1)):
            assert np.array_equal(dg.largest_cluster(spin), d[f"L{L}_sizes"][k]), (L, spin)


@pytest.mark.parametrize("L,ng,p", [(2, 33, 0.5), (16, 64, 0.593), (33, 40, 0.593),
                                    (64, 96, 0.55), (64, 64, 0.7), (128, 40, 0.593),
                                    (170, 3, 0.593), (171, 3, 0.593), (300, 2, 0.6)])
def test_device_matches_oracle(L, ng, p):
    """Shared-memory labels up to L=170, the global work area beyond."""
    g = _random(L, ng, p, L * 7 + ng)
    dg = engine.DeviceGrids(L, ng, g)
    for spin in (1, -1):
        assert np.array_equal(dg.largest_cluster(spin), oracle.largest_cluster(L, g, spin))
    assert np.all(dg.largest_cluster(0) == 0)


def test_device_matches_reference_kernel(ref_gpu):
    L, ng = 64, 64
    g = _random(L, ng, 0.593, 5)
    dg = engine.DeviceGrids(L, ng, g)
    for spin in (1, -1):
        ref = np.zeros(ng, np.float32)
        assert ref_gpu.refgpu_largest_cluster(L, ng, spin, np.ascontiguousarray(g.reshape(-1)),
                                              ref) == 0
        assert np.array_equal(dg.largest_cluster(spin), ref)


DRIVER_CASES = [  # L, ng, seed, beta, h, tot, mag, grid, itask, dn, up, ninputs, init
    (32, 64, 21, 0.50, 0.30, 300, 20, 50, 0, 1.0, 200.0, 1, "down"),
    (24, 64, 22, 0.45, 0.10, 400, 10, 40, 1, 3.0, 150.0, 2, "sparse"),
    (16, 96, 23, 0.40, 0.20, 300, 5, 25, 1, 2.0, 60.0, 3, "random"),
]


def _initial(L, ng, init, seed):
    rng = np.random.default_rng(seed)
    if init == "down":
        return -np.ones((ng, L, L), np.int32)
    p = 0.1 if init == "sparse" else 0.5
    return np.where(rng.random((ng, L, L)) < p, 1, -1).astype(np.int32)


@pytest.mark.parametrize("case", DRIVER_CASES)
@pytest.mark.parametrize("compact", [False, True])
def test_driver_largest_cluster_matches_reference_driver(ref_gpu, case, compact):
    (L, ng, seed, beta, h, tot, mag, grid, itask, dn, up, ninputs, init) = case
    if compact and itask == 0:
        pytest.skip("compaction applies to committor runs")
    g0 = _initial(L, ng, init, seed)
    # reference driver, cv = largest_cluster, initial_spin = -1 (clusters of +1)
    gref = g0.reshape(-1).copy()
    r_fates = np.full(ng, -1, np.int32)
    nres = tot // mag if itask == 0 else ninputs
    r_res = np.zeros(nres + 1, np.float32)
    maxf = tot // min(mag, grid) + 2
    fg = np.zeros(maxf * ng * L * L, np.int32)
    fi = np.zeros(maxf, np.int32)
    fm = np.zeros(maxf * ng, np.float32)
    fl = np.zeros(maxf * ng, np.float32)
    n = ref_gpu.refgpu_run_driver_cv(L, ng, 32, 2, seed, beta, h, tot, mag, grid, itask, dn, up,
                                     ninputs, gref, r_fates.ctypes.data, r_res, maxf,
                                     fg.ctypes.data, fi.ctypes.data, fm.ctypes.data,
                                     b"largest_cluster", -1, fl.ctypes.data)
    assert n >= 1
    n = min(n, maxf)
    dg = engine.DeviceGrids(L, ng, g0)
    rng = engine.RngStates(ng, seed)
    frames = []

    def out(L_, ng_, g, isweep, m, lc):
        frames.append((isweep, g.copy(), m.copy(), lc.copy()))
        return 0

    res, fates, _, _ = engine.run_driver(dg, rng, beta, h, tot, mag, grid, itask=itask,
                                         dn_thr=dn, up_thr=up, ninputs=ninputs, outfunc=out,
                                         compact=compact, cv="largest_cluster", initial_spin=-1)
    assert np.array_equal(res, r_res[:nres])
    assert [f[0] for f in frames] == list(fi[:n])
    nf = 1 if compact else n  # compaction stops resolved replicas (see the magnetisation test)
    for k in range(nf):
        assert np.array_equal(frames[k][1].reshape(-1), fg[k * ng * L * L:(k + 1) * ng * L * L])
        assert np.array_equal(frames[k][2], fm[k * ng:(k + 1) * ng])
        assert np.array_equal(frames[k][3], fl[k * ng:(k + 1) * ng])
    if itask == 1:
        assert np.array_equal(fates, r_fates)
        assert np.any(fates == 1) or np.any(fates == 0)
    else:
        assert np.array_equal(dg.download().reshape(-1), gref)
        assert res[-1] > 0.0  # some replicas grew a cluster above up


def test_pygasp_swarm_with_largest_cluster(ref_gpu, tmp_path, monkeypatch):
    """gasp.run_nucleation_swarm(cv='largest_cluster'): result, the module's
    largest_cluster records and the snapshots' lclus_size, against the
    reference driver on the same seed."""
    from gpu_2dising_b200 import gasp
    monkeypatch.chdir(tmp_path)
    L, ng, seed, beta, h, tot, mag, grid = 32, 64, 31, 0.54, 0.15, 300, 10, 10
    dn, up = 2.0, 300.0
    res = gasp.run_nucleation_swarm(L, ng, tot, beta, h, cv="largest_cluster", up_threshold=up,
                                    dn_threshold=dn, mag_output_int=mag, grid_output_int=grid,
                                    seed=seed)
    g0 = -np.ones((ng, L, L), np.int32).reshape(-1)
    r_res = np.zeros(tot // mag + 1, np.float32)
    maxf = tot // min(mag, grid) + 2
    fl = np.zeros(maxf * ng, np.float32)
    n = ref_gpu.refgpu_run_driver_cv(L, ng, 32, 2, seed, beta, h, tot, mag, grid, 0, dn, up, 1,
                                     g0, None, r_res, maxf, None, None, None,
                                     b"largest_cluster", -1, fl.ctypes.data)
    assert np.array_equal(res, r_res[:tot // mag])
    assert len(gasp.largest_cluster) == n
    for k in range(n):
        assert np.array_equal(np.array(gasp.largest_cluster[k], np.float32),
                              fl[k * ng:(k + 1) * ng])
    snaps = [s for frame in gasp.grids for s in frame]
    assert snaps and all(dn < s.lclus_size < up for s in snaps)
    import h5read
    f = h5read.read("gridstates.hdf5")
    assert f["total_saved_grids"].value == n * ng
    for k in range(n):
        grp = f[f"sweep_{k * grid}"]
        assert [grp[f"grid_{i}"].attrs["lclus_size"] for i in range(ng)] == \
            ["%g" % x for x in gasp.largest_cluster[k]]
    with pytest.warns(UserWarning):
        gasp.run_nucleation_swarm(16, 32, 10, beta, h, cv="largest_cluster", seed=1)
