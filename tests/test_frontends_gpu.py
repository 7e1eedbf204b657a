"""The two front ends on a B200: the PyGASP mirror (gpu_2dising_b200.gasp) and
the `gasp` CLI, each compared with the reference driver (mc_driver_gpu,
compiled unmodified) run with the same seed."""
import os
import subprocess

import numpy as np
import pytest

import h5read
import oracle
from conftest import REPO
from gpu_2dising_b200 import engine
from gpu_2dising_b200._native import lib

pytestmark = pytest.mark.gpu

CLI = os.path.join(REPO, "gpu_2dising_b200", "gasp")


@pytest.fixture(scope="module")
def gasp_mod():
    from gpu_2dising_b200 import gasp
    return gasp


def _ref_driver(ref_gpu, L, ng, seed, beta, h, tot, mag, grid, itask, dn, up, ninputs, g0):
    g = g0.reshape(-1).copy()
    fates = np.full(ng, -1, np.int32)
    nres = tot // mag if itask == 0 else ninputs
    result = np.zeros(max(nres, 1) + 1, np.float32)
    maxf = tot // min(mag, grid) + 2
    fg = np.zeros(maxf * ng * L * L, np.int32)
    fi = np.zeros(maxf, np.int32)
    fm = np.zeros(maxf * ng, np.float32)
    n = ref_gpu.refgpu_run_driver(L, ng, 32, 2, seed, beta, h, tot, mag, grid, itask, dn, up,
                                  ninputs, g, fates.ctypes.data, result, maxf, fg.ctypes.data,
                                  fi.ctypes.data, fm.ctypes.data)
    n = min(n, maxf)
    return result[:nres], fates, fi[:n], fg[:n * ng * L * L].reshape(n, ng, L, L)


def test_pygasp_swarm_matches_reference(ref_gpu, gasp_mod, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    L, ng, tot, mag, grid, beta, h, up, dn, seed = 32, 64, 300, 20, 50, 0.5, 0.3, 0.2, -0.95, 77
    frac = gasp_mod.run_nucleation_swarm(L, ng, tot, beta, h, up_threshold=up, dn_threshold=dn,
                                         mag_output_int=mag, grid_output_int=grid, seed=seed)
    r_res, _, r_fi, r_fg = _ref_driver(ref_gpu, L, ng, seed, beta, h, tot, mag, grid, 0, dn, up,
                                       1, -np.ones((ng, L, L), np.int32))
    assert frac.dtype == np.float32 and np.array_equal(frac, r_res)
    assert len(gasp_mod.magnetisation) == len(r_fi)
    # snapshots: grids strictly between the thresholds at each dump (src/ising_ext.cu:388)
    snaps = [s for lst in gasp_mod.grids for s in lst]
    by_isweep = dict(zip(r_fi, r_fg))
    for s in snaps:
        assert dn < s.magnetisation < up
        assert s.grid.dtype == np.int8 and s.grid.shape == (L, L)
        assert np.array_equal(s.grid.astype(np.int32), by_isweep[s.isweep][s.igrid])
        assert s.committor == -1.0
    nexp = 0
    for i, isw in enumerate(r_fi):
        m = oracle.magnetisation_gpu(L, r_fg[i]).astype(np.float64)
        nexp += int(np.count_nonzero((m > dn) & (m < up)))
    assert len(snaps) == nexp
    # the HDF5 side file: every dump's grids and magnetisations
    # (src/ising_ext.cu:360-366, src/io.c:201-301)
    f = h5read.read("gridstates.hdf5")
    assert (f["L"].value, f["ngrids"].value, f["tot_nsweeps"].value) == (L, ng, tot)
    assert (f["beta"].value, f["h"].value) == (beta, h)
    assert f["total_saved_grids"].value == len(r_fi) * ng
    assert sorted(k for k in f if k.startswith("sweep_")) == sorted(f"sweep_{i}" for i in r_fi)
    for k, isw in enumerate(r_fi):
        grp = f[f"sweep_{isw}"]
        for i in range(ng):
            assert np.array_equal(grp[f"grid_{i}"].value, r_fg[k][i])
            assert grp[f"grid_{i}"].attrs == {
                "magnetisation": "%g" % gasp_mod.magnetisation[k][i], "lclus_size": "null",
                "committor": "null", "committor_error": "null"}


def test_pygasp_committor_matches_reference(ref_gpu, gasp_mod, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    L, ng, tot, mag, grid, beta, h, up, dn, seed = 24, 64, 400, 10, 40, 0.45, 0.10, 0.2, -0.7, 5
    yy, xx = np.mgrid[0:L, 0:L]
    inputs = [np.where((yy - L / 2) ** 2 + (xx - L / 2) ** 2 <= r * r, 1, -1).astype(np.int8)
              for r in (3.0, 4.5)]
    oracle.lib().orc_srand(1)
    out = gasp_mod.run_committor_calc(L, ng, tot, beta, h, up_threshold=up, dn_threshold=dn,
                                      mag_output_int=mag, grid_output_int=grid,
                                      grid_input="NumPy", grid_array=inputs, nsms=4, seed=seed)
    g0 = np.concatenate([np.repeat(a[None].astype(np.int32), ng // 2, axis=0) for a in inputs])
    r_res, r_fates, _, _ = _ref_driver(ref_gpu, L, ng, seed, beta, h, tot, mag, grid, 1, dn, up,
                                       2, g0)
    oracle.lib().orc_srand(1)
    errs = [oracle.lib().orc_bootstrap_errbar(ng // 2, ng // 2,
                                              np.ascontiguousarray(r_fates[i * 32:(i + 1) * 32]))
            for i in range(2)]
    assert [o[0] for o in out] == [float(x) for x in r_res]
    assert [o[1] for o in out] == errs
    f = h5read.read("pBgrids.hdf5")
    ndump = len(gasp_mod.magnetisation)
    assert f["ngrids"].value == ng and f["total_saved_grids"].value == ndump * ng
    assert len([k for k in f if k.startswith("sweep_")]) == ndump
    first = f["sweep_0"]
    assert all(np.array_equal(first[f"grid_{i}"].value, g0[i]) for i in range(ng))
    # compaction gives the same committors
    oracle.lib().orc_srand(1)
    out2 = gasp_mod.run_committor_calc(L, ng, tot, beta, h, up_threshold=up, dn_threshold=dn,
                                       mag_output_int=mag, grid_output_int=grid,
                                       grid_input="NumPy", grid_array=inputs, nsms=4, seed=seed,
                                       compact=True)
    assert out2 == out


def test_pygasp_hdf5_write_failure_raises(gasp_mod, tmp_path, monkeypatch, capfd):
    """A side file that cannot be written stops the run with the reference's
    RuntimeError text (src/ising_ext.cu:360-366)."""
    monkeypatch.chdir(tmp_path)
    os.mkdir("gridstates.hdf5")  # neither creatable nor openable as a file
    with pytest.raises(RuntimeError, match="Error writing HDF5 file"):
        gasp_mod.run_nucleation_swarm(16, 32, 40, 0.5, 0.1, mag_output_int=10,
                                      grid_output_int=20, seed=3)
    err = capfd.readouterr().err
    assert "failed to create HDF5 file 'gridstates.hdf5'" in err
    assert "failed to open HDF5 file 'gridstates.hdf5' for writing" in err


def test_pygasp_validation(gasp_mod):
    with pytest.raises(ValueError):
        gasp_mod.run_nucleation_swarm(16, 32, 10, 0.5, 0.1, cv="energy")
    with pytest.raises(ValueError):
        gasp_mod.run_nucleation_swarm(16, 32, 10, 0.5, 0.1, max_keep_grids=-1)
    with pytest.raises(TypeError):
        gasp_mod.run_committor_calc(16, 32, 10, 0.5, 0.1, grid_input="NumPy", grid_array=(1, 2),
                                    nsms=4)
    with pytest.raises(TypeError):
        gasp_mod.run_committor_calc(16, 32, 10, 0.5, 0.1, grid_input="NumPy",
                                    grid_array=[np.zeros((16, 16), np.int32)], nsms=4)
    with pytest.raises(ValueError):
        gasp_mod.run_committor_calc(16, 30, 10, 0.5, 0.1, grid_input="NumPy",
                                    grid_array=[np.zeros((16, 16), np.int8)], nsms=4)
    with pytest.raises(ValueError):
        gasp_mod.run_committor_calc(16, 32, 10, 0.5, 0.1, grid_input="NumPy",
                                    grid_array=[np.zeros((8, 8), np.int8)], nsms=4)
    with pytest.raises(ValueError):
        gasp_mod.run_committor_calc(16, 32, 10, 0.5, 0.1, nsms=-1)
    with pytest.raises(ValueError):
        gasp_mod.run_nucleation_swarm(16, 32, 10, 0.5, 0.1, rng="philox")


def test_pygasp_production_stream(gasp_mod, tmp_path, monkeypatch):
    """rng="mwc64x" runs both entry points on the production stream: a swarm
    is reproducible per seed, and the committor of an all-up and an
    all-down grid is exact."""
    monkeypatch.chdir(tmp_path)
    a = gasp_mod.run_nucleation_swarm(32, 64, 200, 0.5, 0.12, seed=5, rng="mwc64x",
                                      keep_grids=False)
    b = gasp_mod.run_nucleation_swarm(32, 64, 200, 0.5, 0.12, seed=5, rng="mwc64x",
                                      keep_grids=False)
    assert np.array_equal(a, b)
    grids = [np.ones((16, 16), np.int8), -np.ones((16, 16), np.int8)]
    out = gasp_mod.run_committor_calc(16, 64, 100, 0.54, 0.07, grid_input="NumPy",
                                      grid_array=grids, nsms=2, seed=3, rng="mwc64x",
                                      keep_grids=False)
    assert [round(float(p), 6) for p, _ in out] == [1.0, 0.0]


def test_cli_swarm_matches_reference(ref_gpu, tmp_path):
    L, ng, tot, mag, grid, beta, h, up, seed = 32, 64, 300, 20, 50, 0.5, 0.3, 0.2, 4242
    env = dict(os.environ, GASP_SEED=str(seed), GASP_L=str(L), GASP_UP=str(up))
    r = subprocess.run([CLI, str(tot), str(ng), str(mag), str(grid), "32", "0", "2", str(beta),
                        str(h), "0"], cwd=tmp_path, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln and ln[0] == " " and "Sweep" not in ln]
    r_res, _, r_fi, r_fg = _ref_driver(ref_gpu, L, ng, seed, beta, h, tot, mag, grid, 0, -0.9,
                                       up, 1, -np.ones((ng, L, L), np.int32))
    assert r.stdout.splitlines()[0] == "# isweep    nucleated fraction"
    exp = [f"{i * mag:10d}  {float(x):12.6f}" for i, x in enumerate(r_res)]
    assert lines[:len(exp)] == exp[:len(lines)]
    assert "# Time taken on GPU =" in r.stdout
    frames = oracle.read_gridstates(str(tmp_path / "gridstates.bin"))
    assert [f[2] for f in frames] == list(r_fi)
    for f, rg in zip(frames, r_fg):
        assert f[0] == L and f[1] == ng and np.array_equal(f[3], rg)


def test_cli_committor_reads_gridinput(ref_gpu, tmp_path):
    L, ng, tot, mag, grid, beta, h, seed = 16, 64, 300, 10, 50, 0.45, 0.1, 99
    yy, xx = np.mgrid[0:L, 0:L]
    g = np.where((yy - L / 2) ** 2 + (xx - L / 2) ** 2 <= 9.0, 1, -1).astype(np.int32)
    with open(tmp_path / "gridinput.bin", "wb") as fh:
        fh.write(np.int32(L).tobytes() + oracle.pack_frame(L, g).tobytes())
    env = dict(os.environ, GASP_SEED=str(seed), GASP_L=str(L))
    r = subprocess.run([CLI, str(tot), str(ng), str(mag), str(grid), "32", "0", "2", str(beta),
                        str(h), "1"], cwd=tmp_path, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    r_res, _, _, _ = _ref_driver(ref_gpu, L, ng, seed, beta, h, tot, mag, grid, 1, -0.9, 0.9, 1,
                                 np.repeat(g[None], ng, axis=0))
    assert f"pB estimate : {float(r_res[0]):10.6f}" in r.stdout
    # L mismatch is reported as the reference does, with a failure status
    env["GASP_L"] = str(L + 2)
    r = subprocess.run([CLI, str(tot), str(ng), str(mag), str(grid), "32", "0", "2", str(beta),
                        str(h), "1"], cwd=tmp_path, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode != 0
    assert "does not match L" in r.stderr


@pytest.mark.parametrize("L", [32, 48, 64, 96, 128])
@pytest.mark.parametrize("kind", ["xorwow", "mwc64x"])
@pytest.mark.parametrize("beta,h", [(0.45, 0.1), (0.5, 0.0), (1e-9, 0.1)])
def test_kernel_variants_agree(L, kind, beta, h):
    """The generic (with and without the every-attempt store), row (with
    and without it, in blocks of two or one per loop iteration) and
    bulk-staged kernels give identical results for both RNG kinds (96
    replicas: three tiles).  h = 0 leaves six classes that can reject; at
    beta = 1e-9 every P rounds to 1.0 and ten classes can reject.  The
    retired variants 3, 4 and 8 are refused."""
    ng, seed = 96, 31 + L
    g0 = np.where(np.random.default_rng(seed).random((ng, L, L)) < 0.3, 1, -1).astype(np.int32)
    outs = []
    probe = engine.DeviceGrids(L, ng, g0)
    for variant in (3, 4, 8, 11, -1):
        assert lib().gasp_grids_set_option(probe.handle, 1, variant) != 0
    probe.close()
    for variant in (0, 1, 2, 5, 9, 10):
        dg = engine.DeviceGrids(L, ng, g0)
        dg.set_option(1, variant)
        r = engine.RngStates(ng, seed, kind=kind)
        dg.sweep(r, beta, h, 3)
        dg.sweep(r, beta, h, 2)
        outs.append((dg.download(), dg.magnetisation()))
    for o in outs[1:]:
        assert np.array_equal(outs[0][0], o[0])
        assert np.array_equal(outs[0][1], o[1])
    assert not np.array_equal(outs[0][0], g0)


@pytest.mark.parametrize("compact", [False, True])
def test_bulk_staged_committor_matches_default(compact):
    """Committor shooting through the driver with sweep variant 9: with
    compaction the active lists take the per-lane staging path of the same
    kernel, without it every launch stages whole tiles by bulk copies; fates,
    pB and attempt counts equal variant 0's."""
    L, k, shots = 64, 3, 96
    yy, xx = np.mgrid[0:L, 0:L]
    inputs = np.stack([np.where((yy - L / 2) ** 2 + (xx - L / 2) ** 2 <= r * r, 1, -1)
                       for r in (6.0, 7.0, 8.0)]).astype(np.int32)
    outs = []
    for variant in (0, 9):
        dg = engine.DeviceGrids(L, k * shots)
        dg.upload_inputs(inputs)
        dg.set_option(1, variant)
        rng = engine.RngStates(k * shots, 5, kind="xorwow")
        res, fates, _, att = engine.run_driver(dg, rng, 0.54, 0.07, 3000, 10, 3000, itask=1,
                                               dn_thr=-0.93, up_thr=0.9, ninputs=k,
                                               compact=compact)
        outs.append((np.asarray(res).copy(), fates.copy(), att, dg.download()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2]
    assert np.array_equal(outs[0][3], outs[1][3])


@pytest.mark.parametrize("L,ng", [(64, 40), (96, 33), (128, 1), (32, 65)])
def test_bulk_staged_sweep_ragged(L, ng):
    """Sweep variant 9 (tiles staged by one bulk copy each) on replica counts
    that leave the last tile partly empty: grids, magnetisation and RNG
    states (of the replicas; the padding of the state rows is never written)
    equal the default row kernel's."""
    g0 = np.where(np.random.default_rng(L + ng).random((ng, L, L)) < 0.4, 1, -1).astype(np.int32)
    outs = []
    for variant in (0, 9):
        dg = engine.DeviceGrids(L, ng, g0)
        dg.set_option(1, variant)
        r = engine.RngStates(ng, 7 + ng, kind="xorwow")
        dg.sweep(r, 0.54, 0.07, 4)
        outs.append((dg.download(), dg.magnetisation(), r.read_states()[:, :ng]))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert np.array_equal(outs[0][2], outs[1][2])
    assert not np.array_equal(outs[0][0], g0)
