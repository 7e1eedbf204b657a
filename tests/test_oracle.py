"""Pins the CPU oracle against the reference's own code (oracle/_ref, compiled
unmodified) and against the committed golden fixtures.  CPU only."""
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN


def test_tables_cpu_match_golden():
    d = np.load(os.path.join(GOLDEN, "ref_cpu_tables.npz"))
    for (beta, h), P in zip(d["cases"], d["pacc"]):
        assert np.array_equal(oracle.probs_cpu(beta, h), P)


def test_tables_cpu_match_reference(ref_cpu):
    for beta, h in [(0.54, 0.07), (0.1, 1.3), (2.5, -0.2)]:
        P = np.zeros(20)
        ref_cpu.ref_precompute_probs_cpu(beta, h, P)
        assert np.array_equal(oracle.probs_cpu(beta, h), P)


def test_table_gpu_shape():
    # float table: index 5*(s+1)+nsum+4, only even slots used (src/mc_gpu.cu:26-31)
    P = oracle.probs_gpu(0.54, 0.07)
    assert P.dtype == np.float32
    assert np.all(P[1::2] == 0)
    assert np.isclose(P[8], np.exp(-0.54 * 2 * -1 * (4 + 0.07)), rtol=1e-6)
    assert np.isclose(P[18], np.exp(-0.54 * 2 * (4 + 0.07)), rtol=1e-6)


def test_mt_stream_matches_reference(ref_cpu):
    ref_cpu.ref_init_genrand(31415)
    a = np.array([ref_cpu.ref_genrand_real3() for _ in range(3000)])
    assert np.array_equal(a, oracle.mt_real3_stream(31415, 3000))
    m = oracle.MTReal3(31415)
    b = np.concatenate([m.take(1000), m.take(2000)])
    assert np.array_equal(a, b)


@pytest.mark.parametrize("L,ng,nsw", [(8, 3, 4), (16, 2, 3), (12, 2, 2)])
def test_sweep_cpu_matches_reference(ref_cpu, L, ng, nsw):
    rng = np.random.default_rng(L)
    g0 = np.where(rng.random((ng, L, L)) < 0.4, 1, -1).astype(np.int32)
    beta, h = 0.5, 0.1
    gref = g0.copy().reshape(-1)
    ref_cpu.ref_init_genrand(55)
    for i in range(ng):
        ref_cpu.ref_sweep_cpu(L, gref, i, beta, h, nsw)
    mt = oracle.MTReal3(55)
    P = oracle.probs_cpu(beta, h)
    gor = g0.copy()
    for i in range(ng):
        x = np.ascontiguousarray(gor[i]).reshape(-1)
        oracle.sweep_cpu_stream(L, x, mt.take(3 * L * L * nsw), P)
        gor[i] = x.reshape(L, L)
    assert np.array_equal(gor.reshape(-1), gref)
    # magnetisation flavours agree with the reference
    for i in range(ng):
        assert oracle.magnetisation_cpu(L, gor[i])[0] == ref_cpu.ref_magnetisation_cpu(L, gref, i)


def _golden_cases():
    d = np.load(os.path.join(GOLDEN, "ref_cpu_driver.npz"))
    return d, list(d["names"])


def _case(d, name):
    return {k.split("__", 1)[1]: d[k] for k in d.files if k.startswith(name + "__")}


@pytest.mark.parametrize("name", _golden_cases()[1])
def test_cpu_driver_restatement_matches_golden(name):
    d, _ = _golden_cases()
    c = _case(d, name)
    L, ng = int(c["L"]), int(c["ngrids"])
    beta, h = float(c["beta"]), float(c["h"])
    P = oracle.probs_cpu(beta, h)
    mt = oracle.MTReal3(int(c["seed"]))
    grids = c["initial"].astype(np.int32).copy()

    def sweep_batch(g, batch, spc):
        s = mt.batch(ng, L, spc)
        for i in range(ng):
            x = np.ascontiguousarray(g[i]).reshape(-1)
            oracle.sweep_cpu_stream(L, x, s[i], P)
            g[i] = x.reshape(L, L)

    tr = oracle.driver_cpu_semantics(grids, sweep_batch, lambda g: oracle.magnetisation_cpu(L, g),
                                     int(c["tot"]), int(c["mag"]), int(c["grid"]),
                                     itask=int(c["itask"]), up=float(c["up"]), dn=float(c["dn"]),
                                     ninputs=int(c["ninputs"]))
    assert np.array_equal(tr.result, c["result"])
    assert np.array_equal(grids, c["final"].astype(np.int32))
    assert [d_[0] for d_ in tr.dumps] == list(c["frame_isweep"])
    for (isw, g, m), fg, fm in zip(tr.dumps, c["frame_grids"], c["frame_mag"]):
        assert np.array_equal(g, fg.astype(np.int32))
        assert np.array_equal(m, fm)
    if int(c["itask"]) == 1:
        assert np.array_equal(tr.fates, c["fates"])


def test_bootstrap_restatement_matches_golden():
    d = np.load(os.path.join(GOLDEN, "ref_bootstrap.npz"))
    for i, e in enumerate(d["errbar"]):
        assert oracle.bootstrap_errbar(d[f"fates{i}"], seed=1) == e


def test_bootstrap_restatement_matches_reference(ref_cpu):
    f = np.random.default_rng(9).choice([-1, 0, 1], size=50).astype(np.int32)
    oracle.lib().orc_srand(7)
    ref = ref_cpu.ref_bootstrap_errbar(f.size, f.size, f)
    assert oracle.bootstrap_errbar(f, seed=7) == ref


def test_init_from_array_matches_reference(ref_cpu):
    L, ng, ni = 6, 6, 3
    arr = np.where(np.random.default_rng(1).random((ni, L, L)) < 0.5, 1, -1).astype(np.int32)
    out = np.zeros(ng * L * L, np.int32)
    ref_cpu.ref_init_grids_from_array(L, ng, ni, arr.reshape(-1), out)
    exp = np.repeat(arr, ng // ni, axis=0)
    assert np.array_equal(out.reshape(ng, L, L), exp)


def test_frame_format_matches_viewer_spec(tmp_path):
    # tools/vis_gridstates.py:44-83 reads 12 header bytes then L*L/8 bytes per
    # grid, unpacking bits little-endian row by row.
    L, ng = 8, 3
    g = np.where(np.random.default_rng(3).random((ng, L, L)) < 0.5, 1, -1).astype(np.int32)
    path = str(tmp_path / "gridstates.bin")
    assert oracle.write_frame(path, L, g, 123) == 0
    raw = np.fromfile(path, np.uint8)
    hdr = np.frombuffer(raw[:12].tobytes(), np.int32)
    assert list(hdr) == [L, ng, 123]
    for i in range(ng):
        buf = raw[12 + i * (L * L // 8):12 + (i + 1) * (L * L // 8)]
        bits = np.unpackbits(buf, bitorder="little")
        assert np.array_equal(np.where(bits == 1, 1, -1).reshape(L, L), g[i])
    frames = oracle.read_gridstates(path)
    assert frames[0][2] == 123 and np.array_equal(frames[0][3], g)


def test_frame_format_ragged(tmp_path):
    # L*L*ngrids not a multiple of 8: one running bit cursor (src/io.c:103-117)
    L, ng = 5, 3
    g = np.where(np.random.default_rng(4).random((ng, L, L)) < 0.5, 1, -1).astype(np.int32)
    payload = oracle.pack_frame(L, g)
    assert payload.size == (L * L * ng + 7) // 8
    assert np.array_equal(oracle.unpack_frame(L, ng, payload), g)


def test_read_input_grid(tmp_path):
    L = 6
    g = np.where(np.random.default_rng(8).random((L, L)) < 0.5, 1, -1).astype(np.int32)
    path = str(tmp_path / "gridinput.bin")
    with open(path, "wb") as f:
        f.write(np.int32(L).tobytes())
        f.write(oracle.pack_frame(L, g).tobytes())
    rc, out = oracle.read_input_grid(path, L, 3)
    assert rc == 0 and all(np.array_equal(o, g) for o in out)
    rc, _ = oracle.read_input_grid(path, L + 1, 1)
    assert rc == -2
    rc, _ = oracle.read_input_grid(str(tmp_path / "missing.bin"), L, 1)
    assert rc == -1


def _cluster_golden():
    d = np.load(os.path.join(GOLDEN, "ref_cluster.npz"))
    for L in d["Ls"]:
        yield int(L), d[f"L{L}_grids"].astype(np.int32), d[f"L{L}_sizes"]


def test_largest_cluster_restatement_matches_golden():
    for L, g, sizes in _cluster_golden():
        for k, spin in enumerate((1, -1)):
            assert np.array_equal(oracle.largest_cluster(L, g, spin), sizes[k]), (L, spin)


def test_largest_cluster_restatement_matches_reference(ref_cpu):
    rng = np.random.default_rng(8)
    for L in (4, 7, 20, 45):
        g = np.where(rng.random((6, L, L)) < 0.59, 1, -1).astype(np.int32)
        flat = np.ascontiguousarray(g.reshape(-1))
        for spin in (1, -1):
            ref = np.zeros(6, np.float32)
            for i in range(6):
                ref_cpu.compute_largest_cluster_cpu(L, flat, i, spin, ref)
            assert np.array_equal(oracle.largest_cluster(L, g, spin), ref)


def test_largest_cluster_known_answers():
    L = 6
    g = -np.ones((1, L, L), np.int32)
    assert oracle.largest_cluster(L, g, 1)[0] == 0
    assert oracle.largest_cluster(L, g, -1)[0] == L * L
    g[0, :, 0] = 1  # a column: connected through the periodic wrap in y
    g[0, 2, L - 1] = 1  # joins the column through the wrap in x
    assert oracle.largest_cluster(L, g, 1)[0] == L + 1
    assert oracle.largest_cluster(L, g, 0)[0] == 0
