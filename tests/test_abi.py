"""The C ABI library loads, exports every symbol include/gasp.h declares, and
its host-only entry points behave like the reference's host code.  CPU only:
no call here launches device work."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from conftest import REPO, has_gpu
from gpu_2dising_b200 import _native as nat


def header_symbols():
    text = open(os.path.join(REPO, "include", "gasp.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gasp_[A-Za-z0-9_]+)\s*\(", text)) - {"gasp_grid_output_fn"})


def test_library_exports_header_symbols():
    lib = nat.lib()
    syms = header_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(nat.EXPORTED)


def test_exports_are_c_linkage():
    out = subprocess.run(["nm", "-D", "--defined-only", nat.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    names = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    for s in header_symbols():
        assert s in names, f"{s} missing or mangled"


def test_status_strings():
    lib = nat.lib()
    assert lib.gasp_status_string(0) == b"ok"
    assert lib.gasp_status_string(nat.GASP_ERR_FORMAT) == b"file format mismatch"
    assert b"sm_100a" in lib.gasp_version()


def test_acceptance_table_matches_oracle():
    for beta, h in [(0.54, 0.07), (0.45, 0.03), (3.0, -0.4)]:
        out = np.zeros(20, np.float32)
        assert nat.lib().gasp_acceptance_table(beta, h, out) == 0
        assert np.array_equal(out, oracle.probs_gpu(beta, h))


def test_init_helpers():
    lib = nat.lib()
    L, ng, ni = 5, 6, 3
    out = np.zeros(L * L * ng, np.int32)
    assert lib.gasp_init_grids_uniform(L, ng, -1, out) == 0 and np.all(out == -1)
    arr = np.where(np.random.default_rng(0).random(ni * L * L) < 0.5, 1, -1).astype(np.int32)
    assert lib.gasp_init_grids_from_array(L, ng, ni, arr, out) == 0
    assert np.array_equal(out.reshape(ng, L * L), np.repeat(arr.reshape(ni, L * L), 2, axis=0))
    assert lib.gasp_init_grids_from_array(L, 7, ni, arr, out) == nat.GASP_ERR_INVALID
    f = np.zeros(ng, np.int32)
    assert lib.gasp_init_fates(ng, f) == 0 and np.all(f == -1)


def test_read_input_grid_errors(tmp_path):
    lib = nat.lib()
    L = 8
    g = np.where(np.random.default_rng(2).random((L, L)) < 0.5, 1, -1).astype(np.int32)
    p = str(tmp_path / "gridinput.bin")
    with open(p, "wb") as fh:
        fh.write(np.int32(L).tobytes() + oracle.pack_frame(L, g).tobytes())
    out = np.zeros(3 * L * L, np.int32)
    assert lib.gasp_read_input_grid(p.encode(), L, 3, out) == 0
    rc, exp = oracle.read_input_grid(p, L, 3)
    assert rc == 0 and np.array_equal(out.reshape(3, L, L), exp)
    assert lib.gasp_read_input_grid(p.encode(), L + 2, 1, out) == nat.GASP_ERR_FORMAT
    assert lib.gasp_read_input_grid(str(tmp_path / "nope.bin").encode(), L, 1, out) == nat.GASP_ERR_IO
    with open(p, "wb") as fh:  # truncated payload
        fh.write(np.int32(L).tobytes() + b"\x01\x02")
    assert lib.gasp_read_input_grid(p.encode(), L, 1, out) == nat.GASP_ERR_IO


def test_write_ising_grids_matches_oracle(tmp_path):
    lib = nat.lib()
    for L, ng in [(8, 3), (5, 3), (64, 2)]:
        g = np.where(np.random.default_rng(L).random(L * L * ng) < 0.5, 1, -1).astype(np.int32)
        a, b = str(tmp_path / f"a{L}.bin"), str(tmp_path / f"b{L}.bin")
        for isw in (0, 100):
            assert lib.gasp_write_ising_grids(L, ng, g, isw, None, None, b"magnetisation", -0.9,
                                              0.9, a.encode()) == 0
            assert oracle.write_frame(b, L, g, isw) == 0
        assert open(a, "rb").read() == open(b, "rb").read()


def test_bootstrap_matches_oracle():
    f = np.random.default_rng(11).choice([-1, 0, 1], size=300).astype(np.int32)
    oracle.lib().orc_srand(3)
    a = nat.lib().gasp_bootstrap_errbar(f.size, f.size, f)
    assert a == oracle.bootstrap_errbar(f, seed=3)


def test_committor_from_fates():
    f = np.array([0, 1, 1, -1, 0, 0, 1, 1, 1], np.int32)
    out = np.zeros(3, np.float32)
    assert nat.lib().gasp_committor_from_fates(9, 3, f, out) == 0
    assert np.array_equal(out, oracle.committor_from_fates(f, 3))
    assert nat.lib().gasp_committor_from_fates(9, 2, f, out) == nat.GASP_ERR_INVALID


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_no_device_is_an_error_not_a_fallback():
    dev, nsms = C.c_int(), C.c_int()
    rc = nat.lib().gasp_init_device(-1, 0, C.byref(dev), C.byref(nsms))
    assert rc == nat.GASP_ERR_NO_DEVICE
    h = C.c_void_p()
    assert nat.lib().gasp_init_grid(16, 4, 32, None, C.byref(h)) != 0


def test_cli_usage_without_args():
    exe = os.path.join(REPO, "gpu_2dising_b200", "gasp")
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode != 0
    assert r.stdout.startswith("Usage : GPU_2DIsing nsweeps nreplicas mag_output_int")
