"""The HDF5 side files of PyGASP (gridstates.hdf5 / pBgrids.hdf5,
src/io.c:132-301) written by gasp_create_ising_grids_hdf5 /
gasp_write_ising_grids_hdf5 through the C ABI, read back by tests/h5read.py,
an independent reader written from the HDF5 file format specification that
also checks the structures a conforming reader relies on.  libhdf5 is not
installed here, so the files are not opened by it; the reader itself, and
two of the writer's encodings, are pinned on a file that libhdf5 wrote
(scipy's MATLAB 7.3-format test data, HDF5 after a 512-byte user block)."""
import os
import struct

import numpy as np
import pytest

import h5read
from gpu_2dising_b200._native import GASP_ERR_FORMAT, GASP_ERR_IO, GASP_OK, lib


def _grids(rs, n, L):
    return np.where(rs.random((n, L, L)) < 0.5, 1, -1).astype(np.int32)


def _create(path, L, ng, tot=5000, h=0.07, beta=0.54, itask=0):
    return lib().gasp_create_ising_grids_hdf5(L, ng, tot, h, beta, itask, str(path).encode())


def _write(path, g, isweep, mag=None, lclus=None, cv=b"magnetisation"):
    ng, L = g.shape[0], g.shape[1]
    keep = [np.ascontiguousarray(a, np.float32) if a is not None else None for a in (mag, lclus)]
    ptr = [a.ctypes.data if a is not None else None for a in keep]
    return lib().gasp_write_ising_grids_hdf5(L, ng, np.ascontiguousarray(g).reshape(-1), isweep,
                                             ptr[0], ptr[1], cv, -0.9, 0.9, str(path).encode())


def _attrs(mag, lclus, i):
    return {"magnetisation": "null" if mag is None else "%g" % float(np.float32(mag[i])),
            "lclus_size": "null" if lclus is None else "%g" % float(np.float32(lclus[i])),
            "committor": "null", "committor_error": "null"}


def test_header_scalars_and_superblock(tmp_path):
    p = tmp_path / "gridstates.hdf5"
    assert _create(p, 64, 32768, 50000, 0.07, 0.54) == GASP_OK
    raw = p.read_bytes()
    assert raw[:8] == b"\x89HDF\r\n\x1a\n"
    assert raw[8] == 0 and raw[13] == 8 and raw[14] == 8           # v0, 8-byte offsets
    assert struct.unpack_from("<HH", raw, 16) == (4, 16)             # group K values
    assert struct.unpack_from("<Q", raw, 40)[0] == len(raw)          # end-of-file address
    r = h5read.read(p)
    assert sorted(r) == ["L", "beta", "h", "ngrids", "tot_nsweeps", "total_saved_grids"]
    assert r["L"].value == 64 and r["ngrids"].value == 32768
    assert r["tot_nsweeps"].value == 50000 and r["total_saved_grids"].value == 0
    assert r["h"].value == 0.07 and r["beta"].value == 0.54
    assert r["L"].value.dtype == np.int32 and r["h"].value.dtype == np.float64
    assert r["L"].dtype_desc == {"class": "int", "size": 4, "signed": True, "bit_offset": 0,
                                 "precision": 32}


@pytest.mark.parametrize("L,ng", [(64, 40), (7, 300), (2, 9000)])
def test_dumps_read_back(tmp_path, L, ng):
    """40 grids: one B-tree node; 300: two levels; 9000: three levels and
    18 global heap collections.  Odd L leaves ragged data blocks."""
    p = tmp_path / "f.hdf5"
    rs = np.random.default_rng(L * 7 + ng)
    assert _create(p, L, ng) == GASP_OK
    dumps = []
    for k, isweep in enumerate((0, 1000, 2000)):
        g = _grids(rs, ng, L)
        mag = rs.uniform(-1, 1, ng).astype(np.float32)
        lclus = rs.integers(0, L * L, ng).astype(np.float32) if k == 1 else None
        if k == 2:
            mag[:3] = [1.0, -1.0, 1e-7]
        assert _write(p, g, isweep, mag, lclus) == GASP_OK
        dumps.append((isweep, g, mag, lclus))
    r = h5read.read(p)
    assert r["total_saved_grids"].value == 3 * ng
    assert sorted(k for k in r if k.startswith("sweep_")) == ["sweep_0", "sweep_1000",
                                                            "sweep_2000"]
    for isweep, g, mag, lclus in dumps:
        grp = r[f"sweep_{isweep}"]
        assert len(grp) == ng
        for i in range(ng):
            d = grp[f"grid_{i}"]
            assert d.value.dtype == np.int32 and d.value.shape == (L, L)
            assert np.array_equal(d.value, g[i])
            assert d.attrs == _attrs(mag, lclus, i)
    assert r["sweep_2000"]["grid_2"].attrs["magnetisation"] == "1e-07"


def test_empty_dump_adds_no_group(tmp_path):
    p = tmp_path / "f.hdf5"
    assert _create(p, 8, 4) == GASP_OK
    assert _write(p, np.zeros((0, 8, 8), np.int32), 100) == GASP_OK
    r = h5read.read(p)
    assert "sweep_100" not in r and r["total_saved_grids"].value == 0


def test_errors(tmp_path, capfd):
    rs = np.random.default_rng(3)
    g = _grids(rs, 4, 8)
    missing = tmp_path / "missing.hdf5"
    assert _write(missing, g, 0) == GASP_ERR_IO
    assert "failed to open HDF5 file" in capfd.readouterr().err
    p = tmp_path / "f.hdf5"
    assert _create(p, 8, 4) == GASP_OK
    assert _write(p, g, 10) == GASP_OK
    before = p.read_bytes()
    assert _write(p, g, 10) == GASP_ERR_IO                # the group exists already
    assert "failed to create group '/sweep_10'" in capfd.readouterr().err
    assert p.read_bytes() == before                        # nothing appended
    junk = tmp_path / "junk.hdf5"
    junk.write_bytes(b"\0" * 200)
    assert _write(junk, g, 0) == GASP_ERR_FORMAT
    assert _create(tmp_path / "no_dir" / "x.hdf5", 8, 4) == GASP_ERR_IO
    assert "failed to create HDF5 file" in capfd.readouterr().err


def test_create_truncates(tmp_path):
    p = tmp_path / "f.hdf5"
    rs = np.random.default_rng(9)
    assert _create(p, 8, 4) == GASP_OK
    assert _write(p, _grids(rs, 4, 8), 0) == GASP_OK
    assert _create(p, 16, 2, itask=1) == GASP_OK
    r = h5read.read(p)
    assert "sweep_0" not in r and r["L"].value == 16 and r["ngrids"].value == 2


def _libhdf5_file():
    """scipy's test file testhdf5_7.4_GLNX86.mat: written by MATLAB 7.4 through
    libhdf5 (a 9x1 double dataset 'testdouble' = (0:8) * pi/4 with the
    fixed-length string attribute MATLAB_class = 'double')."""
    try:
        import scipy.io.matlab as sm
    except ImportError:
        return None
    p = os.path.join(os.path.dirname(sm.__file__), "tests", "data", "testhdf5_7.4_GLNX86.mat")
    return p if os.path.exists(p) else None


def _root_symtab(r):
    d = next(d for t, _, d in r.messages(r.root_oh) if t == 0x0011)
    return struct.unpack_from("<QQ", d)


def _root_heap_free_list(r):
    """(free-list head, the first free block's next link or None) of the root
    group's local heap."""
    _, heap = _root_symtab(r)
    size, head, seg = r.u("QQQ", heap + 8)
    nxt = r.u("Q", seg + head)[0] if head < size else None
    return head, nxt


def _entry_header(r, name):
    bt, hp = _root_symtab(r)
    out = []
    r.walk(bt, r.local_heap(hp), out, None, None, None)
    return next(oh for n, oh, _, _ in out if n == name)


def _datatype_message(r, oh):
    return next(d for t, _, d in r.messages(oh) if t == 0x0003)


def test_reader_and_encodings_pinned_on_a_libhdf5_file(tmp_path):
    src = _libhdf5_file()
    if src is None:
        pytest.skip("scipy's HDF5 test file is not installed")
    ref = h5read.H5Read(src)
    content = ref.root()
    assert list(content) == ["testdouble"]
    d = content["testdouble"]
    assert d.value.shape == (9, 1) and d.value.dtype == np.float64
    assert np.allclose(d.value.ravel(), np.arange(9) * np.pi / 4, rtol=0, atol=1e-15)
    assert d.attrs == {"MATLAB_class": "double"}
    # libhdf5 ends a local heap's free list with the value 1; the writer marks
    # "no free block" with the same value
    assert _root_heap_free_list(ref)[1] == 1
    p = tmp_path / "f.hdf5"
    assert _create(p, 8, 4, h=0.25) == GASP_OK
    ours = h5read.H5Read(p)
    assert _root_heap_free_list(ours)[0] == 1
    # the IEEE little-endian double datatype message, byte for byte
    assert (_datatype_message(ours, _entry_header(ours, "h")) ==
            _datatype_message(ref, _entry_header(ref, "testdouble")))
