"""gridstates.bin frame reading and gridinput.bin authoring (host only):
gasp_read_frame against frames written by the oracle's restatement of
write_ising_grids (src/io.c:67-130), gasp_write_input_grid against the
viewer's `w` key output (tools/vis_gridstates.py:109-114) and the oracle's
read_input_grid (src/io.c:4-65), and the headless grid tool."""
import numpy as np
import pytest

import oracle
from gpu_2dising_b200 import engine, gridtool
from gpu_2dising_b200._native import GaspError


def _grids(L, ng, seed):
    rng = np.random.default_rng(seed)
    return np.where(rng.random((ng, L, L)) < 0.4, 1, -1).astype(np.int32)


@pytest.mark.parametrize("L,ng", [(8, 5), (5, 3), (64, 4)])
def test_read_frame_matches_oracle_writer(tmp_path, L, ng):
    path = str(tmp_path / "gridstates.bin")
    frames = [(_grids(L, ng, 10 * L + k), 100 * k) for k in range(3)]
    for g, isw in frames:
        assert oracle.write_frame(path, L, g, isw) == 0
    for k, (g, isw) in enumerate(frames):
        L_, ng_, isw_, got = engine.read_frame(path, k)
        assert (L_, ng_, isw_) == (L, ng, isw)
        assert np.array_equal(got, g)
    with pytest.raises(GaspError):
        engine.read_frame(path, 3)


@pytest.mark.parametrize("L", [8, 5, 64])
def test_write_input_grid_round_trip(tmp_path, L):
    g = _grids(L, 1, L)[0]
    path = str(tmp_path / "gridinput.bin")
    engine.write_input_grid(path, g)
    rc, back = oracle.read_input_grid(path, L, 3)
    assert rc == 0
    assert np.array_equal(back, np.repeat(g[None], 3, axis=0))
    raw = np.fromfile(path, np.uint8)
    assert raw.size == 4 + (L * L + 7) // 8
    assert np.frombuffer(raw[:4].tobytes(), np.int32)[0] == L


def test_extract_equals_viewer_w_key(tmp_path):
    """For L*L % 8 == 0 the viewer writes int32 L followed by the grid's
    slice of the frame payload; the tool writes the same bytes."""
    L, ng, igrid = 16, 6, 4
    frames_path = str(tmp_path / "gridstates.bin")
    g0, g1 = _grids(L, ng, 1), _grids(L, ng, 2)
    oracle.write_frame(frames_path, L, g0, 0)
    oracle.write_frame(frames_path, L, g1, 50)
    out = str(tmp_path / "gridinput.bin")
    got = gridtool.extract(frames_path, 1, igrid, out)
    assert np.array_equal(got, g1[igrid])
    payload = oracle.pack_frame(L, g1)
    per = L * L // 8
    viewer = np.concatenate([np.frombuffer(np.int32(L).tobytes(), np.uint8),
                             payload[igrid * per:(igrid + 1) * per]])
    assert np.array_equal(np.fromfile(out, np.uint8), viewer)


def test_gridtool_cli(tmp_path, capsys):
    L, ng = 8, 3
    path = str(tmp_path / "gridstates.bin")
    for k in range(2):
        oracle.write_frame(path, L, _grids(L, ng, k), 10 * k)
    assert gridtool.main(["info", path]) == 0
    assert "frame     1  isweep         10" in capsys.readouterr().out
    out = str(tmp_path / "in.bin")
    assert gridtool.main(["extract", path, "1", "2", "-o", out]) == 0
    assert "written to" in capsys.readouterr().out
    rc, back = oracle.read_input_grid(out, L, 1)
    assert rc == 0 and np.array_equal(back[0], _grids(L, ng, 1)[2])
    assert gridtool.main(["show", path, "0", "5"]) == 1
    assert gridtool.main(["show", path, "0", "1"]) == 0
    assert capsys.readouterr().out.count("\n") == L + 1
    with pytest.raises(ValueError):
        gridtool.extract(path, 0, 7, out)
