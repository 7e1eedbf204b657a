"""Checkpoint / resume on a B200: a replica set, its RNG states and fates
saved mid-run and loaded into fresh handles continue bit for bit, for both
RNG kinds and through the committor driver."""
import numpy as np
import pytest

from gpu_2dising_b200 import engine

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def device():
    return engine.init_device(0)


@pytest.mark.parametrize("kind", ["xorwow", "mwc64x"])
@pytest.mark.parametrize("L,ng", [(64, 96), (20, 33)])
def test_sweeps_continue_exactly_after_reload(tmp_path, kind, L, ng):
    rs = np.random.default_rng(L + ng)
    g0 = np.where(rs.random((ng, L, L)) < 0.3, 1, -1).astype(np.int32)
    fates = rs.integers(-1, 2, ng).astype(np.int32)
    a = engine.DeviceGrids(L, ng, g0)
    ra = engine.RngStates(ng, 4321, kind=kind)
    a.sweep(ra, 0.5, 0.1, 3)
    path = tmp_path / "run.ckpt"
    engine.save_checkpoint(path, a, ra, fates, isweep=3)
    info = engine.checkpoint_info(path)
    assert info == {"L": L, "ngrids": ng, "rng": kind, "isweep": 3, "has_fates": True}
    b, rb, fb, isw = engine.load_checkpoint(path, seed=999)  # the seed is overwritten
    assert isw == 3 and np.array_equal(fb, fates)
    assert np.array_equal(b.download(), a.download())
    a.sweep(ra, 0.5, 0.1, 4)
    b.sweep(rb, 0.5, 0.1, 4)
    assert np.array_equal(b.download(), a.download())
    assert np.array_equal(b.magnetisation(), a.magnetisation())
    assert not np.array_equal(a.download(), g0)


def test_checkpoint_rejects_other_shapes(tmp_path):
    a = engine.DeviceGrids(16, 32)
    ra = engine.RngStates(32, 1)
    path = tmp_path / "x.ckpt"
    engine.save_checkpoint(path, a, ra)
    assert engine.checkpoint_info(path)["has_fates"] is False
    from gpu_2dising_b200._native import GaspError, lib
    b = engine.DeviceGrids(16, 64)
    rb = engine.RngStates(64, 1)
    with pytest.raises(GaspError):
        from gpu_2dising_b200._native import check
        check(lib().gasp_checkpoint_load(str(path).encode(), b.handle, rb.handle, None, None))
    (tmp_path / "junk.ckpt").write_bytes(b"not a checkpoint at all")
    with pytest.raises(GaspError):
        engine.checkpoint_info(tmp_path / "junk.ckpt")


def test_committor_resumed_from_checkpoint_matches_uninterrupted(tmp_path):
    """Shooting interrupted at a check boundary and resumed from the file gives
    the fates and pB of one uninterrupted run."""
    L, per, seed, beta, h = 32, 64, 77, 0.54, 0.10
    y, x = np.indices((L, L))
    inputs = []
    for r in (3.0, 6.0):
        g = np.where((x - L / 2) ** 2 + (y - L / 2) ** 2 <= r * r, 1, -1)
        inputs.append(g.astype(np.int32))
    inputs = np.stack(inputs)
    ng = per * len(inputs)
    kw = dict(itask=1, dn_thr=-0.9, up_thr=0.5, ninputs=len(inputs), compact=True)
    full = engine.DeviceGrids(L, ng)
    full.upload_inputs(inputs)
    rf = engine.RngStates(ng, seed)
    res_full, fates_full, _, _ = engine.run_driver(full, rf, beta, h, 600, 10, 1000, **kw)

    a = engine.DeviceGrids(L, ng)
    a.upload_inputs(inputs)
    ra = engine.RngStates(ng, seed)
    _, fates_a, _, _ = engine.run_driver(a, ra, beta, h, 200, 10, 1000, **kw)
    path = tmp_path / "shoot.ckpt"
    engine.save_checkpoint(path, a, ra, fates_a, isweep=200)
    b, rb, fb, isw = engine.load_checkpoint(path)
    assert isw == 200
    res_b, fates_b, _, _ = engine.run_driver(b, rb, beta, h, 400, 10, 1000, fates=fb, **kw)
    assert np.array_equal(fates_b, fates_full)
    assert np.array_equal(res_b, res_full)
    assert np.count_nonzero(fates_a == -1) > 0  # the first leg really left work to resume
