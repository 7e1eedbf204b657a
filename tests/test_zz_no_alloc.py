"""gasp_grids_upload_inputs_noalloc (fixed device stage, no allocation)
against gasp_grids_upload_inputs, both called through the C ABI.

Kept in its own file, collected after the others, so that it is exercised
both alone in a fresh process and after the rest of the suite has used the
device."""
import numpy as np
import pytest

from gpu_2dising_b200 import engine
from gpu_2dising_b200._native import GASP_ERR_INVALID, GaspError, check, lib

pytestmark = pytest.mark.gpu

STAGE_INTS = 1 << 18  # GASP_NOALLOC_MAX_INPUT_INTS


@pytest.fixture(scope="module", autouse=True)
def device():
    return engine.init_device(0)


def _inputs(rs, n, L):
    return np.where(rs.random((n, L, L)) < 0.5, 1, -1).astype(np.int32)


def _upload(fn, grids, inputs):
    x = np.ascontiguousarray(inputs, np.int32).reshape(-1)
    return fn(grids.handle, x, inputs.shape[0])


@pytest.mark.parametrize("L,nin,per", [(64, 64, 8), (30, 5, 13), (7, 3, 1)])
def test_noalloc_matches_upload_inputs_on_consecutive_calls(L, nin, per):
    """64 inputs at L=64 fill the stage exactly; 30 and 7 leave ragged tiles."""
    rs = np.random.default_rng(L * 1000 + nin)
    ref = engine.DeviceGrids(L, nin * per)
    out = engine.DeviceGrids(L, nin * per)
    for _ in range(2):  # two calls in a row, new inputs each time
        inputs = _inputs(rs, nin, L)
        check(_upload(lib().gasp_grids_upload_inputs, ref, inputs), "upload_inputs")
        check(_upload(lib().gasp_grids_upload_inputs_noalloc, out, inputs), "noalloc")
        expect = ref.download()
        assert np.array_equal(out.download(), expect)
        assert np.array_equal(expect, np.repeat(inputs, per, axis=0))
        assert np.array_equal(out.magnetisation(), ref.magnetisation())


def test_noalloc_sets_sweep_identically():
    """A set seeded by either call evolves bit-identically."""
    L, nin, per, seed = 64, 4, 32, 99
    rs = np.random.default_rng(seed)
    inputs = _inputs(rs, nin, L)
    sets = []
    for fn in (lib().gasp_grids_upload_inputs, lib().gasp_grids_upload_inputs_noalloc):
        g = engine.DeviceGrids(L, nin * per)
        check(_upload(fn, g, inputs))
        g.sweep(engine.RngStates(nin * per, seed), 0.54, 0.07, 3)
        sets.append(g.download())
    assert np.array_equal(sets[0], sets[1])


def test_noalloc_rejects_inputs_above_the_stage():
    L = 64
    nin = STAGE_INTS // (L * L) + 1
    g = engine.DeviceGrids(L, nin)
    before = g.download()
    rs = np.random.default_rng(1)
    rc = _upload(lib().gasp_grids_upload_inputs_noalloc, g, _inputs(rs, nin, L))
    assert rc == GASP_ERR_INVALID
    assert "GASP_NOALLOC_MAX_INPUT_INTS" in lib().gasp_last_error().decode()
    assert np.array_equal(g.download(), before)  # nothing was copied
    # replica count not a multiple of the inputs
    g2 = engine.DeviceGrids(L, 10)
    with pytest.raises(GaspError):
        check(_upload(lib().gasp_grids_upload_inputs_noalloc, g2, _inputs(rs, 3, L)))


def _free_device_bytes():
    """Free device memory as the driver reports it (cuMemGetInfo on the
    context this thread already uses)."""
    import ctypes as C
    cu = C.CDLL("libcuda.so.1")
    free, total = C.c_size_t(), C.c_size_t()
    assert cu.cuMemGetInfo_v2(C.byref(free), C.byref(total)) == 0
    return free.value


def test_noalloc_takes_no_device_memory():
    """The property the entry point exists for: repeated calls leave the
    device's free memory unchanged, on a set that has no int32 buffer of its
    own (the allocating form would stage there or in a new buffer).  The
    set's download then allocates its 64 MiB int32 buffer, which the same
    measurement sees, so the check is able to see an allocation."""
    L, nin, per = 64, 64, 64  # 4096 replicas; their int32 image is 64 MiB
    rs = np.random.default_rng(5)
    g = engine.DeviceGrids(L, nin * per)
    check(_upload(lib().gasp_grids_upload_inputs_noalloc, g, _inputs(rs, nin, L)))  # warm
    before = _free_device_bytes()
    for _ in range(3):
        check(_upload(lib().gasp_grids_upload_inputs_noalloc, g, _inputs(rs, nin, L)))
    assert _free_device_bytes() == before
    g.download()  # allocates the set's int32 image
    assert _free_device_bytes() <= before - nin * per * L * L * 4
