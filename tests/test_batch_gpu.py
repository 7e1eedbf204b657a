"""Batched groups of uneven L, beta, h on a B200: the graph-captured,
compacting path -- one kernel per group, or all groups in one persistent
launch -- gives exactly the plain per-group path's results."""
import ctypes as C

import numpy as np
import pytest

from gpu_2dising_b200 import _native as nat
from gpu_2dising_b200 import engine

pytestmark = pytest.mark.gpu

GROUPS = [(32, 256, 0.45, 0.12), (48, 128, 0.47, 0.10), (64, 96, 0.46, 0.12),
          (96, 64, 0.50, 0.12), (128, 40, 0.45, 0.12)]


@pytest.fixture(scope="module", autouse=True)
def device():
    return engine.init_device(0)


def _batch(kind="xorwow", groups=GROUPS):
    arr = (nat.GroupT * len(groups))(*[nat.GroupT(L, n, b, h) for L, n, b, h in groups])
    h = C.c_void_p()
    k = nat.RNG_XORWOW if kind == "xorwow" else nat.RNG_MWC64X
    nat.check(nat.lib().gasp_batch_create(arr, len(groups), 4242, k, C.byref(h)), "batch_create")
    return h


def _swarm(h, ngroups, tot, chk, up, mode):
    counts = np.zeros((tot // chk) * ngroups, np.int32)
    att = C.c_longlong()
    el = C.c_double()
    nat.check(nat.lib().gasp_batch_swarm(h, tot, chk, up, mode, counts, C.byref(att), C.byref(el)),
              "batch_swarm")
    return counts.reshape(tot // chk, ngroups), att.value, el.value


@pytest.mark.parametrize("kind", ["xorwow", "mwc64x"])
def test_graph_batch_equals_plain(kind):
    h = _batch(kind)
    try:
        tot, chk, up = 400, 10, 0.5
        cp, ap, _ = _swarm(h, len(GROUPS), tot, chk, up, nat.BATCH_PLAIN)
        cg, ag, _ = _swarm(h, len(GROUPS), tot, chk, up, nat.BATCH_GRAPH)
        assert np.array_equal(cp, cg)
        assert ap == ag
        assert cp[-1].sum() > 0  # some replicas nucleated ...
        assert np.all(np.diff(cp, axis=0) >= 0)  # ... absorbingly
        # a second graph run (graph reused) reproduces the first
        cg2, ag2, _ = _swarm(h, len(GROUPS), tot, chk, up, nat.BATCH_GRAPH)
        assert np.array_equal(cg, cg2) and ag == ag2
        # all groups in one persistent launch: the same trajectories, twice
        for _ in range(2):
            cm, am, _ = _swarm(h, len(GROUPS), tot, chk, up, nat.BATCH_MULTI)
            assert np.array_equal(cp, cm) and ap == am
    finally:
        nat.lib().gasp_batch_free(h)


def test_batch_matches_single_group_driver():
    """Group g of a batch follows the same trajectories as the single-set
    kernels seeded the same way (seed + 1000003*g)."""
    h = _batch("xorwow", GROUPS[:2])
    try:
        tot, chk, up = 200, 10, 0.5
        cg, _, _ = _swarm(h, 2, tot, chk, up, nat.BATCH_GRAPH)
    finally:
        nat.lib().gasp_batch_free(h)
    for g, (L, n, beta, hh) in enumerate(GROUPS[:2]):
        dg = engine.DeviceGrids(L, n, -np.ones((n, L, L), np.int32))
        rng = engine.RngStates(n, 4242 + 1000003 * g)
        done = np.zeros(n, bool)
        for i in range(tot // chk):
            dg.sweep(rng, beta, hh, chk)
            done |= dg.magnetisation().astype(np.float64) > up
            assert cg[i, g] == done.sum()


def test_autotune_choices_valid():
    h = _batch("mwc64x")
    try:
        choice = np.zeros(2 * len(GROUPS), np.int32)
        nat.check(nat.lib().gasp_batch_autotune(h, 2, choice), "autotune")
        for g, (L, *_r) in enumerate(GROUPS):
            v, w = choice[2 * g], choice[2 * g + 1]
            assert v in (0, 2) and 1 <= w <= 8
        t0, t1 = C.c_float(), C.c_float()
        layout = nat.lib().gasp_batch_layout(h, C.byref(t0), C.byref(t1))
        assert layout in (0, 1) and t0.value > 0 and t1.value > 0
        assert layout == (1 if t1.value < t0.value else 0)
        c, a, _ = _swarm(h, len(GROUPS), 100, 10, 0.5, nat.BATCH_GRAPH)
        cp, ap, _ = _swarm(h, len(GROUPS), 100, 10, 0.5, nat.BATCH_PLAIN)
        assert a > 0 and a == ap and np.array_equal(c, cp)
    finally:
        nat.lib().gasp_batch_free(h)
