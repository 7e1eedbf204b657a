"""The one-warp-per-replica sweep (variant 6) on the CPU: its lane substream
multipliers, and the oracle's serial statement of the kernel checked against
an independent Python statement, against the claim the kernel rests on (each
round's attempts can be applied at once) and for the statistics of the
attempts it applies (uniform sites, no bias against neighbouring pairs)."""
import numpy as np
import pytest

from gpu_2dising_b200 import _native as nat

import oracle

A = 4294883355
M = A * 2 ** 32 - 1


def lane_tables():
    mul = np.zeros(32, np.uint64)
    inv = np.zeros(32, np.uint64)
    assert nat.lib().gasp_mwc64x_lane_multipliers(mul, inv) == 0
    return mul, inv


def test_lane_multipliers():
    mul, inv = lane_tables()
    for j in range(32):
        assert int(mul[j]) == pow(A, j << 35, M)
        assert int(inv[j]) == pow(2 ** 32, j << 35, M)
        assert int(mul[j]) * int(inv[j]) % M == 1


def _thr(beta=0.54, h=0.07):
    # any monotone thresholds exercise the logic; these follow exp(-beta dE)
    thr = np.zeros(10, np.uint32)
    for spin01 in (0, 1):
        s = 2 * spin01 - 1
        for up in range(5):
            nsum = 2 * up - 4
            p = np.exp(-beta * 2.0 * s * (nsum + h))
            thr[5 * spin01 + up] = min(int(p * 2 ** 32), 2 ** 32 - 1)
    return thr


def _mwc(x, c):
    t = A * x + c
    return t & 0xFFFFFFFF, t >> 32, x ^ c


def _adjacent(L, a, b):
    ra, ca, rb, cb = a // L, a % L, b // L, b % L
    if ra == rb:
        return cb == (ca + 1) % L or ca == (cb + 1) % L
    if ca == cb:
        return rb == (ra + 1) % L or ra == (rb + 1) % L
    return False


def _apply(L, g, s, u, thr, src=None):
    src = g if src is None else src
    r, c = divmod(s, L)
    up = sum(int(src[(r + dr) % L, (c + dc) % L] > 0)
             for dr, dc in ((1, 0), (-1, 0), (0, 1), (0, -1)))
    if u <= thr[5 * int(src[r, c] > 0) + up]:
        g[r, c] = -src[r, c]


def python_tail(L, grid, nsweeps, x, c, thr, check_rounds=False):
    """Independent statement of the variant-6 sweep (window, conflict rule,
    lane draws, state afterwards); optionally checks every round's parallel
    application against the serial one."""
    mul, inv = lane_tables()
    N, Q = L * L, nsweeps * L * L
    X = x * A + c
    lanes, ahead = [], []

    def pair(j):
        lx, lc, n = lanes[j]
        lx, lc, r1 = _mwc(lx, lc)
        lx, lc, r2 = _mwc(lx, lc)
        lanes[j] = [lx, lc, n + 2]
        return (r1 * N) >> 32, r2

    for j in range(32):
        Xj = X * int(mul[j]) % M
        lanes.append([Xj // A, Xj % A, 0])
        ahead.append(pair(j))  # each lane keeps its next attempt drawn

    def draw(j):
        got = ahead[j]
        ahead[j] = pair(j)
        return got

    g = grid.reshape(L, L)
    win = [draw(j) if j < min(Q, 32) else None for j in range(32)]
    head, pend, drawn, done, order = 0, min(Q, 32), min(Q, 32), 0, []
    while done < Q:
        flagged = [w is not None and any(
            i != j and v is not None and (v[0] == w[0] or _adjacent(L, v[0], w[0]))
            for i, v in enumerate(win)) for j, w in enumerate(win)]
        k = 32
        for p in range(32):
            if flagged[(head + p) % 32]:
                k = p + 1
                break
        k = min(k, pend)
        batch = [win[(head + p) % 32] for p in range(k)]
        if check_rounds:
            par = g.copy()
            before = g.copy()
            for s, u in batch:
                _apply(L, par, s, u, thr, src=before)
        for s, u in batch:
            _apply(L, g, s, u, thr)
            order.append((s, u))
        if check_rounds:
            assert np.array_equal(par, g)
        done += k
        head = (head + k) % 32
        pend -= k
        nnew = min(32 - pend, Q - drawn)
        for j in range(32):
            p2 = (j - head) % 32
            if p2 >= pend:
                win[j] = draw(j) if p2 - pend < nnew else None
        pend += nnew
        drawn += nnew
    js = max(range(32), key=lambda j: (lanes[j][2], -j))
    Xb = (lanes[js][0] * A + lanes[js][1]) * int(inv[js]) % M
    return Xb // A, Xb % A, order


@pytest.mark.parametrize("L,nsweeps", [(8, 2), (5, 3), (16, 1)])
def test_oracle_tail_matches_python_statement(L, nsweeps):
    rs = np.random.default_rng(L)
    g0 = np.where(rs.random((L, L)) < 0.4, 1, -1).astype(np.int32)
    x, c = 123456789, 98765
    thr = _thr()
    mul, inv = lane_tables()
    g1 = g0.copy().reshape(-1)
    x1, c1, order1 = oracle.sweep_tail(L, g1, nsweeps, x, c, thr, mul, inv, record=True)
    g2 = g0.copy()
    x2, c2, order2 = python_tail(L, g2, nsweeps, x, c, thr, check_rounds=True)
    assert np.array_equal(g1.reshape(L, L), g2)
    assert (x1, c1) == (x2, c2)
    assert [tuple(map(int, o)) for o in order1] == order2


def test_replica_stream_advances_past_every_lane_segment():
    L, thr = 6, _thr()
    mul, inv = lane_tables()
    x, c = 42, 4242
    g = -np.ones(L * L, np.int32)
    for _ in range(3):
        X = x * A + c
        x2, c2 = oracle.sweep_tail(L, g, 1, x, c, thr, mul, inv)
        # the new state is the old one advanced by a whole number of draws
        # at least as large as any lane's: find it by stepping
        xs, cs, steps = x, c, 0
        while (xs, cs) != (x2, c2):
            xs, cs, _ = _mwc(xs, cs)
            steps += 1
            assert steps <= 2 * L * L
        assert steps >= 2 * (L * L + 31) // 32  # >= the average lane's share
        assert X * pow(A, steps, M) % M == x2 * A + c2
        x, c = x2, c2


def test_applied_attempts_are_uniform_and_unbiased():
    """The sites of applied attempts are uniform and consecutive applied
    sites are neighbours or equal with probability 5/N, as for i.i.d. draws
    (a rule that dropped or reordered conflicting attempts would show here)."""
    L, nsweeps = 16, 80
    N = L * L
    thr = _thr()
    mul, inv = lane_tables()
    g = np.where(np.random.default_rng(3).random(N) < 0.5, 1, -1).astype(np.int32)
    _, _, order = oracle.sweep_tail(L, g, nsweeps, 7, 77, thr, mul, inv, record=True)
    sites = order[:, 0].astype(np.int64)
    hist = np.bincount(sites, minlength=N)
    exp = sites.size / N
    chi2 = float(((hist - exp) ** 2 / exp).sum())
    assert chi2 < N + 6 * np.sqrt(2 * N)
    near = np.array([s == t or _adjacent(L, int(s), int(t)) for s, t in zip(sites[:-1], sites[1:])])
    p = 5 / N
    z = (near.mean() - p) / np.sqrt(p * (1 - p) / near.size)
    assert abs(z) < 4.5, z
    u = order[:, 1].astype(np.float64) / 2 ** 32
    assert abs(u.mean() - 0.5) < 5 * np.sqrt(1 / 12 / u.size)


def test_serial_mwc_oracle_consumes_two_draws_per_attempt():
    L, thr = 8, _thr()
    g = -np.ones(L * L, np.int32)
    x, c = oracle.sweep_mwc(L, g, 100, 5, 6, thr)
    xs, cs = 5, 6
    for _ in range(200):
        xs, cs, _ = _mwc(xs, cs)
    assert (x, c) == (xs, cs)


def python_shared(L, grids, nsweeps, xs, cs, thr):
    """Independent statement of the shared-site sweep (variant 7) on a tile."""
    n, N = grids.shape[0], L * L
    xs, cs = [int(v) for v in xs], [int(v) for v in cs]
    j, sites = 0, [0] * n
    for _ in range(nsweeps * N):
        if j == 0:
            for r in range(n):
                xs[r], cs[r], v = _mwc(xs[r], cs[r])
                sites[r] = (v * N) >> 32
        s = sites[j]
        j = (j + 1) % n
        for r in range(n):
            xs[r], cs[r], u = _mwc(xs[r], cs[r])
            _apply(L, grids[r], s, u, thr)
    return xs, cs


def test_shared_site_oracle_matches_python_statement():
    L, n, thr = 6, 5, _thr()
    rs = np.random.default_rng(9)
    g0 = np.where(rs.random((n, L, L)) < 0.4, 1, -1).astype(np.int32)
    x0 = rs.integers(1, 2 ** 32 - 1, n).astype(np.uint32)
    c0 = rs.integers(0, A - 1, n).astype(np.uint32)
    g1 = g0.copy()
    x1, c1 = oracle.sweep_shared(L, g1, 3, x0, c0, thr)
    g2 = g0.copy()
    x2, c2 = python_shared(L, g2, 3, x0, c0, thr)
    assert np.array_equal(g1, g2)
    assert [int(v) for v in x1] == x2 and [int(v) for v in c1] == c2


def test_shared_site_tile_of_one_is_the_serial_sweep():
    """A one-replica tile draws site then acceptance per attempt: exactly the
    one-stream serial sweep."""
    L, thr = 8, _thr()
    g = np.where(np.random.default_rng(4).random((1, L, L)) < 0.5, 1, -1).astype(np.int32)
    g2 = g[0].copy().reshape(-1)
    xs, cs = oracle.sweep_shared(L, g, 4, [77], [7], thr)
    x2, c2 = oracle.sweep_mwc(L, g2, 4 * L * L, 77, 7, thr)
    assert np.array_equal(g[0].reshape(-1), g2)
    assert (int(xs[0]), int(cs[0])) == (x2, c2)
