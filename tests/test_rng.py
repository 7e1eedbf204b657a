"""The production RNG (MWC64X) seeding: states checked on the CPU against an
independent Python statement of the generator and of its skip-ahead."""
import numpy as np

from gpu_2dising_b200 import _native as nat

A = 4294883355
M = A * 2 ** 32 - 1


def mwc_step(x, c):
    t = A * x + c
    return t & 0xFFFFFFFF, t >> 32, x ^ c


def splitmix64(z):
    z = (z + 0x9E3779B97F4A7C15) & (2 ** 64 - 1)
    v = z
    v = ((v ^ (v >> 30)) * 0xBF58476D1CE4E5B9) & (2 ** 64 - 1)
    v = ((v ^ (v >> 27)) * 0x94D049BB133111EB) & (2 ** 64 - 1)
    return v ^ (v >> 31)


def test_skip_ahead_equals_stepping():
    x, c = 2024, 77
    X = x * A + c
    for d in (1, 2, 5, 1000):
        xs, cs = x, c
        for _ in range(d):
            xs, cs, _ = mwc_step(xs, cs)
        Xd = X * pow(A, d, M) % M
        assert (Xd // A, Xd % A) == (xs, cs)


def test_seed_states_are_substreams_2_pow_40_apart():
    n, stride, seed = 70, 96, 123456789
    out = np.zeros(2 * stride, np.uint32)
    assert nat.lib().gasp_mwc64x_seed_states(seed, n, stride, out) == 0
    X0 = 1 + splitmix64(seed) % (M - 1)
    P = pow(A, 2 ** 40, M)
    X = X0
    for r in range(n):
        assert (int(out[r]), int(out[stride + r])) == (X // A, X % A)
        assert int(out[stride + r]) < A
        X = X * P % M
    assert np.all(out[n:stride] == 0)


def test_stream_statistics_are_uniform():
    # first draws of many replicas and many draws of one replica look uniform
    n, stride = 4096, 4096
    out = np.zeros(2 * stride, np.uint32)
    nat.lib().gasp_mwc64x_seed_states(7, n, stride, out)
    firsts = np.array([int(out[r]) ^ int(out[stride + r]) for r in range(n)], np.float64) / 2 ** 32
    x, c = int(out[0]), int(out[stride])
    seq = []
    for _ in range(20000):
        x, c, r = mwc_step(x, c)
        seq.append(r / 2 ** 32)
    for u in (firsts, np.array(seq)):
        hist, _ = np.histogram(u, bins=16, range=(0, 1))
        exp = u.size / 16
        chi2 = float(((hist - exp) ** 2 / exp).sum())
        assert chi2 < 45.0  # 15 dof, p ~ 1e-4
        assert abs(u.mean() - 0.5) < 4 * np.sqrt(1 / 12 / u.size)


def test_surrogate_parameter_layout_matches_oracle():
    from oracle import cnn as ocnn
    from gpu_2dising_b200 import surrogate
    assert surrogate.NPARAM == ocnn.NPARAM == 28097
    assert np.array_equal(surrogate.init_params(11), ocnn.init_params(11))
    assert nat.lib().gasp_cnn_param_count() == 28097
