"""Host-side pieces of the surrogate pipeline (no GPU): the training
augmentation draws one of the 8 symmetries of the square per grid."""
import numpy as np

from gpu_2dising_b200.surrogate import _augment


def _symmetries(x):
    out = []
    for k in range(4):
        r = np.rot90(x, k)
        out.append(r)
        out.append(r[:, ::-1])
    return out


def test_augment_applies_one_square_symmetry_per_grid():
    rs = np.random.default_rng(0)
    x = rs.integers(-1, 2, size=(200, 6, 6)).astype(np.int8)
    y = _augment(x, np.random.default_rng(1))
    assert y.shape == x.shape and y.dtype == x.dtype
    seen = set()
    for a, b in zip(x, y):
        hits = [i for i, s in enumerate(_symmetries(a)) if np.array_equal(s, b)]
        assert hits, "not a symmetry of the input"
        seen.add(hits[0])
    assert len(seen) == 8  # all eight are drawn
    # magnetisation (hence the physics) unchanged
    assert np.array_equal(x.reshape(200, -1).sum(1), y.reshape(200, -1).sum(1))
