"""The radiance-cache oracle checked against itself: its float64 backward pass against
central finite differences of its loss, and its BF16-emulating mode against float64."""
import numpy as np

from oracle import nrc


def _loss(records, mlp, table, target, den):
    # The relative-L2 denominator is a stopped gradient: hold it at the unperturbed y.
    x = nrc.encode(records, table, emulate=False)
    y, _ = nrc.forward(x, mlp, emulate=False)
    return float(((y - target) ** 2 / den).sum() / (3 * y.shape[0]))


def test_backward_matches_finite_differences():
    rec = nrc.random_records(24, seed=1)
    mlp, table = nrc.random_params(seed=2)
    mlp = mlp.astype(np.float64); table = table.astype(np.float64)
    target = np.abs(np.random.default_rng(3).normal(size=(24, 3)))
    loss, g, hg, y = nrc.backward(rec, mlp, table, target, emulate=False)
    den = y * y + nrc.LOSS_EPS
    rng = np.random.default_rng(4)
    eps = 1e-6
    # MLP parameters: every layer, including the output layer's live rows.
    picks = list(rng.integers(0, 4 * 64 * 64, 12)) + list(4 * 64 * 64 + rng.integers(0, 3 * 64, 4))
    for p in picks:
        m1 = mlp.copy(); m1[p] += eps
        m0 = mlp.copy(); m0[p] -= eps
        fd = (_loss(rec, m1, table, target, den) - _loss(rec, m0, table, target, den)) / (2 * eps)
        assert abs(fd - g[p]) <= 1e-6 + 1e-4 * abs(fd), (p, fd, g[p])
    # Hash entries that the records touch.
    nz = np.flatnonzero(np.abs(hg.reshape(-1)) > 1e-8)
    for p in rng.choice(nz, 12, replace=False):
        t1 = table.copy(); t1[p] += eps
        t0 = table.copy(); t0[p] -= eps
        fd = (_loss(rec, mlp, t1, target, den) - _loss(rec, mlp, t0, target, den)) / (2 * eps)
        assert abs(fd - hg.reshape(-1)[p]) <= 1e-7 + 1e-4 * abs(fd), (p, fd, hg.reshape(-1)[p])
    # Output rows 3..15 are not parameters.
    assert not np.any(g[4 * 64 * 64 + 3 * 64:])


def test_emulated_rounding_stays_close_to_float64():
    rec = nrc.random_records(256, seed=5)
    mlp, table = nrc.random_params(seed=6)
    target = np.abs(np.random.default_rng(7).normal(size=(256, 3)))
    l64, g64, h64, y64 = nrc.backward(rec, mlp, table, target, emulate=False)
    l16, g16, h16, y16 = nrc.backward(rec, mlp, table, target, emulate=True)
    assert abs(l16 - l64) <= 0.02 * l64
    # BF16 deltas through four layers: a few per cent on the gradients.
    assert np.linalg.norm(g16 - g64) <= 0.1 * np.linalg.norm(g64)
    assert np.linalg.norm(h16 - h64) <= 0.1 * np.linalg.norm(h64)


def test_hash_levels_and_indices():
    assert [int(nrc.level_scale(l)) for l in range(16)] == [16, 22, 30, 42, 58, 80, 111, 153, 212, 294, 406, 561, 776, 1072, 1482, 2048]
    # Dense levels index the grid directly; hashed levels stay inside the table.
    for level, (idx, w) in enumerate(nrc.corners(np.random.default_rng(0).uniform(0, 1, (1000, 3)))):
        assert idx.min() >= 0 and idx.max() < nrc.T
        assert np.allclose(w.sum(1), 1.0)
