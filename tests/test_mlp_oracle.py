"""The cost model's CPU oracle: its analytic gradient agrees with central
finite differences (float64)."""
import numpy as np

from oracle import mlp_ref


def test_analytic_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, mlp_ref.NP)
    X = rng.normal(0, 1, (40, 16))
    y = rng.normal(0, 1, 40)
    g = mlp_ref.grad(p, X, y)
    idx = np.concatenate([rng.integers(0, mlp_ref.NP, 60), [mlp_ref.NP - 1]])
    fd = mlp_ref.fd_grad(p, X, y, idx)
    assert np.allclose(g[idx], fd, rtol=1e-5, atol=1e-7)


def test_grouped_longest_first_order():
    """Tasks of one group take the group's largest cost and stay adjacent in
    task order; ties keep task order; without groups every task sorts by its
    own cost."""
    from compression_b200.costmodel import group_max, lpt_order_host
    cost = np.array([1.0, 9.0, 3.0, 3.0, 7.0, 0.5, 8.0, 2.0])
    groups = np.array([0, 1, 2, 2, 2, 3, 4, 4])
    assert np.array_equal(group_max(cost, groups), [1.0, 9.0, 7.0, 7.0, 7.0, 0.5, 8.0, 8.0])
    assert list(lpt_order_host(cost, groups)) == [1, 6, 7, 2, 3, 4, 0, 5]
    assert list(lpt_order_host(cost)) == [1, 6, 4, 2, 3, 7, 0, 5]
    rng = np.random.default_rng(3)
    g = np.repeat(np.arange(200), rng.integers(1, 33, 200))
    c = rng.random(g.size)
    o = lpt_order_host(c, g)
    assert sorted(o) == list(range(g.size))
    pos = np.empty(g.size, np.int64)
    pos[o] = np.arange(g.size)
    for k in range(200):
        p = pos[g == k]
        assert p.max() - p.min() == p.size - 1 and np.all(np.diff(p) == 1)  # together, in task order


def test_banded_order():
    """Bands of a factor of 2 of cost, costliest band first; inside a band
    one codec after another; inside that, costliest first; groups stay
    together."""
    from compression_b200.costmodel import BAND, group_max, lpt_order_host
    rng = np.random.default_rng(4)
    g = np.repeat(np.arange(300), rng.integers(1, 33, 300))
    codec = rng.integers(0, 5, 300)[g]
    cost = rng.uniform(-3.0, 20.0, g.size).astype(np.float32)
    o = lpt_order_host(cost, g, codec)
    assert sorted(o) == list(range(g.size))
    c = group_max(cost, g).astype(np.float32)[o]
    band = np.clip(np.floor(c / np.float32(BAND)), 0, 255)
    assert np.all(np.diff(band) <= 0)
    for b in np.unique(band):
        m = band == b
        cb, cc = c[m], codec[o][m]
        assert np.all(np.diff(cc) >= 0)
        for k in np.unique(cc):
            assert np.all(np.diff(cb[cc == k]) <= 0)
    pos = np.empty(g.size, np.int64)
    pos[o] = np.arange(g.size)
    for k in range(300):
        assert np.all(np.diff(pos[g == k]) == 1)
