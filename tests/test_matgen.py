"""Shapes, sizes and determinism of the synthetic workload generators."""
import numpy as np

from gsofa_b200 import matgen


def _check_graph(g):
    assert g.beg.dtype == np.int32 and g.end.dtype == np.int32 and g.adj.dtype == np.int32
    assert np.all(g.end >= g.beg)
    assert g.adj.min() >= 0 and g.adj.max() < g.n
    # full diagonal, sorted, duplicate-free lines
    for v in np.random.default_rng(0).integers(0, g.n, size=min(g.n, 200)):
        row = g.adj[g.beg[v]:g.end[v]]
        assert v in row
        assert np.all(np.diff(row) > 0)


def test_plain2d_size():
    g = matgen.config_plain2d()
    assert (g.n, g.nnz) == (4096, 20224)
    _check_graph(g)


def test_nd_order_is_a_permutation():
    for dims in [(5, 4, 3), (8, 8, 8), (7, 9), (1, 5, 2)]:
        p = matgen.nested_dissection_order(dims)
        assert np.array_equal(np.sort(p), np.arange(int(np.prod(dims))))


def test_nd_separator_numbered_last():
    dims = (9, 4, 4)
    p = matgen.nested_dissection_order(dims)
    g = np.arange(9 * 16)
    x = g % 9
    # the first cut halves the longest axis (x) at x = 4; that plane gets the last ids
    sep = p[x == 4]
    assert sep.min() == 9 * 16 - 16


def test_grid3d_shape_and_drops():
    g = matgen.grid3d(10, ordering="nd", drop_frac=0.1, seed=2)
    full = 1000 + 2 * 3 * 9 * 100
    pairs = 3 * 9 * 100
    assert g.nnz < full and abs((full - g.nnz) - 0.1 * pairs) < 0.03 * pairs
    _check_graph(g)


def test_powerlaw_degree_and_determinism():
    a = matgen.powerlaw(20000, seed=3)
    b = matgen.powerlaw(20000, seed=3)
    assert np.array_equal(a.adj, b.adj) and np.array_equal(a.beg, b.beg)
    _check_graph(a)
    deg = np.diff(np.append(a.beg, a.nnz)) - 1
    assert 6.5 < deg.mean() < 9.5
    assert deg.max() <= 4000


def test_mixed_specs():
    spec = matgen.config_batch()
    assert len(spec) == 256
    ns = np.array([n for _, n, _ in spec])
    assert ns.min() >= 2000 and ns.max() <= 200000
    assert {k for k, _, _ in spec} == {"grid2d", "grid3d", "powerlaw"}
    stream = matgen.config_serve(count=100)
    t = np.array([a for a, _, _, _ in stream])
    assert np.all(np.diff(t) > 0)
