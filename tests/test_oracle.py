"""The CPU oracle against the reference's golden values and against itself.

The oracle holds two restatements of the fill computation: the reference's
max-id label propagation, and the two-pass reachability form the GPU library
implements.  Both are pinned to the reference's logged fill total on its
bundled matrix before either is trusted as the GPU's checker."""

import numpy as np
import pytest

import oracle
from gsofa_b200 import matgen
from tests.common import bundled, expected, lower_rows, random_graph


def test_bundled_matrix_matches_reference_log():
    g = bundled()
    exp = expected()["bundled_11948"]
    assert (g.n, g.nnz) == (exp["n"], exp["nnz"])
    tot, lo, hi = oracle.maxid_fills(g.beg, g.end, g.adj)
    assert tot == exp["fill_count"]
    assert int(lo.sum()) == exp["fill_lower"] and int(hi.sum()) == exp["fill_upper"]
    r = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False)
    assert r["fill_count"] == exp["fill_count"]
    assert r["nnz_lu"] == exp["nnz_lu"]


def test_grid2d_64_natural_matches_band_count():
    g = matgen.config_plain2d()
    exp = expected()["grid2d_64x64_natural"]
    assert (g.n, g.nnz) == (exp["n"], exp["nnz"])
    r = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False)
    assert r["fill_count"] == exp["fill_count"]
    assert r["nnz_lu"] == exp["nnz_lu"]
    tot, _, _ = oracle.maxid_fills(g.beg, g.end, g.adj)
    assert tot == exp["fill_count"]


def _line_fills_twopass(g, r, s):
    """Fills of line s from the two-pass result: (U row s u L row s) minus the
    original entries and the diagonal."""
    lp, lc = r["_lrows"]
    row = set(r["u_idx"][r["u_ptr"][s]:r["u_ptr"][s + 1]].tolist())
    row |= set(lc[lp[s]:lp[s + 1]].tolist())
    row -= set(g.adj[g.beg[s]:g.end[s]].tolist())
    row.discard(s)
    return sorted(row)


@pytest.mark.parametrize("seed", range(12))
def test_maxid_and_twopass_agree_line_by_line(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 70))
    g = random_graph(n, float(rng.choice([0.02, 0.05, 0.1, 0.3])), seed)
    r = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=True)
    r["_lrows"] = lower_rows(r["l_ptr"], r["l_idx"], n)
    tot, lo, hi = oracle.maxid_fills(g.beg, g.end, g.adj)
    assert tot == r["fill_count"]
    for s in range(n):
        f = oracle.maxid_line(g.beg, g.end, g.adj, s)
        assert f.tolist() == _line_fills_twopass(g, r, s), (seed, s)
        assert int(lo[s]) == sum(1 for j in f if j < s)
        assert int(hi[s]) == sum(1 for j in f if j > s)


def _all_digraphs(n):
    pairs = [(i, j) for i in range(n) for j in range(n) if i != j]
    for mask in range(1 << len(pairs)):
        rows = [[] for _ in range(n)]
        for b, (i, j) in enumerate(pairs):
            if mask >> b & 1:
                rows[i].append(j)
        yield rows


def _graph_from_rows(rows):
    n = len(rows)
    ptr = np.zeros(n + 1, np.int64)
    ptr[1:] = np.cumsum([len(r) for r in rows])
    adj = np.array([c for r in rows for c in r], np.int32)
    return matgen.Graph.from_csr(ptr, adj)


@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_exhaustive_small_digraphs(n):
    """Every directed pattern on n <= 4 vertices (4,096 of them at n = 4)."""
    for rows in _all_digraphs(n):
        g = _graph_from_rows(rows)
        tot, lo, hi = oracle.maxid_fills(g.beg, g.end, g.adj, nthreads=1)
        r = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False, nthreads=1)
        assert tot == r["fill_count"], rows


def test_supernode_scan_definition():
    # lines 0..5; link flags and counts chosen by hand
    ucnt = np.array([3, 2, 1, 0, 2, 1], np.int32)
    unext = np.array([1, 1, 1, 0, 1, 0], np.uint8)
    lnext = np.array([1, 1, 0, 0, 1, 0], np.uint8)
    assert oracle.supernodes(ucnt, unext, lnext, 0).tolist() == [0, 3, 4]
    assert oracle.supernodes(ucnt, unext, lnext, 2).tolist() == [0, 2, 3, 4]
    assert oracle.supernodes(ucnt, unext, lnext, 1).tolist() == [0, 1, 2, 3, 4, 5]


def test_partitions_sum_to_total():
    """The reference's virtual-GPU partitions (sources s = g + t*N) leave the
    total unchanged (log lines 122-161 show this for 6 and 264 partitions)."""
    g = bundled()
    full = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False)
    n = g.n
    for parts in (6, 264):
        tot = 0
        for p in range(parts):
            src = np.arange(p, n, parts, dtype=np.int32)
            c0, o0, _, _ = oracle.counts(g.beg, g.end, g.adj, 0, sources=src)
            c1, o1, _, _ = oracle.counts(g.beg, g.end, g.adj, 1, sources=src)
            tot += int(c0[src].sum() - o0[src].sum() + c1[src].sum() - o1[src].sum())
        assert tot == full["fill_count"]


def test_invalid_input_rejected():
    g = random_graph(10, 0.2, 1)
    bad = g.adj.copy()
    bad[0] = 10
    with pytest.raises(ValueError):
        oracle.counts(g.beg, g.end, bad, 0)
    beg = g.beg.copy()
    beg[3] = g.end[3] + 1
    with pytest.raises(ValueError):
        oracle.counts(beg, g.end, g.adj, 0)


def test_serial_and_threaded_agree():
    g = matgen.grid3d(12, ordering="nd", drop_frac=0.1, seed=7)
    a = oracle.symbfact(g.beg, g.end, g.adj, nthreads=1)
    b = oracle.symbfact(g.beg, g.end, g.adj, nthreads=0)
    for k in ("u_idx", "l_idx", "u_row_count", "l_col_count", "sn_start"):
        assert np.array_equal(a[k], b[k])
    assert a["fill_count"] == b["fill_count"] and a["e_insp"] == b["e_insp"]


@pytest.mark.parametrize("max_sn", [0, 4])
def test_supernode_structure_claims(max_sn):
    """What the supernodal output relies on, checked on oracle patterns: in a
    supernode [f, l) every U row j is {j+1 .. l-1} plus the same columns >= l,
    and every L column's rows >= l lie inside the last column's."""
    for g in (bundled(), matgen.grid3d(12, ordering="nd", drop_frac=0.1, seed=5),
              matgen.powerlaw(800, seed=9), random_graph(200, 0.03, 4)):
        r = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=True, max_supernode_size=max_sn)
        up, ui, lp, li = r["u_ptr"], r["u_idx"], r["l_ptr"], r["l_idx"]
        xs = np.append(r["sn_start"], g.n)
        for k in range(len(xs) - 1):
            f, l = xs[k], xs[k + 1]
            right = ui[up[f]:up[f + 1]]
            right = right[right >= l]
            last = set(li[lp[l - 1]:lp[l]].tolist())
            for j in range(f, l):
                row = ui[up[j]:up[j + 1]]
                assert np.array_equal(row[:l - j - 1], np.arange(j + 1, l))
                assert np.array_equal(row[row >= l], right)
                col = li[lp[j]:lp[j + 1]]
                assert set(col[col >= l].tolist()) <= last
