"""The ordering step before the path (reverse Cuthill-McKee): the oracle's
restatement against an independent statement of the same rules, its quality
against scipy's reverse_cuthill_mckee, and the host permutation of a pattern.
The GPU ordering is compared with the oracle in tests/test_gpu_order.py."""
import numpy as np
import pytest

import oracle
from gsofa_b200 import matgen
from tests.common import bundled, random_graph


def _sym(g):
    S = [set() for _ in range(g.n)]
    for v in range(g.n):
        for u in g.adj[g.beg[v]:g.end[v]]:
            u = int(u)
            if u != v:
                S[v].add(u)
                S[u].add(v)
    return S


def _rcm_reference_statement(g):
    """Sequential Cuthill-McKee, George-Liu start, (degree, id) ties, reversed."""
    n = g.n
    S = _sym(g)
    deg = [len(x) for x in S]
    key = lambda v: (deg[v], v)  # noqa: E731
    ordered = [False] * n
    cm = []

    def bfs(r):
        lev = {r: 0}
        q = [r]
        i = 0
        while i < len(q):
            v = q[i]
            i += 1
            for u in S[v]:
                if not ordered[u] and u not in lev:
                    lev[u] = lev[v] + 1
                    q.append(u)
        ecc = max(lev.values())
        return ecc, min((v for v in q if lev[v] == ecc), key=key)

    for start in sorted(range(n), key=key):
        if ordered[start]:
            continue
        r = start
        ecc, c = bfs(r)
        while True:
            ecc_c, c2 = bfs(c)
            if ecc_c <= ecc:
                break
            r, ecc, c = c, ecc_c, c2
        q = [r]
        ordered[r] = True
        i = 0
        while i < len(q):
            v = q[i]
            i += 1
            for u in sorted((u for u in S[v] if not ordered[u]), key=key):
                ordered[u] = True
                q.append(u)
        cm += q
    return np.array(cm[::-1], dtype=np.int32)


def _bandwidth(g, perm):
    inv = np.empty(g.n, np.int64)
    inv[perm] = np.arange(g.n)
    rows = np.repeat(np.arange(g.n), g.end - g.beg)
    cols = np.concatenate([g.adj[b:e] for b, e in zip(g.beg, g.end)]) if g.nnz else np.zeros(0, np.int64)
    return int(np.abs(inv[rows] - inv[cols]).max()) if rows.size else 0


CASES = [
    lambda: matgen.grid2d(12),
    lambda: matgen.grid3d(6, ordering="nd"),
    lambda: matgen.powerlaw(800, seed=3, ordering="random"),
    lambda: random_graph(300, 0.01, 5),
    lambda: random_graph(200, 0.002, 7),            # many components
    lambda: matgen.bordered_blocks(12, block=16, border=4, seed=2),
    lambda: matgen.Graph(5, np.arange(5, dtype=np.int32), np.arange(1, 6, dtype=np.int32),
                         np.arange(5, dtype=np.int32), "diagonal_only"),
    lambda: matgen.Graph(1, np.zeros(1, np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32), "one_line"),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_oracle_rcm_matches_an_independent_statement(case):
    g = CASES[case]()
    perm = oracle.rcm(g.beg, g.end, g.adj)
    assert sorted(perm.tolist()) == list(range(g.n))
    assert np.array_equal(perm, _rcm_reference_statement(g))


def test_rcm_quality_against_scipy():
    """Same family of orderings as scipy's: bandwidths within a small factor
    of scipy's on shuffled patterns, far below the shuffled input's."""
    import gsofa_b200
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    shuffled_grid = gsofa_b200.permute_lines(matgen.grid2d(40), np.random.default_rng(1).permutation(1600))
    for g in (matgen.powerlaw(3000, seed=4, ordering="random"), bundled(), shuffled_grid):
        rows = np.repeat(np.arange(g.n), g.end - g.beg)
        cols = np.concatenate([g.adj[b:e] for b, e in zip(g.beg, g.end)])
        A = csr_matrix((np.ones(rows.size, np.int8), (rows, cols)), shape=(g.n, g.n))
        S = (A + A.T).tocsr()
        ours = _bandwidth(g, oracle.rcm(g.beg, g.end, g.adj))
        theirs = _bandwidth(g, reverse_cuthill_mckee(S, symmetric_mode=True).astype(np.int64))
        assert ours <= 2 * theirs + 2, (g.name, ours, theirs)
        assert ours < _bandwidth(g, np.arange(g.n)) or _bandwidth(g, np.arange(g.n)) <= 2


def test_permute_lines_is_the_symmetric_permutation():
    import gsofa_b200
    g = random_graph(150, 0.03, 9)
    perm = np.random.default_rng(3).permutation(g.n).astype(np.int32)
    h = gsofa_b200.permute_lines(g, perm)
    inv = np.empty(g.n, np.int64)
    inv[perm] = np.arange(g.n)
    for k in range(g.n):
        v = perm[k]
        assert np.array_equal(h.adj[h.beg[k]:h.end[k]], np.sort(inv[g.adj[g.beg[v]:g.end[v]]]))
    with pytest.raises(gsofa_b200.GsofaError):
        gsofa_b200.permute_lines(g, np.zeros(g.n, np.int32))   # not a permutation


def test_permute_lines_edge_cases():
    import gsofa_b200
    # identity: every line sorted, ids unchanged
    g = random_graph(60, 0.05, 2)
    h = gsofa_b200.permute_lines(g, np.arange(g.n, dtype=np.int32))
    for v in range(g.n):
        assert np.array_equal(h.adj[h.beg[v]:h.end[v]], np.sort(g.adj[g.beg[v]:g.end[v]]))
    # one line, and no lines
    one = matgen.Graph(1, np.zeros(1, np.int32), np.ones(1, np.int32), np.zeros(1, np.int32), "one")
    h1 = gsofa_b200.permute_lines(one, np.zeros(1, np.int32))
    assert h1.n == 1 and h1.adj.tolist() == [0]
    empty = matgen.Graph(0, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32), "empty")
    assert gsofa_b200.permute_lines(empty, np.zeros(0, np.int32)).n == 0
    # wrong length, out-of-range and repeated entries are errors
    with pytest.raises(gsofa_b200.GsofaError):
        gsofa_b200.permute_lines(g, np.arange(g.n - 1, dtype=np.int32))
    bad = np.arange(g.n, dtype=np.int32)
    bad[3] = g.n
    with pytest.raises(gsofa_b200.GsofaError):
        gsofa_b200.permute_lines(g, bad)



def test_rcm_reduces_fill_of_a_shuffled_pattern():
    """The point of the step before the path, on the oracle: a shuffled 2-D
    grid factorizes with far less fill once ordered by reverse Cuthill-McKee;
    a shuffled power-law pattern, whose random long-range columns no band
    ordering can gather, with somewhat less."""
    import gsofa_b200
    rng = np.random.default_rng(5)
    grid = gsofa_b200.permute_lines(matgen.grid2d(30), rng.permutation(900).astype(np.int32))
    for g, factor in ((grid, 0.5), (matgen.powerlaw(1500, seed=6, ordering="random"), 0.95)):
        h = gsofa_b200.permute_lines(g, oracle.rcm(g.beg, g.end, g.adj))
        before = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False)["nnz_lu"]
        after = oracle.symbfact(h.beg, h.end, h.adj, want_pattern=False)["nnz_lu"]
        assert after < factor * before, (g.name, before, after)
