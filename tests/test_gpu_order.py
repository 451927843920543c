"""GPU reverse Cuthill-McKee (gsofa_order_rcm) against the oracle, bit for
bit, and the ordered pattern through the factorization."""
import numpy as np
import pytest

import gsofa_b200
import oracle
from gsofa_b200 import matgen
from tests.common import bundled, random_graph

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    with gsofa_b200.Context(0) as c:
        yield c


CASES = [
    lambda: matgen.grid2d(64),
    lambda: matgen.grid3d(20, ordering="nd", drop_frac=0.1, seed=2),
    lambda: matgen.powerlaw(20000, seed=5, ordering="random"),
    lambda: matgen.powerlaw(3000, seed=3, ordering="natural"),
    lambda: random_graph(3000, 0.001, 5),            # free-form layout, duplicates, diagonal
    lambda: random_graph(2000, 0.0002, 7),           # hundreds of components and isolated lines
    lambda: matgen.bordered_blocks(200, block=32, border=8, seed=4),
    lambda: bundled(),
    lambda: matgen.Graph(7, np.arange(7, dtype=np.int32), np.arange(1, 8, dtype=np.int32),
                         np.arange(7, dtype=np.int32), "diagonal_only"),
    lambda: matgen.Graph(1, np.zeros(1, np.int32), np.zeros(1, np.int32), np.zeros(0, np.int32), "one_line"),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_rcm_matches_oracle(ctx, case):
    g = CASES[case]()
    got = ctx.order_rcm(g)
    want = oracle.rcm(g.beg, g.end, g.adj)
    assert np.array_equal(got, want), f"{g.name}: first difference at {np.flatnonzero(got != want)[:5]}"


def test_rcm_ordered_pattern_factorizes_like_the_oracle(ctx):
    """The step before the path feeding the path: a shuffled power-law
    pattern, ordered on the GPU, permuted and factorized, equals the oracle
    on the same ordered pattern, with far less fill than the shuffled one."""
    g = matgen.powerlaw(6000, seed=8, ordering="random")
    h = gsofa_b200.permute_lines(g, ctx.order_rcm(g))
    with ctx.upload(h) as m:
        r = ctx.symbfact(m, want_pattern=0)
    ref = oracle.symbfact(h.beg, h.end, h.adj, want_pattern=False)
    assert r.fill_count == ref["fill_count"] and np.array_equal(r.u_row_count, ref["u_row_count"])
    with ctx.upload(g) as m:
        shuffled = ctx.symbfact(m, want_pattern=0)
    assert r.nnz_lu < shuffled.nnz_lu


def test_rcm_rejects_bad_input(ctx):
    g = matgen.grid2d(8)
    bad = matgen.Graph(g.n, g.beg, g.end, np.where(g.adj == 3, 999, g.adj).astype(np.int32))
    with pytest.raises(gsofa_b200.GsofaError):
        ctx.order_rcm(bad)
    assert np.array_equal(ctx.order_rcm(g), oracle.rcm(g.beg, g.end, g.adj))   # context still usable
