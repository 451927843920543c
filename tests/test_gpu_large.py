"""GPU parity at the headline sizes.

* The 80^3 nested-dissection matrix (the benchmark's default workload) and
  the 659,033-line power-law circuit matrix against the full oracle run
  committed in tests/golden/large.json (totals and SHA-256 digests of the
  per-line arrays and supernode starts; tests/golden/make_large_golden.py).
* Bordered block-diagonal matrices of one and two million lines (two visited
  bitmaps, then even one, no longer fit in a CTA's shared memory) against the
  oracle: every line's counts and link flags, the supernodes, and the sorted
  lists of a strided sample of lines.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import gsofa_b200
import oracle
from gsofa_b200 import matgen

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "large.json")


def _sha(a, dtype):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def ctx():
    c = gsofa_b200.Context(0)
    yield c
    c.close()


def _golden(name):
    with open(GOLDEN) as f:
        return json.load(f)[name]


def _check_golden(r, gold, where):
    assert r.fill_count == gold["fill_count"], where
    assert r.nnz_lu == gold["nnz_lu"] and r.nnz_u == gold["nnz_u"] and r.nnz_l == gold["nnz_l"], where
    assert r.n_supernodes == gold["n_supernodes"], where
    got = {"u_row_count": _sha(r.u_row_count, "<i4"), "l_col_count": _sha(r.l_col_count, "<i4"),
           "line_flags": _sha(r.line_flags, "u1"), "sn_start": _sha(r.sn_start, "<i4")}
    for k, v in got.items():
        assert v == gold["sha256"][k], f"{where}: {k} digest differs"


def test_nd3d_80_headline_matrix_matches_full_oracle_run(ctx):
    g = matgen.config_nd3d(80)
    gold = _golden("grid3d_80^3_7pt_nd_drop0.1")
    m = ctx.upload(g)
    r = ctx.symbfact(m)                      # with the pattern, as the benchmark runs it
    _check_golden(r, gold, "80^3 with pattern")
    assert r.u_ptr[-1] == gold["nnz_u"] and r.l_ptr[-1] == gold["nnz_l"]
    assert np.array_equal(np.diff(r.u_ptr), r.u_row_count)
    # the work counters of a run without reuse are the oracle's |X| and E_insp
    r0 = ctx.symbfact(m, want_pattern=0, reuse=0)
    _check_golden(r0, gold, "80^3 counts, no reuse")
    assert r0.x_total == gold["x_total"] and r0.e_insp == gold["e_insp"]


def test_circuit_matrix_matches_full_oracle_run(ctx):
    g = matgen.config_circuit()
    gold = _golden("powerlaw_659033_rcm")
    r = ctx.symbfact(ctx.upload(g), want_pattern=0)
    _check_golden(r, gold, "circuit counts")


def bordered(n_blocks):
    """Bordered block-diagonal: traversals from block lines stay inside their
    32-line block, so the oracle stays cheap at millions of lines."""
    return matgen.bordered_blocks(n_blocks, 32, 8, seed=n_blocks)


def _check_against_oracle(r, g, sample_every, where):
    c0, o0, x0, _ = oracle.counts(g.beg, g.end, g.adj, 0)
    c1, o1, x1, _ = oracle.counts(g.beg, g.end, g.adj, 1)
    assert np.array_equal(r.u_row_count, c0), f"{where}: U row counts"
    assert np.array_equal(r.l_col_count, c1), f"{where}: L column counts"
    assert np.array_equal(r.line_flags, (x0 | (x1 << 1)).astype(np.uint8)), f"{where}: link flags"
    assert np.array_equal(r.sn_start, oracle.supernodes(c0, x0, x1, 0)), f"{where}: supernodes"
    fills = int(c0.sum(dtype=np.int64) + c1.sum(dtype=np.int64) - o0.sum(dtype=np.int64) - o1.sum(dtype=np.int64))
    assert r.fill_count == fills, where
    if r.u_ptr is not None:
        src = np.arange(g.n - 1, -1, -sample_every, dtype=np.int32)
        for pass_, cnt, ptr, idx in ((0, c0, r.u_ptr, r.u_idx), (1, c1, r.l_ptr, r.l_idx)):
            rp, ri = oracle.lists(g.beg, g.end, g.adj, pass_, src, cnt)
            for i, s in enumerate(src.tolist()):
                assert np.array_equal(idx[ptr[s]:ptr[s + 1]], ri[rp[i]:rp[i + 1]]), f"{where}: list {pass_}/{s}"


def test_more_than_a_million_lines(ctx):
    """n = 1,024,000: two bitmaps no longer fit in shared memory.  By default
    the paired traversals keep theirs in global memory; forced into shared
    memory, one traversal per CTA reuses along adjacency chains."""
    g = bordered(32_768)                     # n = 1,048,584
    assert g.n > 1_000_000
    m = ctx.upload(g)
    _check_against_oracle(ctx.symbfact(m), g, 997, "1M bordered, global state")
    r = ctx.symbfact(m, flags=gsofa_b200.FLAG_SHARED_STATE)
    assert r.reused_sources > 0
    _check_against_oracle(r, g, 997, "1M bordered, shared state")


def test_more_lines_than_shared_memory_holds(ctx):
    """n = 2,097,152: not even one bitmap fits in a CTA's shared memory; the
    global-state kernel factorizes it, the pattern straight to a host pool."""
    g = bordered(65_536)                     # n = 2,097,160
    assert g.n > 2_000_000
    m = ctx.upload(g)
    with pytest.raises(gsofa_b200.GsofaError) as e:
        ctx.symbfact(m, want_pattern=0, flags=gsofa_b200.FLAG_SHARED_STATE)
    assert e.value.status == 7
    counts = ctx.symbfact(m, want_pattern=0)
    _check_against_oracle(counts, g, 1, "2M bordered, counts")
    import torch
    pool = torch.empty(counts.nnz_u + counts.nnz_l, dtype=torch.int32).pin_memory().numpy()
    r = ctx.symbfact_ranges(m, pool)
    assert r.pool_used == counts.nnz_u + counts.nnz_l
    src = np.arange(g.n - 1, -1, -1009, dtype=np.int32)
    c0, _, _, _ = oracle.counts(g.beg, g.end, g.adj, 0, sources=src)
    c1, _, _, _ = oracle.counts(g.beg, g.end, g.adj, 1, sources=src)
    for pass_, cnt, row in ((0, c0, r.u_row), (1, c1, r.l_col)):
        rp, ri = oracle.lists(g.beg, g.end, g.adj, pass_, src, cnt)
        for i, s in enumerate(src.tolist()):
            assert np.array_equal(row(s), ri[rp[i]:rp[i + 1]]), f"pass {pass_} line {s}"
