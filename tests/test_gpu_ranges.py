"""GPU parity of the pattern's ranges form (gsofa_symbfact_ranges): the
lists written straight into a caller pool -- device memory, or page-locked
host memory that the lists reach while the traversals run -- and addressed by
per-line begins, the reference's own colbeg/colend layout.  Compared with the
CPU oracle list by list."""
import numpy as np
import pytest

import gsofa_b200
import oracle
from gsofa_b200 import matgen
from tests.common import bundled, random_graph, supernodal_reference

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    c = gsofa_b200.Context(0)
    yield c
    c.close()


def _pinned(count):
    return torch.empty(max(int(count), 1), dtype=torch.int32).pin_memory().numpy()


def _check(r, g, ref, pool, where):
    """Every list of r (ranges form, lists in `pool`) against the oracle."""
    assert r.fill_count == ref["fill_count"] and r.nnz_lu == ref["nnz_lu"], where
    assert np.array_equal(r.u_row_count, ref["u_row_count"]), where
    assert np.array_equal(r.l_col_count, ref["l_col_count"]), where
    assert np.array_equal(r.l_row_count, ref["l_row_count"]), where
    assert np.array_equal(r.sn_start, ref["sn_start"]), where
    up, ui, lp, li = ref["u_ptr"], ref["u_idx"], ref["l_ptr"], ref["l_idx"]
    for s in range(g.n):
        b = int(r.u_beg[s])
        assert np.array_equal(pool[b:b + r.u_row_count[s]], ui[up[s]:up[s + 1]]), f"{where}: U row {s}"
        b = int(r.l_beg[s])
        assert np.array_equal(pool[b:b + r.l_col_count[s]], li[lp[s]:lp[s + 1]]), f"{where}: L col {s}"


MATS = [bundled, lambda: matgen.grid3d(16, ordering="nd", drop_frac=0.1, seed=3),
        lambda: matgen.powerlaw(1500, seed=9), lambda: random_graph(400, 0.02, 7)]


@pytest.mark.parametrize("where", ["host", "host-direct", "device"])
def test_ranges_form_matches_oracle(ctx, where):
    for make in MATS:
        g = make()
        ref = oracle.symbfact(g.beg, g.end, g.adj, max_supernode_size=8)
        need = int(ref["u_idx"].size + ref["l_idx"].size)
        m = ctx.upload(g)
        if where.startswith("host"):
            pool = _pinned(need)
            flags = gsofa_b200.FLAG_DIRECT_HOST if where == "host-direct" else 0
            r = ctx.symbfact_ranges(m, pool, max_supernode_size=8, flags=flags)
            host_pool = pool
        else:
            pool = torch.full((max(need, 1),), -1, dtype=torch.int32, device="cuda")
            # with the supernodal structure built on the device from the pool
            r, sup = ctx.symbfact_ranges(m, pool, max_supernode_size=8, supernodal=True)
            host_pool = pool.cpu().numpy()
            for k, v in supernodal_reference(ref).items():
                assert np.array_equal(getattr(sup, k), v), f"{g.name}: supernodal {k}"
        # exact ranges per chain: the lists fill the pool with no gaps
        assert r.pool_used == need
        _check(r, g, ref, host_pool, f"{g.name} {where}")


def test_batch_shares_one_pool(ctx):
    gs = [matgen.grid2d(17), matgen.grid3d(9, seed=1), matgen.powerlaw(700, seed=2), bundled()]
    refs = [oracle.symbfact(g.beg, g.end, g.adj) for g in gs]
    need = sum(int(r["u_idx"].size + r["l_idx"].size) for r in refs)
    pool = _pinned(need + 100)
    rs = ctx.symbfact_ranges([ctx.upload(g) for g in gs], pool)
    for g, r, ref in zip(gs, rs, refs):
        assert r.pool_used == need
        _check(r, g, ref, pool, f"batch {g.name}")


def test_small_pool_reports_the_need_and_caller_buffers(ctx):
    g = matgen.grid3d(12, ordering="nd", drop_frac=0.1, seed=5)
    ref = oracle.symbfact(g.beg, g.end, g.adj)
    need = int(ref["u_idx"].size + ref["l_idx"].size)
    m = ctx.upload(g)
    with pytest.raises(gsofa_b200.GsofaError) as e:
        ctx.symbfact_ranges(m, _pinned(need // 3))
    assert e.value.status == 3 and e.value.needed == need
    # the exact size fits; the per-line arrays go to caller buffers
    pool = _pinned(need)
    n = g.n
    bufs = {k: np.zeros(n, np.int32) for k in ("u_row_count", "l_col_count", "l_row_count", "sn_start")}
    bufs.update(u_beg=np.zeros(n, np.int64), l_beg=np.zeros(n, np.int64))
    r = ctx.symbfact_ranges(m, pool, out=bufs)
    assert np.shares_memory(r.u_beg, bufs["u_beg"])
    _check(r, g, ref, pool, "caller buffers")
    # pageable host memory is refused (it cannot be written by the GPU)
    with pytest.raises(gsofa_b200.GsofaError) as e:
        ctx.symbfact_ranges(m, np.zeros(need, np.int32))
    assert e.value.status == 1


def test_pattern_larger_than_the_device_budget_streams_to_host():
    """A power-law matrix whose ~0.9 GB pattern is several times the
    context's 160 MB device budget: the CSR form, which holds the pattern on
    the device twice, runs out of memory; the ranges form streams the lists
    into host memory during the traversal and is exact."""
    g = matgen.powerlaw(28_000, seed=28)
    c0, o0, x0, _ = oracle.counts(g.beg, g.end, g.adj, 0)
    c1, o1, x1, _ = oracle.counts(g.beg, g.end, g.adj, 1)
    need = int(c0.sum(dtype=np.int64) + c1.sum(dtype=np.int64))
    budget = 160 << 20
    assert 4 * need > 5 * budget
    with gsofa_b200.Context(0, mem_budget_bytes=budget) as small:
        m = small.upload(g)
        with pytest.raises(gsofa_b200.GsofaError) as e:
            small.symbfact(m)
        assert e.value.status == 2
        pool = _pinned(need)
        r = small.symbfact_ranges(m, pool)
    assert r.pool_used == need
    assert np.array_equal(r.u_row_count, c0) and np.array_equal(r.l_col_count, c1)
    assert np.array_equal(r.line_flags, (x0 | (x1 << 1)).astype(np.uint8))
    assert np.array_equal(r.sn_start, oracle.supernodes(c0, x0, x1, 0))
    src = np.arange(g.n - 1, -1, -37, dtype=np.int32)
    for pass_, cnt, row in ((0, c0, r.u_row), (1, c1, r.l_col)):
        rp, ri = oracle.lists(g.beg, g.end, g.adj, pass_, src, cnt)
        for i, s in enumerate(src.tolist()):
            assert np.array_equal(row(s), ri[rp[i]:rp[i + 1]]), f"pass {pass_} line {s}"
