"""GPU parity: the CUDA library (through its C ABI) against the CPU oracle,
bit for bit -- pattern, per-line counts, supernodes, fill totals."""
import numpy as np
import pytest

import gsofa_b200
import oracle
from gsofa_b200 import matgen
from tests.common import assert_same, bundled, expected, random_graph, supernodal_reference

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = gsofa_b200.Context(0)
    yield c
    c.close()


def _oracle(g, max_sn=0, pattern=True):
    return oracle.symbfact(g.beg, g.end, g.adj, want_pattern=pattern, max_supernode_size=max_sn)


def test_bundled_matrix(ctx):
    g = bundled()
    m = ctx.upload(g)
    exp = expected()["bundled_11948"]
    for max_sn in (0, 4):
        ref = _oracle(g, max_sn)
        r = ctx.symbfact(m, max_supernode_size=max_sn)
        assert r.fill_count == exp["fill_count"] and r.nnz_lu == exp["nnz_lu"]
        assert_same(r, ref, where=f"bundled max_sn={max_sn}")


def test_grid2d_natural_golden(ctx):
    g = matgen.config_plain2d()
    r = ctx.symbfact(ctx.upload(g))
    exp = expected()["grid2d_64x64_natural"]
    assert r.fill_count == exp["fill_count"] and r.nnz_lu == exp["nnz_lu"]
    assert_same(r, _oracle(g), where="grid2d 64")


@pytest.mark.parametrize("side", [6, 13, 20])
def test_grid3d_nd(ctx, side):
    g = matgen.grid3d(side, ordering="nd", drop_frac=0.1, seed=side)
    assert_same(ctx.symbfact(ctx.upload(g)), _oracle(g), where=f"grid3d {side}")


@pytest.mark.parametrize("n", [500, 3000])
def test_powerlaw(ctx, n):
    g = matgen.powerlaw(n, seed=n)
    ref = _oracle(g, 12)
    m = ctx.upload(g)
    for reuse in (-1, 2, 0):
        r = ctx.symbfact(m, reuse=reuse, max_supernode_size=12)
        assert_same(r, ref, where=f"powerlaw {n} reuse {reuse}")


@pytest.mark.parametrize("seed", range(10))
def test_random_free_form_layout(ctx, seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(1, 400))
    g = random_graph(n, float(rng.choice([0.003, 0.01, 0.03, 0.1])), seed)
    assert_same(ctx.symbfact(ctx.upload(g)), _oracle(g), where=f"random {seed}")


def test_empty_and_tiny(ctx):
    for n in (1, 2, 33):
        g = matgen.Graph(n, np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(0, np.int32))
        r = ctx.symbfact(ctx.upload(g))
        assert r.fill_count == 0 and r.nnz_lu == n
        assert_same(r, _oracle(g), where=f"empty {n}")


@pytest.mark.parametrize("block,lanes,reuse,chunk,per_sm", [
    (128, 4, 0, 1, 0), (256, 8, 1, 7, 1), (512, 16, 1, 32, 0), (1024, 32, 0, 3, 0),
    (256, 32, 1, 1, 2), (512, 8, 1, 200, 0), (128, 1, 0, 1, 0), (1024, 1, 1, 16, 1),
    (512, 1, 2, 32, 0), (256, 1, 2, 5, 0), (1024, 1, 2, 64, 1), (512, 1, -1, 3, 2),
    (768, 1, -1, 0, 0), (768, 8, 1, 40, 0), (768, 1, 0, 1, 0)])
def test_parameters_do_not_change_results(ctx, block, lanes, reuse, chunk, per_sm):
    g = matgen.grid3d(14, ordering="nd", drop_frac=0.1, seed=5)
    ref = _oracle(g, 8)
    r = ctx.symbfact(ctx.upload(g), block_size=block, threads_per_source=lanes, reuse=reuse,
                     src_chunk=chunk, ctas_per_sm=per_sm, max_supernode_size=8)
    assert_same(r, ref, where=f"params {block},{lanes},{reuse},{chunk},{per_sm}")


@pytest.mark.parametrize("block,lanes,reuse,chunk,per_sm", [
    (256, 1, -1, 0, 0), (128, 1, -1, 5, 0), (512, 1, -1, 64, 1), (256, 8, 1, 7, 2),
    (128, 1, 0, 1, 0), (256, 1, 2, 32, 0), (512, 32, 0, 3, 0), (128, 4, 2, 16, 3)])
def test_global_state_kernel(ctx, block, lanes, reuse, chunk, per_sm):
    """Visited bitmaps in global memory: the same results as the oracle, for
    the paired (exact reuse), adjacency-reuse and no-reuse traversals."""
    ref = None
    for g in (matgen.grid3d(14, ordering="nd", drop_frac=0.1, seed=5), matgen.powerlaw(1200, seed=12),
              random_graph(300, 0.03, 4)):
        ref = _oracle(g, 8)
        r = ctx.symbfact(ctx.upload(g), block_size=block, threads_per_source=lanes, reuse=reuse,
                         src_chunk=chunk, ctas_per_sm=per_sm, max_supernode_size=8,
                         flags=gsofa_b200.FLAG_GLOBAL_STATE)
        assert_same(r, ref, where=f"global state {g.name} {block},{lanes},{reuse},{chunk},{per_sm}")


def test_wide_register_kernel(ctx):
    for g in (matgen.grid3d(20, ordering="nd", drop_frac=0.1, seed=2), matgen.powerlaw(12000, seed=5)):
        for pattern in (0, 1):
            r = ctx.symbfact(ctx.upload(g), want_pattern=pattern, max_supernode_size=8,
                             flags=gsofa_b200.FLAG_WIDE_REGS)
            assert_same(r, _oracle(g, 8, pattern=bool(pattern)), pattern=bool(pattern),
                        where=f"wide registers {g.name} pattern={pattern}")
    with pytest.raises(gsofa_b200.GsofaError):
        ctx.symbfact(ctx.upload(bundled()), reuse=0, flags=gsofa_b200.FLAG_WIDE_REGS)


def test_state_flags_conflict_is_an_error(ctx):
    with pytest.raises(gsofa_b200.GsofaError) as e:
        ctx.symbfact(ctx.upload(bundled()),
                     flags=gsofa_b200.FLAG_GLOBAL_STATE | gsofa_b200.FLAG_SHARED_STATE)
    assert e.value.status == 1


def test_chain_longer_than_stamp_range(ctx):
    """A path in natural order lets every source reuse its predecessor's
    traversal, so one piece of 65,600 sources is one chain of reuse.  List
    output keys each vertex by a 16-bit chain index, so the chain has to end
    after 65,535 sources; the lists must stay exact across that break."""
    n = 65_600
    g = matgen.grid2d(n, 1)
    ref = _oracle(g)
    r = ctx.symbfact(ctx.upload(g), src_chunk=n)
    assert r.reused_sources >= 2 * (n - 2)   # one chain per pass, but for the break
    assert_same(r, ref, where="path, one 65,600-source piece")


def test_reused_device_slab_gives_exact_results(ctx):
    """A freed matrix leaves its device slab in the context; the next upload
    of similar size takes it over with the old contents still in it."""
    big = matgen.grid3d(16, ordering="nd", drop_frac=0.1, seed=3)
    small = matgen.grid3d(14, ordering="nd", drop_frac=0.1, seed=4)
    m = ctx.upload(big)
    assert_same(ctx.symbfact(m), _oracle(big), where="first slab")
    m.free()
    m2 = ctx.upload(small)      # fits the cached slab (within a factor of two)
    assert_same(ctx.symbfact(m2), _oracle(small), where="reused slab")
    m2.free()
    m3 = ctx.upload(big)
    assert_same(ctx.symbfact(m3), _oracle(big), where="slab reused again")
    m3.free()


@pytest.mark.parametrize("max_sn", [0, 8])
def test_supernodal_structure(ctx, max_sn):
    for g in (bundled(), matgen.grid3d(16, ordering="nd", drop_frac=0.1, seed=3),
              matgen.powerlaw(1500, seed=9), random_graph(400, 0.02, 7)):
        ref = _oracle(g, max_sn)
        want = supernodal_reference(ref)
        m = ctx.upload(g)
        r, s = ctx.symbfact_supernodal(m, max_supernode_size=max_sn)
        assert r.nnz_lu == ref["nnz_lu"] and s.n == g.n and s.nsuper == len(ref["sn_start"])
        for k, v in want.items():
            assert np.array_equal(getattr(s, k), v), f"{g.name} max_sn={max_sn}: {k}"
        # into caller buffers larger than needed: the results are views of them
        out = {k: np.full(v.size + 5, -7, v.dtype) for k, v in want.items()}
        _, s2 = ctx.symbfact_supernodal(m, max_supernode_size=max_sn, out=out)
        for k, v in want.items():
            assert np.array_equal(getattr(s2, k), v) and np.shares_memory(getattr(s2, k), out[k])
    small = {"lsub": np.zeros(1, np.int32)}
    with pytest.raises(gsofa_b200.GsofaError):
        ctx.symbfact_supernodal(ctx.upload(bundled()), out=small)


def test_counts_only_and_pool_retry(ctx):
    g = matgen.powerlaw(2000, seed=9)
    ref = _oracle(g)
    m = ctx.upload(g)
    r = ctx.symbfact(m, want_pattern=0)
    assert_same(r, ref, pattern=False, where="counts only")
    assert r.u_idx is None and r.l_row_count is None
    # a pool far too small: the library reruns with the exact size
    r = ctx.symbfact(m, pool_capacity=16)
    assert_same(r, ref, where="pool retry")


def test_partitions_sum_to_total(ctx):
    g = bundled()
    m = ctx.upload(g)
    for parts in (6, 264):
        tot = sum(ctx.symbfact(m, part_count=parts, part_index=i, want_pattern=0).fill_count
                  for i in range(parts))
        assert tot == expected()["bundled_11948"]["fill_count"]


def test_invalid_inputs_are_statuses(ctx):
    g = random_graph(50, 0.05, 3)
    bad = g.adj.copy()
    bad[len(bad) // 2] = 50
    with pytest.raises(gsofa_b200.GsofaError) as e:
        ctx.upload(g.beg, g.end, bad)
    assert e.value.status == 1
    beg = g.beg.copy()
    beg[7] = len(g.adj) + 5
    with pytest.raises(gsofa_b200.GsofaError):
        ctx.upload(beg, g.end, g.adj)
    # the context stays usable
    assert_same(ctx.symbfact(ctx.upload(g)), _oracle(g), where="after errors")


def test_reference_argv_entry(tmp_path):
    g = bundled()
    (tmp_path / "b.dat").write_text(" ".join(map(str, g.beg.tolist())))
    (tmp_path / "e.dat").write_text(" ".join(map(str, g.end.tolist())))
    (tmp_path / "c.dat").write_text(f"{g.nnz} {g.n}\n" + " ".join(map(str, g.adj.tolist())))
    files = [str(tmp_path / f) for f in ("b.dat", "e.dat", "c.dat")]
    want = expected()["bundled_11948"]["fill_count"]
    for argv in (["gsofa", *files, "1"], ["gsofa", *files, "6", "1"],
                 ["gsofa", *files, "264", "5", "128", "1"],
                 # a 10 MB pool: fewer concurrent traversals, the same total
                 ["gsofa", *files, "1", "0.01"], ["gsofa", *files, "6", "0.01", "0", "1"]):
        fills, ms = gsofa_b200.symbfact_min_id(argv)
        assert fills == want and ms > 0
    # a pool too small for one traversal's state is an out-of-memory status
    with pytest.raises(gsofa_b200.GsofaError) as e:
        gsofa_b200.symbfact_min_id(["gsofa", *files, "1", "0.00001"])
    assert e.value.status == 2
    # the same matrix in the binary form
    bins = [str(tmp_path / f) for f in ("b.bin", "e.bin", "c.bin")]
    gsofa_b200.write_binary(g, *bins)
    fills, ms = gsofa_b200.symbfact_min_id(["gsofa", *bins, "1"])
    assert fills == want


def test_batch_matches_one_by_one(ctx):
    gs = [matgen.grid2d(17), matgen.grid3d(9, seed=1), matgen.powerlaw(700, seed=2),
          random_graph(90, 0.04, 5), bundled(), random_graph(1, 0.0, 1)]
    ms = [ctx.upload(g) for g in gs]
    rs = ctx.symbfact_batch(ms, max_supernode_size=16)
    for g, r in zip(gs, rs):
        assert_same(r, _oracle(g, 16), where=f"batch {g.name}")


def test_exhaustive_n4_in_one_batch(ctx):
    pairs = [(i, j) for i in range(4) for j in range(4) if i != j]
    gs, ms = [], []
    for mask in range(0, 1 << len(pairs), 3):   # every third pattern: 1,366 matrices
        rows = [[] for _ in range(4)]
        for b, (i, j) in enumerate(pairs):
            if mask >> b & 1:
                rows[i].append(j)
        ptr = np.zeros(5, np.int64)
        ptr[1:] = np.cumsum([len(r) for r in rows])
        g = matgen.Graph.from_csr(ptr, np.array([c for r in rows for c in r], np.int32))
        gs.append(g)
        ms.append(ctx.upload(g))
    rs = ctx.symbfact_batch(ms)
    for g, r in zip(gs, rs):
        assert_same(r, _oracle(g), where="n4")
    for m in ms:
        m.free()


def test_fetch_into_caller_buffers(ctx):
    g = matgen.grid3d(11, ordering="nd", drop_frac=0.1, seed=3)
    ref = _oracle(g, 6)
    m = ctx.upload(g)
    n = g.n
    big = 4 * int(ref["u_idx"].shape[0] + 10)
    bufs = {"u_row_count": np.zeros(n, np.int32), "l_col_count": np.zeros(n, np.int32),
            "l_row_count": np.zeros(n, np.int32), "sn_start": np.zeros(n, np.int32),
            "u_ptr": np.zeros(n + 1, np.int64), "l_ptr": np.zeros(n + 1, np.int64),
            "u_idx": np.zeros(big, np.int32), "l_idx": np.zeros(big, np.int32)}
    r = ctx.symbfact_into(m, gsofa_b200.Params.default(max_supernode_size=6), bufs)
    assert_same(r, ref, where="fetch")
    # a stale result cannot be fetched after the next factorization
    p = gsofa_b200.Params.default(flags=gsofa_b200.FLAG_NO_DOWNLOAD)
    r1 = gsofa_b200._CResult()
    L = gsofa_b200.lib()
    assert L.gsofa_symbfact(ctx._h, m.handle, p, r1) == 0
    r2 = gsofa_b200._CResult()
    assert L.gsofa_symbfact(ctx._h, m.handle, p, r2) == 0
    z = np.zeros(n, np.int32)
    i32 = gsofa_b200._i32p
    assert L.gsofa_result_fetch(ctx._h, r1, z.ctypes.data_as(i32), None, None, None, None, None,
                                None, None) == 1
    assert L.gsofa_result_fetch(ctx._h, r2, z.ctypes.data_as(i32), None, None, None, None, None,
                                None, None) == 0
    assert np.array_equal(z, ref["u_row_count"])
    L.gsofa_result_free(r1)
    L.gsofa_result_free(r2)


def test_graph_replay(ctx):
    gs = [matgen.grid3d(9, seed=1), matgen.powerlaw(600, seed=2), bundled()]
    ms = [ctx.upload(g) for g in gs]
    p = gsofa_b200.Params.default(flags=gsofa_b200.FLAG_GRAPH, max_supernode_size=8)
    refs = [_oracle(g, 8) for g in gs]
    for rep in range(3):
        rs = ctx.symbfact_batch(ms, p)
        for g, r, ref in zip(gs, rs, refs):
            assert_same(r, ref, where=f"graph replay {rep} {g.name}")
    # a different job replaces the captured one
    rs = ctx.symbfact_batch(ms[1:], p)
    for g, r, ref in zip(gs[1:], rs, refs[1:]):
        assert_same(r, ref, where=f"graph recapture {g.name}")


def test_autotune_choice_is_cached_and_exact(ctx, tmp_path):
    from gsofa_b200 import autotune
    gs = [matgen.grid3d(12, seed=3), matgen.powerlaw(900, seed=4), matgen.grid2d(30)]
    ms = [ctx.upload(g) for g in gs]
    cache = str(tmp_path / "tune.json")
    best, rep = autotune.autotune(ctx, ms, cache_path=cache)
    assert not rep["cached"] and len(rep["timings"]) == len(autotune.DEFAULT_CANDIDATES)
    best2, rep2 = autotune.autotune(ctx, ms, cache_path=cache)
    assert rep2["cached"] and rep2["choice"] == rep["choice"]
    for g, r in zip(gs, ctx.symbfact_batch(ms, best2)):
        assert_same(r, _oracle(g), where=f"autotuned {g.name}")


@pytest.mark.parametrize("make,parts", [(lambda: matgen.grid3d(16, ordering="nd", drop_frac=0.1, seed=3), 4),
                                        (lambda: matgen.powerlaw(1500, seed=9), 3), (bundled, 5)])
def test_line_range_partitions_keep_reuse_and_sum_to_the_whole(ctx, make, parts):
    """Contiguous ranges from the work-predicted partitioner: every range
    keeps traversal reuse, fills exactly its own lines (counts, link flags
    and, with the pattern, its lists), and the ranges add up to the full
    factorization."""
    from gsofa_b200 import distributed, partition_lines
    g = make()
    ref = _oracle(g, 8)
    m = ctx.upload(g)
    cuts, work = partition_lines(g, parts)
    assert cuts[0] == 0 and cuts[-1] == g.n and len(work) == parts
    u = np.zeros(g.n, np.int64); lc = np.zeros(g.n, np.int64); fl = np.zeros(g.n, np.int64); fills = 0
    for k in range(parts):
        lo, hi = int(cuts[k]), int(cuts[k + 1])
        r = ctx.symbfact(m, line_lo=lo, line_hi=hi, max_supernode_size=8)
        if hi - lo > 2:
            assert r.reused_sources > 0, (lo, hi)
        inside = np.zeros(g.n, bool); inside[lo:hi] = True
        assert np.all(r.u_row_count[~inside] == 0) and np.all(r.l_col_count[~inside] == 0)
        assert np.array_equal(r.u_row_count[inside], ref["u_row_count"][inside])
        for s_ in range(lo, hi):
            assert np.array_equal(r.u_idx[r.u_ptr[s_]:r.u_ptr[s_ + 1]],
                                  ref["u_idx"][ref["u_ptr"][s_]:ref["u_ptr"][s_ + 1]]), s_
            assert np.array_equal(r.l_idx[r.l_ptr[s_]:r.l_ptr[s_ + 1]],
                                  ref["l_idx"][ref["l_ptr"][s_]:ref["l_ptr"][s_ + 1]]), s_
        u += r.u_row_count; lc += r.l_col_count; fl += r.line_flags; fills += r.fill_count
    out = distributed.combine(g.n, u, lc, fl, fills, lambda x: x, max_supernode_size=8)
    assert out["fill_count"] == ref["fill_count"] and out["nnz_lu"] == ref["nnz_lu"]
    assert np.array_equal(out["sn_start"], ref["sn_start"])
    # the same through symbfact_sharded, one range per "rank" on this GPU
    tot = None
    shares = []
    for rank in range(parts):
        p = distributed.rank_params(rank, parts, cuts, max_supernode_size=8)
        r = ctx.symbfact(m, p)
        shares.append(np.concatenate([r.u_row_count, r.l_col_count, r.line_flags, [r.fill_count]]).astype(np.int64))
    tot = np.sum(shares, axis=0)
    res = distributed.symbfact_sharded(ctx, m, 0, parts, lambda x: tot, max_supernode_size=8, cuts=cuts)
    assert res["fill_count"] == ref["fill_count"] and np.array_equal(res["sn_start"], ref["sn_start"])


def test_line_range_errors(ctx):
    m = ctx.upload(bundled())
    with pytest.raises(gsofa_b200.GsofaError):   # with an interleaved partition
        ctx.symbfact(m, line_lo=0, line_hi=10, part_count=2, part_index=0)
    with pytest.raises(gsofa_b200.GsofaError):   # on a batch
        ctx.symbfact_batch([m, m], line_lo=0, line_hi=10)


def test_sharded_partitions_assemble_on_one_gpu(ctx):
    """The multi-GPU assembly with three partitions run one after another on
    this GPU: summing their per-line arrays gives the full factorization."""
    from gsofa_b200 import distributed
    g = bundled()
    m = ctx.upload(g)
    world = 3
    parts = []
    for rank in range(world):
        r = ctx.symbfact(m, want_pattern=0, part_count=world, part_index=rank)
        parts.append(np.concatenate([r.u_row_count.astype(np.int64), r.l_col_count.astype(np.int64),
                                     r.line_flags.astype(np.int64), [r.fill_count]]))
    total = np.sum(parts, axis=0)
    out = distributed.combine(g.n, parts[0][:g.n], parts[0][g.n:2 * g.n], parts[0][2 * g.n:3 * g.n],
                              int(parts[0][-1]), lambda x: total, max_supernode_size=8)
    ref = _oracle(g, 8, pattern=False)
    assert out["fill_count"] == ref["fill_count"] and out["nnz_lu"] == ref["nnz_lu"]
    assert np.array_equal(out["u_row_count"], ref["u_row_count"])
    assert np.array_equal(out["sn_start"], ref["sn_start"])
    full = ctx.symbfact(m, want_pattern=0, max_supernode_size=8)
    assert np.array_equal(full.line_flags, out["line_flags"])
