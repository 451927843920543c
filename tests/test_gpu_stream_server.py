"""The persistent serving kernel: requests published while others run give
the same results as standalone factorizations."""
import numpy as np
import pytest

import gsofa_b200
from gsofa_b200 import matgen, serve
from tests.common import bundled, random_graph

pytestmark = pytest.mark.gpu


def _same(a, b, where):
    assert (a.fill_count, a.nnz_lu, a.n_supernodes) == (b.fill_count, b.nnz_lu, b.n_supernodes), where
    assert np.array_equal(a.u_row_count, b.u_row_count), where
    assert np.array_equal(a.l_col_count, b.l_col_count), where
    assert np.array_equal(a.line_flags, b.line_flags), where
    assert np.array_equal(a.sn_start, b.sn_start), where


@pytest.mark.parametrize("flags", [0, gsofa_b200.FLAG_SHARED_STATE])
def test_stream_server_matches_standalone(flags):
    """Both kernel forms: bitmaps in global memory (default, six traversals
    per SM) and in shared memory (two per SM)."""
    reqs = serve.make_stream(40, 200, 6000, rate_hz=2000.0, seed=21, build=matgen.make)
    reqs.append(serve.Request(len(reqs), reqs[-1].arrival_s, bundled()))
    reqs.append(serve.Request(len(reqs), reqs[-1].arrival_s, random_graph(300, 0.02, 4)))
    with gsofa_b200.Context(0) as ctx, gsofa_b200.StreamServer(0, mem_budget_bytes=8 << 30,
                                                              max_supernode_size=16, flags=flags) as srv:
        out = serve.ContinuousServer(srv).run(reqs)
        rep = out["report"]
        assert rep["requests"] == len(reqs) and rep["p50_ms"] <= rep["p99_ms"]
        p = gsofa_b200.Params.default(want_pattern=0, max_supernode_size=16)
        for c, r in zip(out["completions"], reqs):
            _same(c.result, ctx.symbfact(ctx.upload(r.graph), p), f"request {r.rid} ({r.graph.name})")


def test_stream_server_admission_and_reuse_of_memory():
    """A budget that holds only a few requests at a time: the rest wait, the
    server recycles device memory of finished ones while its kernel runs."""
    gs = [matgen.grid3d(14, seed=s) for s in range(6)] + [matgen.powerlaw(2500, seed=s) for s in range(6)]
    with gsofa_b200.Context(0) as ctx, gsofa_b200.StreamServer(0, mem_budget_bytes=1 << 30, max_n=20000) as srv:
        ids = {}
        pending = list(enumerate(gs))
        results = {}
        busy_seen = False
        while pending or ids:
            while pending:
                i, g = pending[0]
                rid = srv.submit(g)
                if rid is None:
                    busy_seen = True
                    break
                ids[rid] = i
                pending.pop(0)
            for rid in srv.poll():
                results[ids.pop(rid)] = srv.result(rid)
        p = gsofa_b200.Params.default(want_pattern=0)
        for i, g in enumerate(gs):
            _same(results[i], ctx.symbfact(ctx.upload(g), p), f"matrix {i}")
        srv.drain()
        # after draining, the device is free for the cooperative path
        _same(ctx.symbfact(ctx.upload(gs[0]), p), results[0], "after drain")
        assert busy_seen or len(gs) * srv.request_bytes(gs[0].n, gs[0].nnz) < (1 << 30)


def test_stream_server_rejects_oversize_and_bad_input():
    with gsofa_b200.StreamServer(0, mem_budget_bytes=1 << 30, max_n=1000) as srv:
        assert srv.max_n == 1000
        with pytest.raises(gsofa_b200.GsofaError) as e:
            srv.submit(matgen.grid2d(40))
        assert e.value.status == 7
        g = random_graph(50, 0.05, 1)
        bad = matgen.Graph(g.n, g.beg, g.end, np.where(g.adj == g.adj[0], 99, g.adj).astype(np.int32))
        with pytest.raises(gsofa_b200.GsofaError) as e:
            srv.submit(bad)
        assert e.value.status == 1
        rid = srv.submit(g)      # still usable
        import time
        t0 = time.time()
        done = []
        while not done and time.time() - t0 < 30:
            done = srv.poll()
        assert done == [rid]
        srv.result(rid)


def test_size_classes_match_standalone_and_free_large_requests():
    """Requests above max_n run alone on the factorization kernel (the large
    class), the rest on the serving kernel; every result equals a standalone
    factorization, and the large requests' matrices are freed."""
    reqs = serve.make_stream(24, 200, 4000, rate_hz=2000.0, seed=23, build=matgen.make)
    with gsofa_b200.Context(0) as ctx, gsofa_b200.StreamServer(0, mem_budget_bytes=8 << 30,
                                                              max_supernode_size=16) as srv:
        params = gsofa_b200.Params.default(want_pattern=0, max_supernode_size=16)
        cs = serve.ContinuousServer(srv, oversize=lambda g: serve.run_alone(ctx, g, params), max_n=1500)
        out = cs.run(reqs)
        assert out["report"]["run_alone"] == sum(1 for r in reqs if r.graph.n > 1500) > 0
        assert ctx._mats == []
        for c in out["completions"]:
            g = reqs[c.rid].graph
            with ctx.upload(g) as m:
                _same(c.result, ctx.symbfact(m, params), f"request {c.rid} (n={g.n})")
        assert ctx._mats == []
