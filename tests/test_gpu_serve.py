"""Serving loop: continuous batching gives every request the result it gets
alone, and reports latency percentiles."""
import numpy as np
import pytest

import gsofa_b200
from gsofa_b200 import matgen, serve

pytestmark = pytest.mark.gpu


def test_results_identical_alone_and_in_the_mix():
    reqs = serve.make_stream(24, 200, 4000, rate_hz=400.0, seed=11, build=matgen.make)
    with gsofa_b200.Context(0) as ctx:
        p = gsofa_b200.Params.default(want_pattern=0, max_supernode_size=16)
        out = serve.Server(ctx, p, max_batch=8).run(reqs)
        rep = out["report"]
        assert rep["requests"] == len(reqs)
        assert rep["launches"] < len(reqs)          # requests were batched
        assert rep["p50_ms"] <= rep["p99_ms"]
        for c, r in zip(out["completions"], reqs):
            alone = ctx.symbfact(ctx.upload(r.graph), p)
            got = c.result
            assert (got.fill_count, got.nnz_lu, got.n_supernodes) == \
                   (alone.fill_count, alone.nnz_lu, alone.n_supernodes), r.rid
            assert np.array_equal(got.u_row_count, alone.u_row_count)
            assert np.array_equal(got.l_col_count, alone.l_col_count)
            assert np.array_equal(got.sn_start, alone.sn_start)
        single = serve.one_at_a_time(ctx, reqs, p)["report"]
        assert single["launches"] == len(reqs)


def test_admission_respects_the_budget():
    g = matgen.grid3d(10, seed=1)
    with gsofa_b200.Context(0) as ctx:
        srv = serve.Server(ctx, gsofa_b200.Params.default(want_pattern=0), mem_budget_bytes=1 << 20)
        with pytest.raises(ValueError):
            srv.run([serve.Request(0, 0.0, g)])
