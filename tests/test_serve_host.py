"""Host-side pieces of the serving loop (no GPU)."""
from gsofa_b200 import matgen, serve


def test_stream_is_seeded_and_ordered():
    a = serve.make_stream(30, 100, 2000, 50.0, 3, matgen.make)
    b = serve.make_stream(30, 100, 2000, 50.0, 3, matgen.make)
    assert [r.arrival_s for r in a] == [r.arrival_s for r in b]
    assert all(x.arrival_s < y.arrival_s for x, y in zip(a, a[1:]))
    assert all(ra.graph.nnz == rb.graph.nnz for ra, rb in zip(a, b))


def test_matrix_bytes_grow_with_size():
    small, big = matgen.grid2d(10), matgen.grid2d(40)
    assert 0 < serve.matrix_bytes(small) < serve.matrix_bytes(big)


def _oracle_result(g):
    """A Result for g computed by the oracle (counts only)."""
    import numpy as np
    import oracle
    from gsofa_b200 import Result
    r = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False)
    return Result(n=g.n, fill_count=r["fill_count"], nnz_lu=r["nnz_lu"], nnz_u=0, nnz_l=0,
                  n_supernodes=len(r["sn_start"]), edges_inspected=0, sources=0, x_total=0,
                  e_insp=0, kernel_ms=0.0, u_row_count=r["u_row_count"],
                  sn_start=np.asarray(r["sn_start"]))


class _FakeServer:
    """The StreamServer interface with the oracle standing in for the GPU
    kernel: a request is done on the poll after its submission."""

    def __init__(self, cap=3):
        self.cap = cap
        self.live = {}
        self.next_id = 1

    def submit(self, g):
        if len(self.live) >= self.cap:
            return None                     # no room now: the loop must wait
        rid = self.next_id
        self.next_id += 1
        self.live[rid] = g
        return rid

    def poll(self):
        return list(self.live)

    def result(self, rid):
        return _oracle_result(self.live.pop(rid))

    def drain(self):
        pass


def _make(spec):
    k, n, s = spec
    return matgen.make(k, n, s)


def test_lazy_stream_is_served_in_full_with_bounded_admission():
    """A stream whose matrices a spawn pool builds while it is served: every
    request completes once, its latency counts from when it could arrive, and
    only the first keep_graphs requests keep their matrices."""
    import multiprocessing as mp
    import numpy as np
    import oracle
    spec = matgen.mixed_spec(24, 100, 1500, 7)
    arrivals = np.cumsum(np.full(len(spec), 0.002))
    with mp.get_context("spawn").Pool(2) as pool:
        stream = serve.LazyStream(pool, _make, spec, arrivals, ahead=5)
        out = serve.ContinuousServer(_FakeServer(cap=3)).run(stream, keep_graphs=4)
    done = out["completions"]
    assert sorted(c.rid for c in done) == list(range(len(spec)))
    assert out["report"]["requests"] == len(spec)
    for c in done:
        assert c.done_s >= c.start_s >= c.arrival_s - 1e-9 and c.arrival_s >= arrivals[c.rid] - 1e-9
        g = _make(spec[c.rid])
        assert c.result.fill_count == oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False)["fill_count"]
    assert all(r.graph is not None for r in stream.reqs[:4])
    assert all(r.graph is None for r in stream.reqs[4:])


class _FakeContext:
    """The Context calls Server makes, with the oracle standing in for the GPU."""

    def __init__(self):
        self.launches = []

    def predict_scratch_bytes(self, n, nnz, params):
        return 64 * n

    def upload(self, g):
        class _M:
            def __init__(self, g):
                self.g = g

            def free(self):
                pass
        return _M(g)

    def symbfact_batch(self, mats, params):
        self.launches.append(len(mats))
        return [_oracle_result(m.g) for m in mats]


def test_one_request_per_launch_serves_every_request():
    import numpy as np
    import oracle
    spec = matgen.mixed_spec(6, 100, 800, 3)
    reqs = [serve.Request(i, 0.001 * i, matgen.make(*s)) for i, s in enumerate(spec)]
    ctx = _FakeContext()
    out = serve.one_at_a_time(ctx, reqs)
    assert ctx.launches == [1] * len(reqs)
    rep = out["report"]
    assert rep["requests"] == len(reqs) and rep["launches"] == len(reqs) and rep["mean_batch"] == 1.0
    for c, r in zip(out["completions"], reqs):
        assert c.rid == r.rid
        assert c.result.fill_count == oracle.symbfact(r.graph.beg, r.graph.end, r.graph.adj,
                                                      want_pattern=False)["fill_count"]
        assert np.isfinite(c.latency_s) and c.latency_s >= 0


def test_large_requests_run_alone_after_a_drain():
    """Requests above max_n (the large class) go through `oversize`, each once,
    after what runs on the serving kernel has finished; the rest are served
    by the serving kernel."""
    import oracle
    spec = [("grid2d", 300, 1), ("grid2d", 2500, 2), ("grid3d", 400, 3), ("powerlaw", 3000, 4),
            ("grid2d", 200, 5)]
    reqs = [serve.Request(i, 0.0005 * i, matgen.make(*s)) for i, s in enumerate(spec)]
    fake = _FakeServer(cap=2)
    drains = []
    fake.drain = lambda: drains.append(len(fake.live))
    alone = []

    def oversize(g):
        alone.append(g.n)
        return _oracle_result(g)

    out = serve.ContinuousServer(fake, oversize=oversize, max_n=1000).run(reqs)
    assert out["report"]["requests"] == len(reqs)
    assert out["report"]["run_alone"] == len(alone) == sum(1 for r in reqs if r.graph.n > 1000)
    assert all(d == 0 for d in drains) and len(drains) == len(alone)
    for c in out["completions"]:
        g = reqs[c.rid].graph
        assert c.result.fill_count == oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False)["fill_count"]
