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


class _FakeServer:
    """The StreamServer interface with the oracle standing in for the GPU
    kernel: a request is done on the poll after its submission."""

    def __init__(self, cap=3):
        import oracle
        self._oracle = oracle
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
        import numpy as np
        from gsofa_b200 import Result
        g = self.live.pop(rid)
        r = self._oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False)
        return Result(n=g.n, fill_count=r["fill_count"], nnz_lu=r["nnz_lu"], nnz_u=0, nnz_l=0,
                      n_supernodes=len(r["sn_start"]), edges_inspected=0, sources=0, x_total=0,
                      e_insp=0, kernel_ms=0.0, u_row_count=r["u_row_count"],
                      sn_start=np.asarray(r["sn_start"]))

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
