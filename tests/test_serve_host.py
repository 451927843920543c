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
