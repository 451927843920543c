"""Seeded generators for the synthetic matrices the benchmarks run on.

The reference measures on SuperLU_DIST-reordered SuiteSparse matrices (the
bundled n = 11,948 dump and pre2).  These generators produce seeded stand-ins
with the shapes, sizes and orderings of the named workloads:

* ``grid2d``   -- 5-point Laplacian pattern, natural row-major ordering
                  (64x64: n = 4,096, nnz = 20,224).
* ``grid3d``   -- 7-point stencil pattern, geometric nested dissection
                  (recursive bisection of the longest axis, separator planes
                  numbered last), one side of a seeded 10% of off-diagonal
                  pairs dropped, diagonal kept (80^3: n = 512,000).
* ``powerlaw`` -- circuit-like unsymmetric pattern: power-law off-diagonal row
                  degrees (alpha 2.1, mean ~8, cap 4,000), 70% of columns
                  within +/-64 of the row and 30% uniform, full diagonal,
                  ordered by a seeded random permutation followed by reverse
                  Cuthill-McKee (n = 659,033: ~5.9M nonzeros).

Every matrix is returned as a :class:`Graph` in the reference's line layout
(``beg``/``end`` offsets into ``adj``; here contiguous, sorted, one line per
row).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Graph:
    """A matrix pattern in gSoFa's colbeg/colend/csr line layout."""

    n: int
    beg: np.ndarray  # int32[n]
    end: np.ndarray  # int32[n]
    adj: np.ndarray  # int32[nnz]
    name: str = ""

    @property
    def nnz(self) -> int:
        return int(self.adj.shape[0])

    @staticmethod
    def from_csr(rowptr: np.ndarray, col: np.ndarray, name: str = "") -> "Graph":
        rowptr = np.asarray(rowptr, dtype=np.int64)
        n = rowptr.shape[0] - 1
        return Graph(n, rowptr[:-1].astype(np.int32), rowptr[1:].astype(np.int32),
                     np.ascontiguousarray(col, dtype=np.int32), name)


def _csr_from_pairs(n: int, rows: np.ndarray, cols: np.ndarray, name: str) -> Graph:
    """Sorted, duplicate-free CSR from (row, col) pairs."""
    key = rows.astype(np.int64) * n + cols.astype(np.int64)
    key = np.unique(key)
    r = (key // n).astype(np.int64)
    c = (key % n).astype(np.int32)
    rowptr = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(r, minlength=n), out=rowptr[1:])
    return Graph.from_csr(rowptr, c, name)


def _permute(n: int, rows: np.ndarray, cols: np.ndarray, new_id: np.ndarray):
    return new_id[rows], new_id[cols]


# ----------------------------------------------------------------------------
# Orderings


def nested_dissection_order(dims) -> np.ndarray:
    """Geometric nested dissection of a box grid.

    Returns ``new_id[g]`` for grid index g = x + nx*(y + ny*z) (2D: z absent).
    A box is split at the middle plane of its longest axis (ties: lowest axis);
    the lower half is numbered first, then the upper half, then the separator
    plane in natural order.  Boxes whose longest side is <= 2 are numbered
    naturally.
    """
    dims = tuple(int(d) for d in dims)
    nd = len(dims)
    strides = [1]
    for d in dims[:-1]:
        strides.append(strides[-1] * d)
    n = int(np.prod(dims))
    order = np.empty(n, np.int64)
    pos = 0

    def natural(lo, hi):
        axes = [np.arange(lo[a], hi[a], dtype=np.int64) * strides[a] for a in range(nd)]
        g = axes[0]
        for a in range(1, nd):
            g = (axes[a][:, None] + g[None, :]).reshape(-1)
        return g

    stack = [(tuple(0 for _ in dims), dims, False)]
    # Explicit stack: entries are (lo, hi, is_separator).  Children are pushed in
    # reverse so the lower half is numbered first.
    while stack:
        lo, hi, sep = stack.pop()
        ext = [hi[a] - lo[a] for a in range(nd)]
        if min(ext) <= 0:
            continue
        if sep or max(ext) <= 2:
            g = natural(lo, hi)
            order[pos:pos + g.shape[0]] = g
            pos += g.shape[0]
            continue
        a = int(np.argmax(ext))
        mid = lo[a] + ext[a] // 2
        lo_hi = list(hi); lo_hi[a] = mid
        up_lo = list(lo); up_lo[a] = mid + 1
        s_lo = list(lo); s_lo[a] = mid
        s_hi = list(hi); s_hi[a] = mid + 1
        stack.append((tuple(s_lo), tuple(s_hi), True))
        stack.append((tuple(up_lo), tuple(hi), False))
        stack.append((tuple(lo), tuple(lo_hi), False))
    assert pos == n
    new_id = np.empty(n, np.int64)
    new_id[order] = np.arange(n, dtype=np.int64)
    return new_id


def rcm_order(n: int, rows: np.ndarray, cols: np.ndarray) -> np.ndarray:
    """Reverse Cuthill-McKee on the symmetrised pattern; returns new_id[old]."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import reverse_cuthill_mckee

    A = sp.csr_matrix((np.ones(rows.shape[0], np.int8), (rows, cols)), shape=(n, n))
    S = (A + A.T).tocsr()
    S.sort_indices()
    perm = reverse_cuthill_mckee(S, symmetric_mode=True)  # perm[new] = old
    new_id = np.empty(n, np.int64)
    new_id[perm] = np.arange(n, dtype=np.int64)
    return new_id


# ----------------------------------------------------------------------------
# Patterns


def _grid_edges(dims):
    """Undirected nearest-neighbour pairs (u < v) of a box grid."""
    dims = tuple(int(d) for d in dims)
    n = int(np.prod(dims))
    g = np.arange(n, dtype=np.int64)
    coords = []
    rem = g.copy()
    for d in dims:
        coords.append(rem % d)
        rem //= d
    stride = 1
    us, vs = [], []
    for a, d in enumerate(dims):
        m = coords[a] < d - 1
        us.append(g[m])
        vs.append(g[m] + stride)
        stride *= d
    return n, np.concatenate(us), np.concatenate(vs)


def _grid_graph(dims, ordering: str, drop_frac: float, seed: int, name: str) -> Graph:
    n, u, v = _grid_edges(dims)
    rng = np.random.default_rng(seed)
    if drop_frac > 0:
        sel = rng.random(u.shape[0]) < drop_frac
        side = rng.random(u.shape[0]) < 0.5
        keep_uv = ~(sel & side)      # drop u->v where selected and side
        keep_vu = ~(sel & ~side)     # drop v->u otherwise
        rows = np.concatenate([u[keep_uv], v[keep_vu]])
        cols = np.concatenate([v[keep_uv], u[keep_vu]])
    else:
        rows = np.concatenate([u, v])
        cols = np.concatenate([v, u])
    diag = np.arange(n, dtype=np.int64)
    rows = np.concatenate([rows, diag])
    cols = np.concatenate([cols, diag])
    if ordering == "nd":
        new_id = nested_dissection_order(dims)
        rows, cols = _permute(n, rows, cols, new_id)
    elif ordering != "natural":
        raise ValueError(f"unknown ordering {ordering!r}")
    return _csr_from_pairs(n, rows, cols, name)


def grid2d(nx: int, ny: int | None = None, ordering: str = "natural", drop_frac: float = 0.0,
           seed: int = 0) -> Graph:
    """5-point stencil on an nx x ny grid (x fastest)."""
    ny = nx if ny is None else ny
    return _grid_graph((nx, ny), ordering, drop_frac, seed, f"grid2d_{nx}x{ny}_{ordering}")


def grid3d(nx: int, ny: int | None = None, nz: int | None = None, ordering: str = "nd",
           drop_frac: float = 0.1, seed: int = 0) -> Graph:
    """7-point stencil on an nx x ny x nz grid."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    return _grid_graph((nx, ny, nz), ordering, drop_frac, seed,
                       f"grid3d_{nx}x{ny}x{nz}_{ordering}_drop{drop_frac:g}")


# Continuous Pareto scale giving a mean off-diagonal degree of ~8 for
# alpha = 2.1 after flooring, the 4,000 cap and duplicate removal.
_PL_XMIN = 1.72


def powerlaw(n: int, alpha: float = 2.1, cap: int = 4000, local_frac: float = 0.7,
             local_width: int = 64, seed: int = 0, ordering: str = "rcm") -> Graph:
    """Circuit-like unsymmetric pattern with power-law row degrees."""
    rng = np.random.default_rng(seed)
    u = rng.random(n)
    deg = np.floor(_PL_XMIN * (1.0 - u) ** (-1.0 / (alpha - 1.0)))
    deg = np.minimum(deg, min(cap, max(n - 1, 0))).astype(np.int64)
    total = int(deg.sum())
    rows = np.repeat(np.arange(n, dtype=np.int64), deg)
    local = rng.random(total) < local_frac
    off = rng.integers(1, local_width + 1, size=total) * np.where(rng.random(total) < 0.5, -1, 1)
    lc = rows + off
    lc = np.where(lc < 0, -lc, lc)                       # reflect at the edges
    lc = np.where(lc >= n, 2 * (n - 1) - lc, lc)
    lc = np.clip(lc, 0, n - 1)
    uc = rng.integers(0, n, size=total)
    cols = np.where(local, lc, uc).astype(np.int64)
    keep = cols != rows
    rows, cols = rows[keep], cols[keep]
    diag = np.arange(n, dtype=np.int64)
    rows = np.concatenate([rows, diag])
    cols = np.concatenate([cols, diag])
    if ordering in ("rcm", "random"):
        perm = rng.permutation(n).astype(np.int64)      # new_id after the shuffle
        rows, cols = perm[rows], perm[cols]
        if ordering == "rcm":
            new_id = rcm_order(n, rows, cols)
            rows, cols = new_id[rows], new_id[cols]
    elif ordering != "natural":
        raise ValueError(f"unknown ordering {ordering!r}")
    return _csr_from_pairs(n, rows, cols, f"powerlaw_{n}_{ordering}")


def bordered_blocks(n_blocks: int, block: int = 32, border: int = 8, per_line: int = 5,
                    seed: int = 0) -> Graph:
    """Bordered block-diagonal pattern, the shape nested dissection gives at
    its top level: `n_blocks` diagonal blocks of `block` lines (each line with
    `per_line` seeded entries inside its block), then `border` separator lines
    numbered last.  Every block couples to one or two random border lines
    (entries both ways) and the border lines to each other.  A traversal from
    a block line stays inside its block (border lines are numbered above it),
    so X(s) holds at most `block` lines and any n stays cheap for the oracle;
    only the border lines traverse the whole matrix."""
    rng = np.random.default_rng(seed)
    nb = n_blocks * block
    n = nb + border
    rows = np.repeat(np.arange(nb, dtype=np.int64), per_line)
    base = (rows // block) * block
    cols = base + rng.integers(0, block, size=rows.shape[0])
    # block -> border couplings (one or two per block, both directions)
    k = rng.integers(1, 3, size=n_blocks)
    blk = np.repeat(np.arange(n_blocks, dtype=np.int64), k)
    line = blk * block + rng.integers(0, block, size=blk.shape[0])
    sep = nb + rng.integers(0, border, size=blk.shape[0])
    # border lines: a ring among themselves
    b = np.arange(border, dtype=np.int64)
    diag = np.arange(n, dtype=np.int64)
    r = np.concatenate([rows, line, sep, nb + b, diag])
    c = np.concatenate([cols, sep, line, nb + (b + 1) % border, diag])
    return _csr_from_pairs(n, r, c, f"bordered_{n_blocks}x{block}+{border}")


# ----------------------------------------------------------------------------
# The named workloads

SEEDS = {"plain2d": 1, "nd3d": 2, "circuit": 3, "batch": 4, "serve": 5}


def config_plain2d() -> Graph:
    """64x64 5-point Laplacian, natural ordering (n = 4,096)."""
    return grid2d(64, 64, "natural")


def config_nd3d(side: int = 80) -> Graph:
    """80^3 7-point stencil, geometric ND, 10% one-sided drops (n = 512,000)."""
    return grid3d(side, side, side, "nd", 0.1, SEEDS["nd3d"])


def config_circuit(n: int = 659_033) -> Graph:
    """Power-law circuit-like pattern with RCM ordering (n = 659,033)."""
    return powerlaw(n, seed=SEEDS["circuit"])


def mixed_spec(count: int, n_lo: int, n_hi: int, seed: int):
    """(kind, n, seed) triples: n log-uniform in [n_lo, n_hi], kinds mixed."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(math.log(n_lo), math.log(n_hi), size=count))
    kinds = rng.integers(0, 3, size=count)
    seeds = rng.integers(0, 2**31 - 1, size=count)
    names = ("grid2d", "grid3d", "powerlaw")
    return [(names[int(k)], int(round(x)), int(s)) for k, x, s in zip(kinds, ns, seeds)]


def make(kind: str, n: int, seed: int) -> Graph:
    """One matrix of a mix: the grid side is chosen so the size is close to n."""
    if kind == "grid2d":
        side = max(2, int(round(math.sqrt(n))))
        return grid2d(side, side, "natural")
    if kind == "grid3d":
        side = max(2, int(round(n ** (1.0 / 3.0))))
        return grid3d(side, side, side, "nd", 0.1, seed)
    if kind == "powerlaw":
        return powerlaw(max(n, 2), seed=seed)
    raise ValueError(kind)


def config_batch(count: int = 256, n_lo: int = 2_000, n_hi: int = 200_000):
    """The mixed-size batch: specs of `count` matrices (build with make())."""
    return mixed_spec(count, n_lo, n_hi, SEEDS["batch"])


def config_serve(count: int = 10_000, n_lo: int = 1_000, n_hi: int = 1_000_000, rate_hz: float = 50.0):
    """The serving stream: (arrival_s, kind, n, seed) with Poisson arrivals."""
    spec = mixed_spec(count, n_lo, n_hi, SEEDS["serve"])
    rng = np.random.default_rng(SEEDS["serve"] + 1)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, size=count))
    return [(float(a), k, n, s) for a, (k, n, s) in zip(t, spec)]
