"""Shared helpers of the test-suite: fixtures, random graphs, comparisons."""
import json
import os

import numpy as np

from gsofa_b200.matgen import Graph

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def expected():
    with open(os.path.join(GOLDEN, "expected.json")) as f:
        return json.load(f)


def bundled() -> Graph:
    z = np.load(os.path.join(GOLDEN, "bundled_11948.npz"))
    return Graph(int(z["n"]), z["beg"], z["end"], z["adj"], "bundled_11948")


def random_graph(n: int, density: float, seed: int, shuffle_ranges=True, dups=True,
                 diag=True, unsorted=True) -> Graph:
    """A random directed pattern in the reference's free-form line layout:
    ranges placed in random order inside adj, unsorted lists, duplicates and
    diagonal entries, empty lines."""
    rng = np.random.default_rng(seed)
    lines = []
    for v in range(n):
        k = rng.binomial(n, density) if n > 0 else 0
        cols = rng.integers(0, n, size=k) if n > 0 else np.zeros(0, np.int64)
        if diag and rng.random() < 0.7:
            cols = np.append(cols, v)
        if dups and k > 0 and rng.random() < 0.3:
            cols = np.append(cols, cols[: rng.integers(1, k + 1)])
        if unsorted:
            rng.shuffle(cols)
        else:
            cols = np.unique(cols)
        lines.append(cols.astype(np.int32))
    order = rng.permutation(n) if shuffle_ranges else np.arange(n)
    beg = np.zeros(n, np.int32)
    end = np.zeros(n, np.int32)
    chunks = []
    pos = 0
    for v in order:
        # occasional gap of unused entries between ranges
        if shuffle_ranges and rng.random() < 0.2:
            gap = rng.integers(0, max(n, 1), size=int(rng.integers(1, 4))).astype(np.int32)
            chunks.append(gap)
            pos += gap.shape[0]
        beg[v] = pos
        chunks.append(lines[v])
        pos += lines[v].shape[0]
        end[v] = pos
    adj = np.concatenate(chunks).astype(np.int32) if chunks else np.zeros(0, np.int32)
    return Graph(n, beg, end, adj, f"random_{n}_{density}_{seed}")


def lower_rows(res_l_ptr, res_l_idx, n):
    """L by columns -> for each row s the sorted columns j < s."""
    cols = np.repeat(np.arange(n, dtype=np.int64), np.diff(res_l_ptr))
    rows = res_l_idx.astype(np.int64)
    order = np.lexsort((cols, rows))
    rows, cols = rows[order], cols[order]
    ptr = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=ptr[1:])
    return ptr, cols


FIELDS_ALWAYS = ("fill_count", "nnz_lu", "u_row_count", "l_col_count", "sn_start")
FIELDS_PATTERN = ("u_ptr", "u_idx", "l_ptr", "l_idx", "l_row_count")


def assert_same(gpu, ref: dict, pattern: bool = True, where: str = ""):
    """Bit-exact comparison of a gsofa_b200.Result with an oracle record."""
    for f in FIELDS_ALWAYS + (FIELDS_PATTERN if pattern else ()):
        g = getattr(gpu, f)
        r = ref[f]
        if isinstance(r, np.ndarray):
            assert g is not None, f"{where}: {f} missing"
            assert g.shape == r.shape, f"{where}: {f} shape {g.shape} != {r.shape}"
            if not np.array_equal(g, r):
                bad = np.nonzero(g != r)[0][:5]
                raise AssertionError(f"{where}: {f} differs at {bad.tolist()}: "
                                     f"{g[bad].tolist()} != {r[bad].tolist()}")
        else:
            assert int(g) == int(r), f"{where}: {f} {g} != {r}"


def supernodal_reference(ref: dict) -> dict:
    """The supernodal structure built from an oracle result with the pattern:
    per supernode, the diagonal block's rows then the rows below it of its
    last column, and the columns right of the block of its first row."""
    n = ref["n"]
    up, ui, lp, li = ref["u_ptr"], ref["u_idx"], ref["l_ptr"], ref["l_idx"]
    xsup = np.append(np.asarray(ref["sn_start"], np.int64), n)
    lsub, usub, xl, xu = [], [], [0], [0]
    supno = np.zeros(n, np.int32)
    for k in range(len(xsup) - 1):
        f, l = int(xsup[k]), int(xsup[k + 1])
        supno[f:l] = k
        rows = np.concatenate([np.arange(f, l), li[lp[l - 1]:lp[l]]])
        cols = ui[up[f]:up[f + 1]][l - f - 1:]
        lsub.append(rows)
        usub.append(cols)
        xl.append(xl[-1] + len(rows))
        xu.append(xu[-1] + len(cols))
    cat = lambda parts: np.concatenate(parts).astype(np.int32) if parts else np.zeros(0, np.int32)  # noqa: E731
    return {"xsup": xsup.astype(np.int32), "supno": supno, "xlsub": np.array(xl, np.int64),
            "lsub": cat(lsub), "xusub": np.array(xu, np.int64), "usub": cat(usub)}
