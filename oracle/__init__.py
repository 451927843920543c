"""CPU oracle for gSoFa symbolic factorization -- TEST INFRASTRUCTURE ONLY.

Only the test-suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker.  The shipped
library (``gsofa_b200``) never imports, links or calls it.

The C restatement lives in ``gsofa_oracle.c`` (see its header for the
reference lines each function follows).  This module loads the compiled
``liboracle.so`` through ctypes and assembles the same result record the GPU
library returns, so tests can compare them field by field.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_u64p = ctypes.POINTER(ctypes.c_uint64)


def build() -> str:
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.gsofa_oracle_counts.argtypes = [ctypes.c_int32, _i32p, _i32p, _i32p, ctypes.c_int64,
                                          ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int32,
                                          _i32p, _i32p, _u8p, _u64p]
        L.gsofa_oracle_counts.restype = ctypes.c_int
        L.gsofa_oracle_pattern.argtypes = [ctypes.c_int32, _i32p, _i32p, _i32p, ctypes.c_int64,
                                           ctypes.c_int, ctypes.c_int, _i64p, _i32p]
        L.gsofa_oracle_pattern.restype = ctypes.c_int
        L.gsofa_oracle_supernodes.argtypes = [ctypes.c_int32, _i32p, _u8p, _u8p, ctypes.c_int32, _i32p]
        L.gsofa_oracle_supernodes.restype = ctypes.c_int32
        L.gsofa_oracle_maxid_fills.argtypes = [ctypes.c_int32, _i32p, _i32p, _i32p, ctypes.c_int64,
                                               ctypes.c_int, _i64p, _i64p]
        L.gsofa_oracle_maxid_fills.restype = ctypes.c_int64
        L.gsofa_oracle_threads.argtypes = []
        L.gsofa_oracle_threads.restype = ctypes.c_int
        L.gsofa_oracle_maxid_counts.argtypes = [ctypes.c_int32, _i32p, _i32p, _i32p, ctypes.c_int64,
                                                ctypes.c_int, _i32p, ctypes.c_int32, _i64p, _i64p]
        L.gsofa_oracle_maxid_counts.restype = ctypes.c_int64
        L.gsofa_oracle_lists.argtypes = [ctypes.c_int32, _i32p, _i32p, _i32p, ctypes.c_int64,
                                         ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_int32, _i64p, _i32p]
        L.gsofa_oracle_lists.restype = ctypes.c_int
        L.gsofa_oracle_maxid_line.argtypes = [ctypes.c_int32, _i32p, _i32p, _i32p, ctypes.c_int64,
                                              ctypes.c_int32, _i32p]
        L.gsofa_oracle_maxid_line.restype = ctypes.c_int32
        L.gsofa_oracle_rcm.argtypes = [ctypes.c_int32, _i32p, _i32p, _i32p, ctypes.c_int64, _i32p]
        L.gsofa_oracle_rcm.restype = ctypes.c_int
        _lib = L
    return _lib


def threads() -> int:
    """Threads the OpenMP restatements use by default."""
    return int(lib().gsofa_oracle_threads())


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def _inputs(beg, end, adj):
    beg = np.ascontiguousarray(beg, dtype=np.int32)
    end = np.ascontiguousarray(end, dtype=np.int32)
    adj = np.ascontiguousarray(adj, dtype=np.int32)
    return beg, end, adj


def counts(beg, end, adj, pass_: int, nthreads: int = 0, sources=None):
    """Per-line |hi(s)|, distinct original entries > s, the s+1 link flag and
    the work counters (|X|, E_insp) of one reachability pass (0: G, 1: G^T)."""
    beg, end, adj = _inputs(beg, end, adj)
    n = beg.shape[0]
    cnt = np.zeros(n, np.int32)
    orig = np.zeros(n, np.int32)
    nxt = np.zeros(n, np.uint8)
    work = np.zeros(2, np.uint64)
    src = None if sources is None else np.ascontiguousarray(sources, dtype=np.int32)
    rc = lib().gsofa_oracle_counts(n, _p(beg, _i32p), _p(end, _i32p), _p(adj, _i32p), adj.shape[0],
                                   pass_, nthreads, _p(src, _i32p), 0 if src is None else src.shape[0],
                                   _p(cnt, _i32p), _p(orig, _i32p), _p(nxt, _u8p), _p(work, _u64p))
    if rc != 0:
        raise ValueError(f"oracle counts failed (rc={rc})")
    return cnt, orig, nxt, work


def pattern(beg, end, adj, pass_: int, cnt, nthreads: int = 0):
    """Sorted hi(s) lists of one pass as (ptr int64[n+1], idx int32[])."""
    beg, end, adj = _inputs(beg, end, adj)
    n = beg.shape[0]
    ptr = np.zeros(n + 1, np.int64)
    np.cumsum(cnt, out=ptr[1:])
    idx = np.zeros(int(ptr[-1]), np.int32)
    rc = lib().gsofa_oracle_pattern(n, _p(beg, _i32p), _p(end, _i32p), _p(adj, _i32p), adj.shape[0],
                                    pass_, nthreads, _p(ptr, _i64p), _p(idx, _i32p))
    if rc != 0:
        raise ValueError(f"oracle pattern failed (rc={rc})")
    return ptr, idx


def supernodes(ucnt, unext, lnext, max_size: int):
    ucnt = np.ascontiguousarray(ucnt, dtype=np.int32)
    unext = np.ascontiguousarray(unext, dtype=np.uint8)
    lnext = np.ascontiguousarray(lnext, dtype=np.uint8)
    n = ucnt.shape[0]
    out = np.zeros(max(n, 1), np.int32)
    k = lib().gsofa_oracle_supernodes(n, _p(ucnt, _i32p), _p(unext, _u8p), _p(lnext, _u8p),
                                      int(max_size), _p(out, _i32p))
    return out[:k].copy()


def maxid_fills(beg, end, adj, nthreads: int = 0):
    """Faithful max-id traversal: (total, fills_lo[n], fills_hi[n])."""
    beg, end, adj = _inputs(beg, end, adj)
    n = beg.shape[0]
    lo = np.zeros(n, np.int64)
    hi = np.zeros(n, np.int64)
    tot = lib().gsofa_oracle_maxid_fills(n, _p(beg, _i32p), _p(end, _i32p), _p(adj, _i32p),
                                         adj.shape[0], nthreads, _p(lo, _i64p), _p(hi, _i64p))
    if tot < 0:
        raise ValueError("oracle max-id traversal failed")
    return int(tot), lo, hi


def maxid_counts(beg, end, adj, sources, nthreads: int = 0):
    """Faithful max-id traversal of the listed lines only: (total fills,
    fills_lo[n], fills_hi[n]) with entries set at those lines."""
    beg, end, adj = _inputs(beg, end, adj)
    n = beg.shape[0]
    src = np.ascontiguousarray(sources, dtype=np.int32)
    lo = np.zeros(n, np.int64)
    hi = np.zeros(n, np.int64)
    tot = lib().gsofa_oracle_maxid_counts(n, _p(beg, _i32p), _p(end, _i32p), _p(adj, _i32p), adj.shape[0],
                                          nthreads, _p(src, _i32p), src.shape[0], _p(lo, _i64p), _p(hi, _i64p))
    if tot < 0:
        raise ValueError("oracle max-id traversal failed")
    return int(tot), lo, hi


def lists(beg, end, adj, pass_: int, sources, cnt, nthreads: int = 0):
    """Sorted hi(s) lists of one pass for the listed (distinct) sources, as
    (ptr int64[k+1], idx int32[]) in the order given; cnt holds the per-line
    counts of that pass (at least at the listed lines)."""
    beg, end, adj = _inputs(beg, end, adj)
    n = beg.shape[0]
    src = np.ascontiguousarray(sources, dtype=np.int32)
    ptr = np.zeros(src.shape[0] + 1, np.int64)
    np.cumsum(np.asarray(cnt)[src], out=ptr[1:])
    idx = np.zeros(int(ptr[-1]), np.int32)
    rc = lib().gsofa_oracle_lists(n, _p(beg, _i32p), _p(end, _i32p), _p(adj, _i32p), adj.shape[0], pass_,
                                  nthreads, _p(src, _i32p), src.shape[0], _p(ptr, _i64p), _p(idx, _i32p))
    if rc != 0:
        raise ValueError(f"oracle lists failed (rc={rc})")
    return ptr, idx


def maxid_line(beg, end, adj, s: int):
    """Sorted fills of line s from the faithful max-id traversal."""
    beg, end, adj = _inputs(beg, end, adj)
    n = beg.shape[0]
    out = np.zeros(max(n, 1), np.int32)
    k = lib().gsofa_oracle_maxid_line(n, _p(beg, _i32p), _p(end, _i32p), _p(adj, _i32p),
                                      adj.shape[0], int(s), _p(out, _i32p))
    if k < 0:
        raise ValueError("oracle max-id line failed")
    return out[:k].copy()


def symbfact(beg, end, adj, want_pattern: bool = True, max_supernode_size: int = 0,
             nthreads: int = 0) -> dict:
    """The full oracle result record (same field names as gsofa_b200.Result)."""
    beg, end, adj = _inputs(beg, end, adj)
    n = beg.shape[0]
    ucnt, uorig, unext, work = counts(beg, end, adj, 0, nthreads)
    lcnt, lorig, lnext, _ = counts(beg, end, adj, 1, nthreads)
    res = {
        "n": n,
        "u_row_count": ucnt,
        "l_col_count": lcnt,
        "u_next": unext,
        "l_next": lnext,
        "x_total": int(work[0]),
        "e_insp": int(work[1]),
        "fill_count": int(ucnt.sum(dtype=np.int64) - uorig.sum(dtype=np.int64)
                          + lcnt.sum(dtype=np.int64) - lorig.sum(dtype=np.int64)),
        "nnz_lu": int(ucnt.sum(dtype=np.int64) + lcnt.sum(dtype=np.int64) + n),
    }
    res["sn_start"] = supernodes(ucnt, unext, lnext, max_supernode_size)
    if want_pattern:
        uptr, uidx = pattern(beg, end, adj, 0, ucnt, nthreads)
        lptr, lidx = pattern(beg, end, adj, 1, lcnt, nthreads)
        res.update(u_ptr=uptr, u_idx=uidx, l_ptr=lptr, l_idx=lidx)
        res["l_row_count"] = np.bincount(lidx, minlength=n).astype(np.int32)
    return res


def rcm(beg, end, adj):
    """Reverse Cuthill-McKee order of A + A^T (perm[new] = old), with the
    tie-breaking rules of gsofa_oracle.c."""
    beg, end, adj = _inputs(beg, end, adj)
    n = beg.shape[0]
    perm = np.zeros(n, np.int32)
    rc = lib().gsofa_oracle_rcm(n, _p(beg, _i32p), _p(end, _i32p), _p(adj, _i32p), adj.shape[0], _p(perm, _i32p))
    if rc != 0:
        raise ValueError(f"oracle rcm failed (rc={rc})")
    return perm
