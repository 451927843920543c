"""Autotuner for the factorization launch parameters.

Chooses (threads per CTA, lanes per frontier vertex, sources per work piece)
from measured kernel times on the caller's own matrices, and caches the
choice per workload signature (size buckets of n and nnz, matrix count) in a
JSON file, so later runs skip the search.  The parameters only change speed:
every choice returns bit-identical results.
"""
from __future__ import annotations

import json
import math
import os
from typing import Dict, Iterable, List, Optional, Sequence, Tuple

from . import Context, Matrix, Params

DEFAULT_CANDIDATES: Tuple[Tuple[int, int, int], ...] = (
    # (block_size, threads_per_source, src_chunk)
    (0, 1, 0), (1024, 1, 128), (1024, 1, 512), (512, 1, 0), (256, 1, 0), (1024, 8, 0),
)

_CACHE_ENV = "GSOFA_AUTOTUNE_CACHE"


def signature(mats: Sequence[Matrix]) -> str:
    """Workload key: log2 buckets of the largest n, of the total nnz, and of
    the matrix count."""
    nmax = max((m.n for m in mats), default=0)
    nnz = sum(m.nnz for m in mats)
    b = lambda x: int(math.log2(max(x, 1)))  # noqa: E731
    return f"n{b(nmax)}-nnz{b(nnz)}-k{b(len(mats))}"


def _cache_path(path: Optional[str]) -> str:
    if path:
        return path
    env = os.environ.get(_CACHE_ENV)
    if env:
        return env
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "gsofa_b200", "autotune.json")


def _load(path: str) -> Dict[str, dict]:
    try:
        with open(path) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(path: str, table: Dict[str, dict]) -> None:
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def _params(base: Params, block: int, lanes: int, chunk: int) -> Params:
    p = Params()
    ctypes_copy(p, base)
    p.block_size = block
    p.threads_per_source = lanes
    p.src_chunk = chunk
    return p


def ctypes_copy(dst: Params, src: Params) -> None:
    for name, _ in Params._fields_:
        setattr(dst, name, getattr(src, name))


def measure(ctx: Context, mats: Sequence[Matrix], params: Params, reps: int = 1) -> float:
    """Best kernel time (ms) of `reps` batched launches."""
    best = math.inf
    for _ in range(max(reps, 1)):
        rs = ctx.symbfact_batch(list(mats), params)
        best = min(best, rs[0].kernel_ms)
    return best


def autotune(ctx: Context, mats: Sequence[Matrix], base: Optional[Params] = None,
             candidates: Iterable[Tuple[int, int, int]] = DEFAULT_CANDIDATES, reps: int = 1,
             cache_path: Optional[str] = None, use_cache: bool = True) -> Tuple[Params, dict]:
    """Returns the fastest parameters for `mats` (timed as one batch) and a
    report {signature, choice, timings}."""
    base = base if base is not None else Params.default()
    key = signature(mats)
    path = _cache_path(cache_path)
    table = _load(path) if use_cache else {}
    if use_cache and key in table:
        c = table[key]["choice"]
        return _params(base, *c), {"signature": key, "choice": c, "cached": True}
    timings: List[dict] = []
    best, best_ms = None, math.inf
    for block, lanes, chunk in candidates:
        p = _params(base, block, lanes, chunk)
        ms = measure(ctx, mats, p, reps)
        timings.append({"block": block, "lanes": lanes, "chunk": chunk, "kernel_ms": ms})
        if ms < best_ms:
            best, best_ms = (block, lanes, chunk), ms
    report = {"signature": key, "choice": list(best), "timings": timings, "cached": False}
    if use_cache:
        table[key] = {"choice": list(best), "kernel_ms": best_ms}
        _store(path, table)
    return _params(base, *best), report
