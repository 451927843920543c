"""Symbolic factorization of one matrix sharded over several GPUs.

Every source line is independent, so the lines are split over the ranks.
The reference interleaves them (rank r of W takes s = r, r + W, r + 2W, ...;
with_space_optimization/symbfact.cuh:1084-1099), which leaves no two
consecutive sources on one GPU, so no traversal can start from its
predecessor's state.  Here rank r takes the contiguous range
[cuts[r], cuts[r+1]) from gsofa_partition_lines -- cut on equal shares of the
work predicted from the symmetric structure, at lines that start a chain --
and keeps reuse.  Each rank factorizes its range on its own GPU, which fills
only its own lines of the per-line arrays; one sum-all-reduce of the per-line
arrays and of the fill count assembles the full answer on every rank, and the
supernode scan then runs on the host over the summed lines.  The only
exchange is that all-reduce (n int32 + n int32 + n int32 flags + one int64
per rank).  The interleaved split stays available (interleave=True).
"""
from __future__ import annotations

import ctypes
from typing import Callable, Dict, Optional

import numpy as np

from . import Context, Matrix, Params, partition_lines, supernodes_from_lines
from .matgen import Graph

AllReduce = Callable[[np.ndarray], np.ndarray]


def torch_allreduce(group=None) -> AllReduce:
    """Sum-all-reduce over a torch.distributed process group (gloo on CPU
    tensors, NCCL on CUDA tensors)."""
    import torch
    import torch.distributed as dist

    def fn(x: np.ndarray) -> np.ndarray:
        backend = dist.get_backend(group)
        t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.int64))
        if backend == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return t.cpu().numpy()

    return fn


def combine(n: int, u_row_count: np.ndarray, l_col_count: np.ndarray, line_flags: np.ndarray,
            fill_count: int, allreduce: AllReduce, max_supernode_size: int = 0) -> Dict:
    """Sums one rank's partition arrays with every other rank's and finishes
    the factorization (totals and supernodes) on the host."""
    packed = np.concatenate([np.asarray(u_row_count, np.int64), np.asarray(l_col_count, np.int64),
                             np.asarray(line_flags, np.int64), np.array([fill_count], np.int64)])
    tot = allreduce(packed)
    u = tot[:n].astype(np.int32)
    lc = tot[n:2 * n].astype(np.int32)
    fl = tot[2 * n:3 * n].astype(np.uint8)
    fills = int(tot[3 * n])
    sn = supernodes_from_lines(u, fl, max_supernode_size)
    return {"n": n, "fill_count": fills, "nnz_lu": int(u.sum(dtype=np.int64) + lc.sum(dtype=np.int64) + n),
            "u_row_count": u, "l_col_count": lc, "line_flags": fl, "sn_start": sn}


def rank_params(rank: int, world: int, cuts: Optional[np.ndarray], params: Optional[Params] = None,
                max_supernode_size: int = 0, interleave: bool = False) -> Params:
    """The library parameters of one rank's share: its line range (or its
    interleaved partition), counts only."""
    if params is not None:
        p = Params()
        ctypes.pointer(p)[0] = params     # a copy: the caller's stays as it is
    else:
        p = Params.default()
    p.want_pattern = 0
    p.max_supernode_size = max_supernode_size
    if interleave:
        p.part_count, p.part_index = world, rank
        p.line_lo = p.line_hi = 0
    else:
        p.part_count, p.part_index = 1, 0
        lo, hi = int(cuts[rank]), int(cuts[rank + 1])
        if lo == hi:      # an empty share: [n, n) (the library reads 0, 0 as all lines)
            lo = hi = int(cuts[-1])
        p.line_lo, p.line_hi = lo, hi
    return p


def symbfact_sharded(ctx: Optional[Context], m: Optional[Matrix], rank: int, world: int, allreduce: AllReduce,
                     max_supernode_size: int = 0, params: Params = None, graph: Optional[Graph] = None,
                     cuts: Optional[np.ndarray] = None, interleave: bool = False,
                     factorize: Optional[Callable] = None) -> Dict:
    """This rank's share of the factorization of one matrix, combined across
    ranks.  The line ranges come from `cuts` or, given the host `graph`, from
    partition_lines (every rank computes the same cuts).  `factorize(p)` runs
    the share with parameters p and returns an object with u_row_count,
    l_col_count, line_flags, fill_count and kernel_ms (default:
    ctx.symbfact(m, p) on this rank's GPU)."""
    if not interleave and cuts is None:
        if graph is None:
            raise ValueError("range partitions need the host graph or the cuts")
        cuts, _ = partition_lines(graph, world)
    p = rank_params(rank, world, cuts, params, max_supernode_size, interleave)
    run = factorize if factorize is not None else (lambda pp: ctx.symbfact(m, pp))
    r = run(p)
    n = len(r.u_row_count)
    out = combine(n, r.u_row_count, r.l_col_count, r.line_flags, r.fill_count, allreduce, max_supernode_size)
    out["kernel_ms"] = r.kernel_ms
    out["cuts"] = None if cuts is None else np.asarray(cuts)
    return out
