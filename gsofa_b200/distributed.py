"""Symbolic factorization of one matrix sharded over several GPUs.

Every source line is independent, so the sources are split in the
reference's interleaved way (rank r of W takes s = r, r + W, r + 2W, ...;
with_space_optimization/symbfact.cuh:1093).  Each rank runs the partition on
its own GPU (counts mode), which fills only its own lines of the per-line
arrays; one sum-all-reduce of the per-line arrays and of the fill count
assembles the full answer on every rank, and the supernode scan then runs on
the host over the summed lines.  The only exchange is that all-reduce
(n int32 + n int32 + n int32 flags + one int64 per rank).
"""
from __future__ import annotations

from typing import Callable, Dict

import numpy as np

from . import Context, Matrix, Params, supernodes_from_lines

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


def symbfact_sharded(ctx: Context, m: Matrix, rank: int, world: int, allreduce: AllReduce,
                     max_supernode_size: int = 0, params: Params = None) -> Dict:
    """This rank's share of the factorization of `m`, combined across ranks."""
    p = params if params is not None else Params.default()
    p.want_pattern = 0
    p.part_count = world
    p.part_index = rank
    p.max_supernode_size = max_supernode_size
    r = ctx.symbfact(m, p)
    out = combine(m.n, r.u_row_count, r.l_col_count, r.line_flags, r.fill_count, allreduce,
                  max_supernode_size)
    out["kernel_ms"] = r.kernel_ms
    return out
