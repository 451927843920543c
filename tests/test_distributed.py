"""The sharded (multi-GPU) path on CPU: two or three gloo ranks each run
distributed.symbfact_sharded on their share -- a contiguous range from the
work-predicted partitioner, or the reference's interleaved partition -- with
the oracle standing in for the rank's GPU (it fills only the share's lines,
exactly as the kernel does), then combine through the library's all-reduce
assembly and host supernode scan."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from gsofa_b200 import distributed, matgen, supernodes_from_lines
from tests.common import bundled


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class _Share:
    """The per-line arrays one rank's GPU returns for its share."""

    def __init__(self, u, lc, fl, fills):
        self.u_row_count, self.l_col_count, self.line_flags, self.fill_count = u, lc, fl, fills
        self.kernel_ms = 0.0


def _oracle_share(g):
    """factorize(p) for symbfact_sharded: the oracle over the lines p names."""
    def run(p):
        if p.line_hi > p.line_lo:
            src = np.arange(p.line_lo, p.line_hi, dtype=np.int32)
        else:
            src = np.arange(p.part_index, g.n, p.part_count, dtype=np.int32)
        return _Share(*_partition_arrays(g, src))
    return run


def _partition_arrays(g, src):
    """What the kernel returns for the sources src (counts mode)."""
    c0, o0, x0, _ = oracle.counts(g.beg, g.end, g.adj, 0, nthreads=1, sources=src)
    c1, o1, x1, _ = oracle.counts(g.beg, g.end, g.adj, 1, nthreads=1, sources=src)
    u = np.zeros(g.n, np.int32); u[src] = c0[src]
    lc = np.zeros(g.n, np.int32); lc[src] = c1[src]
    fl = np.zeros(g.n, np.uint8); fl[src] = x0[src] | (x1[src] << 1)
    fills = int(c0[src].sum() - o0[src].sum() + c1[src].sum() - o1[src].sum())
    return u, lc, fl, fills


def _graph(kind):
    return bundled() if kind == "bundled" else matgen.grid3d(12, ordering="nd", drop_frac=0.1, seed=9)


def _worker(rank, world, port, kind, interleave, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = _graph(kind)
        out = distributed.symbfact_sharded(None, None, rank, world, distributed.torch_allreduce(), 8,
                                           graph=g, interleave=interleave, factorize=_oracle_share(g))
        cuts = None if out["cuts"] is None else out["cuts"].tolist()
        q.put((rank, out["fill_count"], out["nnz_lu"], out["u_row_count"].tolist(),
               out["l_col_count"].tolist(), out["sn_start"].tolist(), cuts))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind,world,interleave", [("bundled", 2, False), ("grid3d", 2, False),
                                                   ("grid3d", 3, False), ("bundled", 3, True)])
def test_gloo_ranks_assemble_the_full_factorization(kind, world, interleave):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, kind, interleave, q)) for r in range(world)]
    for p in procs:
        p.start()
    outs = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = _graph(kind)
    ref = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False, max_supernode_size=8)
    for rank, fills, nnz, u, lc, sn, cuts in outs:
        assert fills == ref["fill_count"] and nnz == ref["nnz_lu"], rank
        assert np.array_equal(np.array(u), ref["u_row_count"])
        assert np.array_equal(np.array(lc), ref["l_col_count"])
        assert np.array_equal(np.array(sn), ref["sn_start"])
        if not interleave:   # every rank computed the same ranges
            assert cuts == outs[0][-1] and cuts[0] == 0 and cuts[-1] == g.n


def test_partitioner_balances_predicted_work_and_counts_are_bounds():
    """The predicted list lengths are exact on symmetric patterns and upper
    bounds otherwise; the ranges split the predicted work evenly."""
    for g, symmetric in ((matgen.grid2d(30), True), (matgen.grid3d(12, ordering="nd", drop_frac=0.0, seed=1), True),
                         (bundled(), True), (matgen.grid3d(12, ordering="nd", drop_frac=0.1, seed=1), False),
                         (matgen.powerlaw(2000, seed=3), False)):
        from gsofa_b200 import predict_line_counts, partition_lines
        pc = predict_line_counts(g)
        ref = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False)
        assert np.all(pc >= ref["u_row_count"]) and np.all(pc >= ref["l_col_count"]), g.name
        if symmetric:
            assert np.array_equal(pc, ref["u_row_count"]) and np.array_equal(pc, ref["l_col_count"]), g.name
        _, whole = partition_lines(g, 1)
        for parts in (1, 2, 4, 7):
            cuts, work = partition_lines(g, parts)
            assert cuts[0] == 0 and cuts[-1] == g.n and np.all(np.diff(cuts) > 0)
            # the parts split the same predicted total
            assert abs(work.sum() - whole[0]) <= 1e-9 * whole[0]
            # the work model grows with the predicted list lengths: the last
            # lines (separators, longest lists) cost the most per line
            per_line = work / np.diff(cuts)
            assert per_line[-1] >= per_line[0] or parts == 1, (g.name, parts, per_line)


def test_host_supernode_scan_matches_oracle():
    for g in (bundled(), matgen.powerlaw(3000, seed=2), matgen.grid2d(40)):
        ref = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False, max_supernode_size=5)
        flags = (ref["u_next"] | (ref["l_next"] << 1)).astype(np.uint8)
        for ms in (0, 5):
            want = oracle.supernodes(ref["u_row_count"], ref["u_next"], ref["l_next"], ms)
            assert np.array_equal(supernodes_from_lines(ref["u_row_count"], flags, ms), want)


def test_partition_cuts_are_monotone_for_any_part_count():
    import gsofa_b200
    from tests.common import random_graph
    for g in (matgen.grid2d(10), random_graph(40, 0.05, 3)):
        for parts in (1, 3, g.n, g.n + 5):
            cuts, work = gsofa_b200.partition_lines(g, parts)
            assert cuts[0] == 0 and cuts[-1] == g.n and len(cuts) == parts + 1
            assert np.all(np.diff(cuts) >= 0)
            if parts <= g.n:
                assert np.all(np.diff(cuts) >= 1)    # no empty part while lines remain for each
            assert np.all(work >= 0)
