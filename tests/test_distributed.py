"""The sharded (multi-GPU) path on CPU: two or three gloo ranks each compute their
interleaved source partition (with the oracle standing in for the rank's
GPU, exactly as the kernel fills only its own lines), then combine through
the library's all-reduce assembly and host supernode scan."""
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


def _partition_arrays(g, rank, world):
    """What the kernel returns for one interleaved partition (counts mode)."""
    src = np.arange(rank, g.n, world, dtype=np.int32)
    c0, o0, x0, _ = oracle.counts(g.beg, g.end, g.adj, 0, nthreads=1, sources=src)
    c1, o1, x1, _ = oracle.counts(g.beg, g.end, g.adj, 1, nthreads=1, sources=src)
    u = np.zeros(g.n, np.int32); u[src] = c0[src]
    lc = np.zeros(g.n, np.int32); lc[src] = c1[src]
    fl = np.zeros(g.n, np.uint8); fl[src] = x0[src] | (x1[src] << 1)
    fills = int(c0[src].sum() - o0[src].sum() + c1[src].sum() - o1[src].sum())
    return u, lc, fl, fills


def _worker(rank, world, port, kind, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = bundled() if kind == "bundled" else matgen.grid3d(12, ordering="nd", drop_frac=0.1, seed=9)
        u, lc, fl, fills = _partition_arrays(g, rank, world)
        out = distributed.combine(g.n, u, lc, fl, fills, distributed.torch_allreduce(), 8)
        q.put((rank, out["fill_count"], out["nnz_lu"], out["u_row_count"].tolist(),
               out["l_col_count"].tolist(), out["sn_start"].tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind,world", [("bundled", 2), ("grid3d", 2), ("grid3d", 3)])
def test_gloo_ranks_assemble_the_full_factorization(kind, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, kind, q)) for r in range(world)]
    for p in procs:
        p.start()
    outs = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = bundled() if kind == "bundled" else matgen.grid3d(12, ordering="nd", drop_frac=0.1, seed=9)
    ref = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False, max_supernode_size=8)
    for rank, fills, nnz, u, lc, sn in outs:
        assert fills == ref["fill_count"] and nnz == ref["nnz_lu"], rank
        assert np.array_equal(np.array(u), ref["u_row_count"])
        assert np.array_equal(np.array(lc), ref["l_col_count"])
        assert np.array_equal(np.array(sn), ref["sn_start"])


def test_host_supernode_scan_matches_oracle():
    for g in (bundled(), matgen.powerlaw(3000, seed=2), matgen.grid2d(40)):
        ref = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False, max_supernode_size=5)
        flags = (ref["u_next"] | (ref["l_next"] << 1)).astype(np.uint8)
        for ms in (0, 5):
            want = oracle.supernodes(ref["u_row_count"], ref["u_next"], ref["l_next"], ms)
            assert np.array_equal(supernodes_from_lines(ref["u_row_count"], flags, ms), want)
