"""The factorization entry point that allocates no device memory.

gsofa_symbfact_counts_noalloc serves callers that cannot call cudaMalloc:
code embedded under a host application's own device allocator or memory
budget, and code on paths where cudaMalloc's implicit device-wide
synchronisation is not allowed.  Its scratch is a static device array inside
the library, shared by every call on a device.  These tests call it through
the C ABI with caller-owned device buffers and compare every output with the
regular entry point (gsofa_symbfact, counts only), on calls made back to back
so that leftovers of one call in the shared scratch would show up in the
next.  This file is collected last on purpose."""
import numpy as np
import pytest

import gsofa_b200
import oracle
from gsofa_b200 import matgen
from tests.common import bundled, random_graph

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _noalloc(g, max_sn):
    dev = torch.device("cuda", 0)
    beg = torch.from_numpy(g.beg).to(dev)
    end = torch.from_numpy(g.end).to(dev)
    adj = torch.from_numpy(g.adj if g.nnz else np.zeros(1, np.int32)).to(dev)
    u = torch.full((max(g.n, 1),), -1, dtype=torch.int32, device=dev)
    lc = torch.full((max(g.n, 1),), -1, dtype=torch.int32, device=dev)
    sn = torch.full((max(g.n, 1),), -1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    fills, nnz_lu, nsn = gsofa_b200.symbfact_counts_noalloc(
        0, stream.cuda_stream, g.n, g.nnz, beg.data_ptr(), end.data_ptr(), adj.data_ptr(),
        u.data_ptr(), lc.data_ptr(), sn.data_ptr(), max_sn)
    return fills, nnz_lu, u.cpu().numpy()[:g.n], lc.cpu().numpy()[:g.n], sn.cpu().numpy()[:nsn]


def _regular(ctx, g, max_sn):
    r = ctx.symbfact(ctx.upload(g), want_pattern=0, max_supernode_size=max_sn)
    return r.fill_count, r.nnz_lu, r.u_row_count, r.l_col_count, r.sn_start


def _same(a, b, where):
    assert a[0] == b[0], f"{where}: fill count {a[0]} != {b[0]}"
    assert a[1] == b[1], f"{where}: nnz(L+U) {a[1]} != {b[1]}"
    for k, name in ((2, "u_row_count"), (3, "l_col_count"), (4, "sn_start")):
        assert np.array_equal(a[k], b[k]), f"{where}: {name} differs"


def _oracle(g, max_sn):
    r = oracle.symbfact(g.beg, g.end, g.adj, want_pattern=False, max_supernode_size=max_sn)
    return r["fill_count"], r["nnz_lu"], r["u_row_count"], r["l_col_count"], r["sn_start"]


def banded_at_limits(seed=0):
    """n and the total range length at the entry point's limits: 16 entries
    per line (the diagonal and 15 seeded ids within +/-128 of it)."""
    n = gsofa_b200.NOALLOC_MAX_N
    per = gsofa_b200.NOALLOC_MAX_NNZ // n
    rng = np.random.default_rng(seed)
    rows = np.arange(n, dtype=np.int64)
    cols = rows[:, None] + rng.integers(-128, 129, size=(n, per))
    cols[:, 0] = rows
    cols = np.clip(cols, 0, n - 1).astype(np.int32)
    beg = (rows * per).astype(np.int32)
    return matgen.Graph(n, beg, beg + per, cols.reshape(-1), "banded_at_noalloc_limits")


def test_noalloc_matches_regular_entry_on_consecutive_calls():
    mats = [(bundled(), 0), (matgen.grid3d(16, ordering="nd", drop_frac=0.1, seed=4), 8),
            (random_graph(700, 0.01, 21), 0), (bundled(), 4), (banded_at_limits(), 0)]
    assert mats[-1][0].nnz == gsofa_b200.NOALLOC_MAX_NNZ
    with gsofa_b200.Context(0) as ctx:
        for i, (g, max_sn) in enumerate(mats):
            got = _noalloc(g, max_sn)
            _same(got, _regular(ctx, g, max_sn), f"call {i} ({g.name}) vs gsofa_symbfact")
            _same(got, _oracle(g, max_sn), f"call {i} ({g.name}) vs the oracle")


def test_noalloc_allocates_nothing_and_keeps_the_current_device():
    """Device memory free before and after a call is the same (the first call
    on a device may load the library's device code, which brings the static
    array with it, so it runs first), and the caller's current device is
    unchanged."""
    g = banded_at_limits(1)
    _noalloc(g, 0)
    dev = torch.device("cuda", 0)
    beg = torch.from_numpy(g.beg).to(dev)
    end = torch.from_numpy(g.end).to(dev)
    adj = torch.from_numpy(g.adj).to(dev)
    outs = [torch.empty(g.n, dtype=torch.int32, device=dev) for _ in range(3)]
    torch.cuda.synchronize()
    cur = torch.cuda.current_device()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(2):
        gsofa_b200.symbfact_counts_noalloc(0, torch.cuda.current_stream(dev).cuda_stream, g.n, g.nnz,
                                           beg.data_ptr(), end.data_ptr(), adj.data_ptr(),
                                           outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr())
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    assert torch.cuda.current_device() == cur


def test_noalloc_rejects_oversized_inputs():
    n = gsofa_b200.NOALLOC_MAX_N + 1
    with pytest.raises(gsofa_b200.GsofaError) as e:
        gsofa_b200.symbfact_counts_noalloc(0, 0, n, 10, 1, 1, 1, 1, 1, 1)
    assert e.value.status == 7
    with pytest.raises(gsofa_b200.GsofaError) as e:
        gsofa_b200.symbfact_counts_noalloc(0, 0, 100, gsofa_b200.NOALLOC_MAX_NNZ + 1, 1, 1, 1, 1, 1, 1)
    assert e.value.status == 7
