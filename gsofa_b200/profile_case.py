"""Small cases for a profiler: every kernel family of the library once.

``python -m gsofa_b200.profile_case factor [side]`` factorizes the side^3
nested-dissection stencil (default 48: n = 110,592, about 45 MB of pattern)
into a device pool in the ranges form twice, then once each counts only,
unpaired with adjacency reuse, with global-memory state and with the
supernodal structure.  ``python -m gsofa_b200.profile_case serve`` serves one
request through the persistent serving kernel with a 2 ms idle exit, so a
replaying profiler never waits on an idle kernel.  ``python -m
gsofa_b200.profile_case order`` orders a shuffled 50,000-line power-law
pattern by reverse Cuthill-McKee on the GPU.
"""
import sys
import time

import torch

import gsofa_b200
from gsofa_b200 import matgen


def factor(side: int = 48) -> None:
    g = matgen.config_nd3d(side)
    nd = gsofa_b200.FLAG_NO_DOWNLOAD
    with gsofa_b200.Context(0) as ctx:
        m = ctx.upload(g)
        need = ctx.symbfact(m, want_pattern=0, flags=nd)
        pool = torch.empty(need.nnz_u + need.nnz_l, dtype=torch.int32, device="cuda")
        for _ in range(2):
            ctx.symbfact_ranges(m, pool, gsofa_b200.Params.default(flags=nd))
        ctx.symbfact(m, want_pattern=0, flags=nd)
        ctx.symbfact(m, want_pattern=0, reuse=2, flags=nd)
        ctx.symbfact(m, want_pattern=0, flags=nd | gsofa_b200.FLAG_GLOBAL_STATE)
        ctx.symbfact_supernodal(m)


def serve(side: int = 48) -> None:
    g = matgen.config_nd3d(side)
    srv = gsofa_b200.StreamServer(0, mem_budget_bytes=8 << 30, max_n=200000, idle_exit_us=2000)
    try:
        rid = srv.submit(g)
        t0 = time.time()
        while not srv.poll():
            if time.time() - t0 > 60:
                raise RuntimeError("serving kernel did not finish the request within 60 s")
        srv.result(rid)
        srv.drain()
    finally:
        srv.close()


def order(side: int = 48) -> None:
    g = matgen.powerlaw(50_000, seed=7, ordering="random")
    with gsofa_b200.Context(0) as ctx:
        ctx.order_rcm(g)


if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "factor"
    side = int(sys.argv[2]) if len(sys.argv) > 2 else 48
    {"factor": factor, "serve": serve, "order": order}[which](side)
    print("ok", which)
