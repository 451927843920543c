"""Writes tests/golden/large.json: the full oracle result of the two large
headline matrices, as totals and SHA-256 digests of the per-line arrays.

    python tests/golden/make_large_golden.py [nd3d] [circuit]

* nd3d    -- 80^3 7-point stencil, geometric nested dissection, seeded 10%
             one-sided drops (n = 512,000); the pattern is materialised by the
             GPU library, the digests pin its per-line counts and supernodes.
* circuit -- the power-law circuit-like matrix (n = 659,033, random
             permutation + RCM), counts only (its pattern holds ~1.2e11
             entries).

Each entry is the CPU oracle (oracle/gsofa_oracle.c, both reachability
passes over every source, OpenMP) run in full; the GPU tests compare the
library's arrays with these digests.  The circuit matrix takes about an hour
on eight host cores.
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from gsofa_b200 import matgen  # noqa: E402

OUT = os.path.join(HERE, "large.json")


def digest(a, dtype) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()).hexdigest()


def entry(g, seed, how):
    t0 = time.time()
    ucnt, uorig, unext, work = oracle.counts(g.beg, g.end, g.adj, 0)
    lcnt, lorig, lnext, _ = oracle.counts(g.beg, g.end, g.adj, 1)
    sn = oracle.supernodes(ucnt, unext, lnext, 0)
    flags = (unext.astype(np.uint8) | (lnext.astype(np.uint8) << 1)).astype(np.uint8)
    nnz_u = int(ucnt.sum(dtype=np.int64))
    nnz_l = int(lcnt.sum(dtype=np.int64))
    return {
        "n": int(g.n), "nnz": int(g.nnz), "seed": seed, "generator": how,
        "fill_count": nnz_u + nnz_l - int(uorig.sum(dtype=np.int64)) - int(lorig.sum(dtype=np.int64)),
        "nnz_lu": nnz_u + nnz_l + int(g.n), "nnz_u": nnz_u, "nnz_l": nnz_l,
        "n_supernodes": int(sn.shape[0]), "x_total": int(work[0]), "e_insp": int(work[1]),
        "sha256": {"u_row_count": digest(ucnt, "<i4"), "l_col_count": digest(lcnt, "<i4"),
                   "line_flags": digest(flags, "u1"), "sn_start": digest(sn, "<i4")},
        "oracle_seconds": round(time.time() - t0, 1),
    }


def main(which):
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    if "nd3d" in which:
        data["grid3d_80^3_7pt_nd_drop0.1"] = entry(matgen.config_nd3d(80), matgen.SEEDS["nd3d"],
                                                   "matgen.config_nd3d(80)")
        _save(data)
    if "circuit" in which:
        data["powerlaw_659033_rcm"] = entry(matgen.config_circuit(), matgen.SEEDS["circuit"],
                                            "matgen.config_circuit()")
        _save(data)


def _save(data):
    with open(OUT, "w") as f:
        json.dump(data, f, indent=2, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1:] or ["nd3d", "circuit"])
