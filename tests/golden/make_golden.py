"""Regenerates the golden fixtures under tests/golden/ (run in a container that
holds the reference checkout; the GPU box only reads the committed files).

    python tests/golden/make_golden.py /path/to/reference

* bundled_11948.npz -- the reference's bundled SuperLU_DIST dump (n = 11,948,
  nnz = 149,090; with_space_optimization/dataset/{colbeg,colend,csr}_11948.dat),
  converted losslessly from text to int32 arrays.
* expected.json     -- the values the fixtures must reproduce and where each
  one is pinned.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_ints(path):
    with open(path) as f:
        return np.array(f.read().split(), dtype=np.int64)


def main(ref_root):
    d = os.path.join(ref_root, "with_space_optimization", "dataset")
    csr = read_ints(os.path.join(d, "csr_11948.dat"))
    nnz, n = int(csr[0]), int(csr[1])
    adj = csr[2:2 + nnz].astype(np.int32)
    beg = read_ints(os.path.join(d, "colbeg_11948.dat"))[:n].astype(np.int32)
    end = read_ints(os.path.join(d, "colend_11948.dat"))[:n].astype(np.int32)
    assert adj.shape[0] == nnz and beg.shape[0] == n and end.shape[0] == n
    np.savez_compressed(os.path.join(HERE, "bundled_11948.npz"), beg=beg, end=end, adj=adj,
                        n=np.int64(n), nnz=np.int64(nnz))
    expected = {
        "bundled_11948": {
            "n": n, "nnz": nnz, "fill_count": 980136, "fill_lower": 490068, "fill_upper": 490068,
            "nnz_lu": 1129226,
            "pinned_by": "reference run log with_space_optimization/"
                          "space_optimization_log_1_264_GPU_warp_centric.dat:2 (fill total)",
        },
        "grid2d_64x64_natural": {
            "n": 4096, "nnz": 20224, "fill_count": 500094, "nnz_lu": 520318,
            "pinned_by": "analytic band count of a 64x64 5-point grid in natural order",
        },
    }
    with open(os.path.join(HERE, "expected.json"), "w") as f:
        json.dump(expected, f, indent=2)
        f.write("\n")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GSOFA_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <reference checkout>  (or set GSOFA_REFERENCE_ROOT)")
    main(root)
