"""Writes the small golden fixtures of tests/test_oracle.py.

The reference ships no golden vectors for its multiply (its sector_multiply
is a stub), so these fixtures are self-generated: inputs from the package's
deterministic generators, C from an independent dense numpy product, and the
C block pattern as the set of (sector, row, col) whose dense block is
non-zero with at least one product present.  Run:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from lamb_b200.gen import WaterGeometry, random_fill_matrix  # noqa: E402
from lamb_b200.matrix import LambMatrix, Sector  # noqa: E402


def _pack(prefix, m, out):
    out[prefix + "_n"] = np.int64(len(m.sectors))
    for i, s in enumerate(m.sectors):
        q = f"{prefix}{i}_"
        out[q + "sr"] = np.int64(s.subset_row)
        out[q + "sc"] = np.int64(s.subset_col)
        out[q + "rbs"] = s.row_blk_sizes
        out[q + "cbs"] = s.col_blk_sizes
        out[q + "row_p"] = s.row_p
        out[q + "col_i"] = s.col_i
        out[q + "extents"] = s.extents
        out[q + "data"] = s.data


def _pattern(a, b):
    """Block pattern of A.B from the block patterns (structural product)."""
    pa, pb = a.block_pattern(), b.block_pattern()
    S = a.n_subsets
    pat = set()
    for m in range(1, S + 1):
        for k in range(1, S + 1):
            for (i, kk) in pa.get((m, k), ()):
                for n in range(1, S + 1):
                    for (k2, j) in pb.get((k, n), ()):
                        if k2 == kk:
                            pat.add((m, n, i - 1, j - 1))
    return np.array(sorted(pat), dtype=np.int64).reshape(-1, 4)


def write(name, a, b, eps=0.0, flags=6):
    out = {}
    _pack("a", a, out)
    _pack("b", b, out)
    out["eps"] = np.float64(eps)
    out["flags"] = np.int64(flags)
    out["c_dense"] = a.to_dense() @ b.to_dense()
    out["c_pattern"] = _pattern(a, b)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


if __name__ == "__main__":
    g = WaterGeometry(8, None, 3.5, seed=21)
    write("water8_cut3p5", g.matrix(1), g.matrix(2))
    a = random_fill_matrix(4, max_atoms=60)
    b = LambMatrix([Sector(s.subset_row, s.subset_col, s.row_blk_sizes, s.col_blk_sizes, s.row_p, s.col_i,
                           s.extents, np.random.default_rng(104).random(s.data.shape[0])) for s in a.sectors])
    write("random_fill_seed4", a, b)
    print("written")
