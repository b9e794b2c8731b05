"""Comparison helpers shared by the tests."""
import numpy as np

from lamb_b200.matrix import LambMatrix


def block_values(m: LambMatrix):
    """{(subset_row, subset_col, row, col): block (rows, cols)} for every block."""
    out = {}
    for s in m.sectors:
        rows = s.block_rows()
        for b in range(s.n_blks):
            r, c = int(rows[b]), int(s.col_i[b]) - 1
            mm, nn = int(s.row_blk_sizes[r]), int(s.col_blk_sizes[c])
            f = int(s.extents[b, 0])
            out[(s.subset_row, s.subset_col, r, c)] = s.data[f - 1:f - 1 + mm * nn].reshape(nn, mm).T
    return out


def assert_same_pattern(got: LambMatrix, ref: LambMatrix):
    assert len(got.sectors) == len(ref.sectors)
    for g, r in zip(got.sectors, ref.sectors):
        assert (g.subset_row, g.subset_col) == (r.subset_row, r.subset_col)
        assert np.array_equal(g.row_blk_sizes, r.row_blk_sizes)
        assert np.array_equal(g.col_blk_sizes, r.col_blk_sizes)
        assert np.array_equal(g.row_p, r.row_p), "row_p differs"
        assert np.array_equal(g.col_i, r.col_i), "col_i differs"


def rel_frobenius_error(got: LambMatrix, ref: LambMatrix) -> float:
    """|got - ref|_F / |ref|_F over the union of the block patterns."""
    gv, rv = block_values(got), block_values(ref)
    num = 0.0
    den = 0.0
    for k in set(gv) | set(rv):
        g = gv.get(k)
        r = rv.get(k)
        if r is None:
            num += float(np.sum(g ** 2))
        elif g is None:
            num += float(np.sum(r ** 2))
            den += float(np.sum(r ** 2))
        else:
            num += float(np.sum((g - r) ** 2))
            den += float(np.sum(r ** 2))
    return float(np.sqrt(num) / np.sqrt(den)) if den > 0 else float(np.sqrt(num))
