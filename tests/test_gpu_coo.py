"""Device matrices from coordinate block lists and DBCSR dumps (through the C
ABI), against the oracle's restatement of the reference's single-rank
load path (lamb_load_dbcsr -> internal_distribute -> fill_local_sectors)."""
import numpy as np
import pytest

import oracle
from oracle import dbcsr as od
from lamb_b200.gpu import LambError

from test_dbcsr import water_dump

pytestmark = pytest.mark.gpu


def same_sectors(x, y):
    """Same sector index (bit-exact) and the same block values."""
    assert len(x.sectors) == len(y.sectors)
    for s, t in zip(x.sectors, y.sectors):
        assert (s.subset_row, s.subset_col) == (t.subset_row, t.subset_col)
        assert np.array_equal(s.row_blk_sizes, t.row_blk_sizes) and np.array_equal(s.col_blk_sizes, t.col_blk_sizes)
        assert np.array_equal(s.row_p, t.row_p) and np.array_equal(s.col_i, t.col_i)
        for b in range(s.n_blks):
            assert np.array_equal(s.block(b), t.block(b))


@pytest.mark.parametrize("n_chunks,n_x", [(1, 1), (3, 2), (5, 3)])
def test_load_dbcsr_matches_oracle(gpu_ctx, tmp_path, n_chunks, n_x):
    ctx = gpu_ctx
    p = str(tmp_path / "w.dbcsr")
    g, a = water_dump(p, n_mol=32, cutoff=5.5, n_chunks=n_chunks, seed=n_chunks)
    xyz = g.positions.astype(np.float32)
    d = ctx.load_dbcsr(p, xyz if n_x > 1 else None, n_x)
    coo = od.read_dbcsr(p)
    sub = od.x_subsets(xyz, g.n_atoms, n_x)
    want = od.coo_to_matrix(coo, sub, sub)
    same_sectors(d.download(), want)
    d.destroy()


def test_from_coo_sorts_shuffled_blocks_and_multiplies(gpu_ctx):
    ctx = gpu_ctx
    from lamb_b200.gen import WaterGeometry
    g = WaterGeometry(40, None, 5.0, seed=3)
    a, b = g.matrix(1), g.matrix(2)
    glob = {(int(g.subset[i]), int(g.local[i])): i for i in range(g.n_atoms)}
    rows, cols, ext, data = [], [], [], []
    pos = 1
    for s in a.sectors:
        br = s.block_rows()
        for k in range(s.n_blks):
            rows.append(glob[(s.subset_row, int(br[k]))] + 1)
            cols.append(glob[(s.subset_col, int(s.col_i[k]) - 1)] + 1)
            x = s.block(k).ravel(order="F")
            ext.append((pos, pos + x.size - 1))
            data.append(x)
            pos += x.size
    perm = np.random.default_rng(0).permutation(len(rows))
    rows, cols, ext = np.array(rows)[perm], np.array(cols)[perm], np.array(ext)[perm]
    da = ctx.from_coo(g.blk, g.blk, g.subset, g.subset, rows, cols, ext, np.concatenate(data))
    same_sectors(da.download(), a)
    # the loaded matrix multiplies like the uploaded one
    db = ctx.upload(b)
    dc = ctx.create_like(da)
    ctx.multiply(da, db, dc, 1e-8)
    ref, _ = oracle.multiply(a, b, 1e-8)
    c = dc.download()
    for s, t in zip(c.sectors, ref.sectors):
        assert np.array_equal(s.row_p, t.row_p) and np.array_equal(s.col_i, t.col_i)
    err = np.linalg.norm(c.to_dense() - ref.to_dense()) / np.linalg.norm(ref.to_dense())
    assert err <= 1e-12
    for m in (dc, db, da):
        m.destroy()


def test_from_coo_rejects_bad_input(gpu_ctx):
    ctx = gpu_ctx
    bs = np.array([2, 1], np.int8)
    sub = np.array([1, 1], np.int32)
    data = np.arange(1.0, 10.0)
    ok = dict(blk_row=[1, 2], blk_col=[2, 1], extents=[(1, 2), (3, 4)])
    d = ctx.from_coo(bs, bs, sub, sub, ok["blk_row"], ok["blk_col"], ok["extents"], data)
    assert d.download().to_dense().tolist() == [[0, 0, 1], [0, 0, 2], [3, 4, 0]]
    d.destroy()
    cases = [
        ([1, 1], [2, 2], [(1, 2), (3, 4)], "duplicate"),
        ([1, 3], [2, 1], [(1, 2), (3, 4)], "out of range"),
        ([1, 2], [2, 1], [(1, 3), (4, 5)], "extent"),
        ([1, 2], [2, 1], [(1, 2), (9, 10)], "extent"),
    ]
    for r, c, e, what in cases:
        with pytest.raises(LambError, match=what):
            ctx.from_coo(bs, bs, sub, sub, r, c, e, data)


def test_from_coo_empty(gpu_ctx):
    ctx = gpu_ctx
    bs = np.array([3, 4, 5], np.int8)
    sub = np.array([1, 2, 1], np.int32)
    d = ctx.from_coo(bs, bs, sub, sub, [], [], np.zeros((0, 2)), np.zeros(0))
    m = d.download()
    assert sum(s.n_blks for s in m.sectors) == 0 and len(m.sectors) == 4
    d.destroy()
