"""DBCSR dump reader (host side of lamb_gpu_matrix_load_dbcsr) against the
oracle restatement of lamb_load_dbcsr (src/lamb_io_operations.F90:267-756).

The reference's own fixture (small.dbcsr) is not in its tree, so the oracle
reader is pinned here on a file written field by field from the format
description (src/lamb_io_operations.F90:300-330), then the library's reader
is compared with the oracle on multi-chunk dumps of water matrices.
"""
import struct

import numpy as np
import pytest

from oracle import dbcsr as od
from lamb_b200 import gpu
from lamb_b200.gen import WaterGeometry


def _hand_written(path):
    """2 x 3 block rows/columns, sizes (2, 1) x (1, 2, 1); two chunks.
    chunk 1: blocks (1,2) and (2,1); chunk 2: block (1,3).  blk_p 1-based."""
    rbs, cbs = [2, 1], [1, 2, 1]
    with open(path, "wb") as f:
        f.write(b"DBCSR-1.0 ")
        f.write(b"hand".ljust(80))
        f.write(b"N")
        f.write(struct.pack("<4i", 2, 3, 2, 3))
        f.write(struct.pack("<2i", *rbs))
        f.write(struct.pack("<3i", *cbs))
        f.write(struct.pack("<2i", 2, 5))     # chunk 1: 2 blocks, data area 5 (+1 unused)
        f.write(struct.pack("<2i", 1, 2))     # chunk 2: 1 block, area 2
        f.write(struct.pack("<3i", 0, 1, 2))  # chunk 1 row_p
        f.write(struct.pack("<2i", 2, 1))     # col_i
        f.write(struct.pack("<2i", 2, 1))     # blk_p: (1,2) at 2..5 (2x2), (2,1) at 1..1 (1x1)
        f.write(struct.pack("<3i", 0, 1, 1))  # chunk 2 row_p
        f.write(struct.pack("<1i", 3))
        f.write(struct.pack("<1i", 1))        # (1,3) at 1..2 (2x1)
        f.write(struct.pack("<5d", 7.0, 1.0, 2.0, 3.0, 4.0))
        f.write(struct.pack("<2d", 5.0, 6.0))


def test_oracle_reader_pinned_on_hand_written_file(tmp_path):
    p = str(tmp_path / "hand.dbcsr")
    _hand_written(p)
    coo = od.read_dbcsr(p)
    assert coo.name == "hand" and coo.matrix_type == "N" and coo.data_type == 3
    assert coo.rows.tolist() == [1, 2, 1] and coo.cols.tolist() == [2, 1, 3]
    assert coo.extents.tolist() == [[2, 5], [1, 1], [1, 2]]
    assert coo.store.tolist() == [0, 0, 1]
    m = od.coo_to_matrix(coo, np.ones(2, np.int32), np.ones(3, np.int32))
    dense = m.to_dense()
    want = np.array([[0, 1, 3, 5], [0, 2, 4, 6], [7, 0, 0, 0]], float)
    assert np.array_equal(dense, want)


def test_library_reader_matches_oracle_on_hand_written_file(tmp_path):
    p = str(tmp_path / "hand.dbcsr")
    _hand_written(p)
    r = gpu.dbcsr_read(p)
    assert r["info"]["n_chunks"] == 2 and r["info"]["n_blks"] == 3 and r["info"]["data_len"] == 7
    assert r["rows"].tolist() == [1, 2, 1] and r["cols"].tolist() == [2, 1, 3]
    # chunk 2's store follows chunk 1's 5 doubles
    assert r["extents"].tolist() == [[2, 5], [1, 1], [6, 7]]
    assert r["data"].tolist() == [7.0, 1.0, 2.0, 3.0, 4.0, 5.0, 6.0]


def water_dump(path, n_mol=24, cutoff=5.0, n_chunks=3, seed=0):
    g = WaterGeometry(n_mol, None, cutoff, seed=seed)
    a = g.matrix(seed + 1)
    glob = {(int(g.subset[i]), int(g.local[i])): i for i in range(g.n_atoms)}
    blocks = {}
    for s in a.sectors:
        rows = s.block_rows()
        for b in range(s.n_blks):
            blocks[(glob[(s.subset_row, int(rows[b]))], glob[(s.subset_col, int(s.col_i[b]) - 1)])] = s.block(b)
    od.write_dbcsr(path, "water", g.blk, g.blk, od.chunks_from_dense_blocks(g.n_atoms, blocks, g.blk, g.blk,
                                                                            n_chunks, seed=seed))
    return g, a


@pytest.mark.parametrize("n_chunks", [1, 3, 7])
def test_library_reader_matches_oracle(tmp_path, n_chunks):
    p = str(tmp_path / "w.dbcsr")
    g, a = water_dump(p, n_chunks=n_chunks, seed=n_chunks)
    coo = od.read_dbcsr(p)
    r = gpu.dbcsr_read(p)
    assert r["info"]["n_chunks"] == n_chunks and r["info"]["n_blks"] == coo.rows.size
    assert np.array_equal(r["rows"], coo.rows) and np.array_equal(r["cols"], coo.cols)
    base = np.cumsum([0] + [x.size for x in coo.stores])
    assert np.array_equal(r["extents"], coo.extents + base[coo.store][:, None])
    assert np.array_equal(r["data"], np.concatenate(coo.stores))
    # the oracle's sectors reproduce the generator's matrix for the generator's subsets
    m = od.coo_to_matrix(coo, g.subset.astype(np.int32), g.subset.astype(np.int32))
    for s0, s1 in zip(a.sectors, m.sectors):
        assert np.array_equal(s0.row_p, s1.row_p) and np.array_equal(s0.col_i, s1.col_i)
    assert np.array_equal(m.to_dense(), a.to_dense())


def test_x_subset_rule_uses_largest_x():
    xyz = np.array([[0.0, 0, 0], [4.9, 0, 0], [5.0, 0, 0], [9.9, 0, 0], [10.0, 0, 0]], np.float32)
    # h11 = 10: the atom at the largest x wraps to subset 1 (mod n)
    assert od.x_subsets(xyz, 5, 2).tolist() == [1, 1, 2, 2, 1]
    assert od.x_subsets(xyz, 5, 1).tolist() == [1] * 5


@pytest.mark.parametrize("damage", ["truncated", "trailing", "negative_blk_p", "extent_beyond_area"])
def test_reader_rejects_damaged_files(tmp_path, damage):
    p = str(tmp_path / "hand.dbcsr")
    _hand_written(p)
    raw = bytearray(open(p, "rb").read())
    h1 = 10 + 80 + 1 + 16 + 4 * 2 + 4 * 3
    h3 = h1 + 16
    if damage == "truncated":
        raw = raw[:-8]
    elif damage == "trailing":
        raw += b"\0" * 8
    elif damage == "negative_blk_p":
        raw[h3 + 20:h3 + 24] = struct.pack("<i", -2)   # chunk 1 blk_p of block (1,2)
    else:
        raw[h1 + 12:h1 + 16] = struct.pack("<i", 1)   # chunk 2 data area 1 < its extent 2
        raw = raw[:-8]
    open(p, "wb").write(bytes(raw))
    with pytest.raises(gpu.LambError):
        gpu.dbcsr_read(p)
    with pytest.raises(ValueError):
        od.read_dbcsr(p)
