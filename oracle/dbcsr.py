"""DBCSR dump files and LAMB's single-rank sector layout -- TEST INFRASTRUCTURE ONLY.

Restates, in numpy, what the reference does when it loads a DBCSR dump into a
LAMB matrix at one rank (``lamb_load_dbcsr``, src/lamb_io_operations.F90:267-756):

* ``read_dbcsr``   -- the file layout of the \\page dbcsr_file_format comment
  (src/lamb_io_operations.F90:300-330) and the offsets computed by
  ``load_dbcsr_chunks`` (:559-596): sub-header 1, then one sub-header 2 per
  chunk, one sub-header 3 (row_p, col_i, blk_p) per chunk, then the chunks'
  data areas.  Every chunk becomes coordinate blocks (global row, global
  column, extents, data store) as at :647-665.
* ``coo_to_matrix`` -- ``lamb_dist_localize_index`` + ``internal_distribute``
  + ``fill_local_sectors`` (src/lamb_matrix_operations.F90:88-371) at one
  rank: each atom's subset follows the float32 rule of
  ``lamb_partition_which_cube1`` (src/lamb_partition_methods.F90:85-96) with
  the multiplier n_cubes / h11 of src/lamb_partition_types.F90:139-143, local
  indices follow global order, and each sector's index becomes row-sorted CSR
  with 1-based extents into one data store per sector.
* ``write_dbcsr``   -- the inverse of ``read_dbcsr``, for fixtures (the
  reference's own small.dbcsr is not part of its tree).

The GPU loader (``lamb_gpu_matrix_load_dbcsr``) is checked against this file
block for block.
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional, Sequence

import numpy as np

from lamb_b200.matrix import LambMatrix, Sector

VERSION_LEN = 10   # dbcsr_version_len, src/lamb_io_operations.F90:332
NAME_LEN = 80      # dbcsr_default_string_length, :333


@dataclasses.dataclass
class DbcsrCoo:
    """Blocks of a DBCSR dump in coordinate form (global, 1-based atoms)."""
    name: str
    matrix_type: str
    data_type: int
    row_blk_size: np.ndarray   # int32 [nblkrows]
    col_blk_size: np.ndarray   # int32 [nblkcols]
    rows: np.ndarray           # int32 [n]  (global_idx(1,:))
    cols: np.ndarray           # int32 [n]  (global_idx(2,:))
    extents: np.ndarray        # int64 [n,2], 1-based inclusive into the block's data store
    store: np.ndarray          # int32 [n], 0-based chunk (data store) of each block
    stores: List[np.ndarray]   # float64 data areas, one per chunk (read up to the largest extent)


def read_dbcsr(path: str) -> DbcsrCoo:
    raw = np.fromfile(path, dtype=np.uint8)
    pos = 0

    def take(n_bytes):
        nonlocal pos
        if pos + n_bytes > raw.size:
            raise ValueError("DBCSR file truncated")
        out = raw[pos:pos + n_bytes]
        pos += n_bytes
        return out

    def ints(n):
        return take(4 * n).view(np.int32).copy()

    bytes(take(VERSION_LEN))
    name = bytes(take(NAME_LEN)).decode("ascii", "replace").rstrip()
    mtype = chr(int(take(1)[0]))
    numnodes, data_type, nbr, nbc = (int(x) for x in ints(4))
    rbs, cbs = ints(nbr), ints(nbc)
    if numnodes < 1 or nbr < 0 or nbc < 0:
        raise ValueError("DBCSR header: bad sizes")
    h2 = ints(2 * numnodes).reshape(numnodes, 2)          # (nblks, data_area_size) per chunk
    rows, cols, ext, store, stores = [], [], [], [], []
    idx3 = [ ]
    for c in range(numnodes):
        nb = int(h2[c, 0])
        row_p, col_i, blk_p = ints(nbr + 1), ints(nb), ints(nb)
        idx3.append((row_p, col_i, blk_p))
    for c in range(numnodes):
        row_p, col_i, blk_p = idx3[c]
        nb, area = int(h2[c, 0]), int(h2[c, 1])
        r = np.zeros(nb, np.int32)
        for bin_ in range(nbr):           # global_idx(1, row_p(bin)+1 : row_p(bin+1)) = bin
            r[row_p[bin_]:row_p[bin_ + 1]] = bin_ + 1
        e1 = blk_p.astype(np.int64)
        e2 = e1 - 1 + rbs[r - 1].astype(np.int64) * cbs[col_i - 1].astype(np.int64)
        if nb and (e1.min() < 1):
            raise ValueError("DBCSR: non-positive blk_p (transposed blocks) is not supported")
        to_read = int(e2.max()) if nb else 0
        if to_read > area:
            raise ValueError("DBCSR: data block extent exceeds data area")
        stores.append(take(8 * area).view(np.float64)[:to_read].copy())
        rows.append(r)
        cols.append(col_i.astype(np.int32))
        ext.append(np.stack([e1, e2], axis=1))
        store.append(np.full(nb, c, np.int32))
    if pos != raw.size:
        raise ValueError("DBCSR file has trailing bytes")
    cat = (lambda xs, dt: np.concatenate(xs).astype(dt) if xs else np.zeros(0, dt))
    return DbcsrCoo(name, mtype, data_type, rbs, cbs, cat(rows, np.int32), cat(cols, np.int32),
                    np.concatenate(ext) if ext else np.zeros((0, 2), np.int64), cat(store, np.int32), stores)


def write_dbcsr(path: str, name: str, row_blk_size, col_blk_size, chunks, data_type: int = 3,
                matrix_type: str = "N") -> None:
    """chunks: list of (row_p int32 [nbr+1] 0-based, col_i int32 1-based, blk_p int32 1-based,
    data float64) -- the DBCSR dump of one process each."""
    rbs = np.asarray(row_blk_size, np.int32)
    cbs = np.asarray(col_blk_size, np.int32)
    with open(path, "wb") as f:
        f.write(b"DBCSRv1.0 "[:VERSION_LEN].ljust(VERSION_LEN))
        f.write(name.encode("ascii")[:NAME_LEN].ljust(NAME_LEN))
        f.write(matrix_type.encode("ascii")[:1])
        f.write(np.array([len(chunks), data_type, rbs.size, cbs.size], np.int32).tobytes())
        f.write(rbs.tobytes())
        f.write(cbs.tobytes())
        for _, col_i, _, data in chunks:
            f.write(np.array([len(col_i), len(data)], np.int32).tobytes())
        for row_p, col_i, blk_p, _ in chunks:
            f.write(np.asarray(row_p, np.int32).tobytes())
            f.write(np.asarray(col_i, np.int32).tobytes())
            f.write(np.asarray(blk_p, np.int32).tobytes())
        for _, _, _, data in chunks:
            f.write(np.asarray(data, np.float64).tobytes())


def chunks_from_dense_blocks(n_rows: int, blocks, rbs, cbs, n_chunks: int, seed: int = 0):
    """Splits {(row, col): block (rbs[row] x cbs[col], column-major)} (0-based
    atoms) over n_chunks DBCSR chunks, each holding its blocks in row-sorted
    CSR with its own data area; blocks go to chunks at random and each
    chunk's data area stores them in a shuffled order (blk_p need not follow
    the index order)."""
    rng = np.random.default_rng(seed)
    keys = sorted(blocks)
    owner = rng.integers(0, n_chunks, len(keys))
    out = []
    for c in range(n_chunks):
        mine = [k for k, o in zip(keys, owner) if o == c]
        order = rng.permutation(len(mine))
        data, blk_p = [], np.zeros(len(mine), np.int32)
        pos = 1
        for t in order:
            blk_p[t] = pos
            x = np.asarray(blocks[mine[t]], np.float64).ravel(order="F")
            data.append(x)
            pos += x.size
        row_p = np.zeros(n_rows + 1, np.int32)
        for r, _ in mine:
            row_p[r + 1] += 1
        row_p = np.cumsum(row_p).astype(np.int32)
        col_i = np.array([cc + 1 for _, cc in mine], np.int32)
        out.append((row_p, col_i, blk_p, np.concatenate(data) if data else np.zeros(0)))
    return out


def x_subsets(coords: Optional[np.ndarray], n_atoms: int, n_x_cubes: int) -> np.ndarray:
    """1-based subset of every atom: 1 + mod(int(x * (n / h11)), n) in float32,
    h11 = max x of the coordinates (src/lamb_io_operations.F90:448-457)."""
    if n_x_cubes <= 1 or n_atoms == 0:
        return np.ones(n_atoms, np.int32)
    x = np.asarray(coords, np.float32).reshape(n_atoms, 3)[:, 0]
    h11 = np.float32(x.max())
    mult = np.float32(n_x_cubes) / h11
    c = np.trunc((x * mult).astype(np.float32)).astype(np.int64) % n_x_cubes
    return (c + 1).astype(np.int32)


def coo_to_matrix(coo: DbcsrCoo, row_subset: np.ndarray, col_subset: np.ndarray, name: str = "dbcsr") -> LambMatrix:
    """Single-rank sectors of a coordinate block list: sector (m, n) holds the
    blocks whose row atom is in subset m and column atom in subset n, indexed
    by local atoms (global order within a subset), rows sorted and columns
    sorted within a row, data appended block after block in that order."""
    R, S = int(row_subset.max(initial=1)), int(col_subset.max(initial=1))
    rloc = np.zeros(row_subset.size, np.int64)
    cloc = np.zeros(col_subset.size, np.int64)
    for s in range(1, R + 1):
        m = row_subset == s
        rloc[m] = np.arange(int(m.sum()))
    for s in range(1, S + 1):
        m = col_subset == s
        cloc[m] = np.arange(int(m.sum()))
    key = np.stack([coo.rows, coo.cols], 1)
    if len(np.unique(key, axis=0)) != len(key):
        raise ValueError("duplicate block")
    secs = []
    for m_ in range(1, R + 1):
        ratoms = np.nonzero(row_subset == m_)[0]
        for n_ in range(1, S + 1):
            catoms = np.nonzero(col_subset == n_)[0]
            sel = np.nonzero((row_subset[coo.rows - 1] == m_) & (col_subset[coo.cols - 1] == n_))[0]
            lr, lc = rloc[coo.rows[sel] - 1], cloc[coo.cols[sel] - 1]
            order = np.lexsort((lc, lr))
            sel, lr, lc = sel[order], lr[order], lc[order]
            row_p = np.zeros(len(ratoms) + 1, np.int64)
            np.add.at(row_p, lr + 1, 1)
            row_p = np.cumsum(row_p)
            data, ext, pos = [], np.zeros((len(sel), 2), np.int64), 1
            for t, b in enumerate(sel):
                e1, e2 = coo.extents[b]
                x = coo.stores[coo.store[b]][e1 - 1:e2]
                ext[t] = (pos, pos + x.size - 1)
                pos += x.size
                data.append(x)
            secs.append(Sector(m_, n_, coo.row_blk_size[ratoms].astype(np.int8),
                               coo.col_blk_size[catoms].astype(np.int8), row_p, (lc + 1).astype(np.int16), ext,
                               np.concatenate(data) if data else np.zeros(0)))
    return LambMatrix(secs, name)
