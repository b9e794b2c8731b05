"""Host-side LAMB matrices in the reference's single-rank sector storage.

A ``LambMatrix`` mirrors ``lamb_matrix_d_type`` (src/lamb_matrix_X_types.F90:78-86):
a list of sectors, one per (row subset, column subset) pair.  A ``Sector``
mirrors ``lamb_sector_d_type`` (src/lamb_sector_X_types.F90:79-87) with its
``lamb_index_type`` (src/lamb_index_types.F90:86-105) flattened into arrays:

* ``row_p``   int64 [n_rows+1], exclusive offsets (index_count_to_offset,
  src/lamb_index_methods.F90:264-274);
* ``col_i``   int16 [n_blks], 1-based local columns, ascending within a row;
* ``extents`` int64 [n_blks, 2], 1-based inclusive (first, last) into ``data``;
* ``data``    float64, blocks column-major (DBCSR ``blk_p`` convention,
  src/lamb_io_operations.F90:666-682).
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional

import numpy as np


@dataclasses.dataclass
class Sector:
    subset_row: int
    subset_col: int
    row_blk_sizes: np.ndarray
    col_blk_sizes: np.ndarray
    row_p: np.ndarray
    col_i: np.ndarray
    extents: np.ndarray
    data: np.ndarray

    @property
    def n_rows(self) -> int:
        return int(self.row_blk_sizes.shape[0])

    @property
    def n_cols(self) -> int:
        return int(self.col_blk_sizes.shape[0])

    @property
    def n_blks(self) -> int:
        return int(self.col_i.shape[0])

    def block_rows(self) -> np.ndarray:
        """0-based local row of every block."""
        return np.repeat(np.arange(self.n_rows, dtype=np.int64), np.diff(self.row_p))

    def get_blk_n(self, row: int, col: int) -> int:
        """Block id (0-based) of local (row, col), both 1-based, or -1.

        Binary search of ``get_blk_n`` (src/lamb_index_methods.F90:81-107).
        """
        first, last = int(self.row_p[row - 1]), int(self.row_p[row]) - 1
        while first <= last:
            mid = (first + last) // 2
            c = int(self.col_i[mid])
            if c == col:
                return mid
            if c < col:
                first = mid + 1
            else:
                last = mid - 1
        return -1

    def block(self, blk: int) -> np.ndarray:
        """Block ``blk`` (0-based) as a (rows, cols) view, column-major storage."""
        r = int(np.searchsorted(self.row_p, blk, side="right") - 1)
        c = int(self.col_i[blk]) - 1
        m, n = int(self.row_blk_sizes[r]), int(self.col_blk_sizes[c])
        f, l = int(self.extents[blk, 0]), int(self.extents[blk, 1])
        assert l - f + 1 == m * n
        return self.data[f - 1:l].reshape(n, m).T

    def validate(self) -> None:
        if self.row_p.shape[0] != self.n_rows + 1 or self.row_p[0] != 0:
            raise ValueError("row_p must have n_rows+1 entries starting at 0")
        if np.any(np.diff(self.row_p) < 0) or self.row_p[-1] != self.n_blks:
            raise ValueError("row_p must be non-decreasing and end at n_blks")
        if self.n_blks:
            if self.col_i.min() < 1 or self.col_i.max() > self.n_cols:
                raise ValueError("col_i out of range")
            rows = self.block_rows()
            same = rows[1:] == rows[:-1]
            if np.any(same & (np.diff(self.col_i.astype(np.int64)) <= 0)):
                raise ValueError("col_i must increase strictly within a row")
            sz = self.row_blk_sizes[rows].astype(np.int64) * self.col_blk_sizes[self.col_i - 1].astype(np.int64)
            ln = self.extents[:, 1] - self.extents[:, 0] + 1
            if np.any(ln != sz):
                raise ValueError("extent length does not match the block size")
            if np.any((self.extents[:, 0] < 1) & (sz > 0)) or np.any(self.extents[:, 1] > self.data.shape[0]):
                raise ValueError("extent outside the data store")


@dataclasses.dataclass
class LambMatrix:
    sectors: List[Sector]
    name: str = "matrix"

    @property
    def n_subsets(self) -> int:
        return max(max(s.subset_row, s.subset_col) for s in self.sectors)

    def sector(self, m: int, n: int) -> Optional[Sector]:
        for s in self.sectors:
            if s.subset_row == m and s.subset_col == n:
                return s
        return None

    def subset_blk_sizes(self, axis: int) -> List[np.ndarray]:
        """Block sizes of every subset along rows (axis 0) or columns (axis 1)."""
        out = {}
        for s in self.sectors:
            if axis == 0:
                out[s.subset_row] = s.row_blk_sizes
            else:
                out[s.subset_col] = s.col_blk_sizes
        return [out[k] for k in sorted(out)]

    def validate(self) -> None:
        for s in self.sectors:
            s.validate()

    def to_dense(self) -> np.ndarray:
        """Dense matrix with subset-1 atoms first, then subset 2, ... (test helper)."""
        rbs = self.subset_blk_sizes(0)
        cbs = self.subset_blk_sizes(1)
        r_off = [np.concatenate([[0], np.cumsum(b.astype(np.int64))]) for b in rbs]
        c_off = [np.concatenate([[0], np.cumsum(b.astype(np.int64))]) for b in cbs]
        r_base = np.concatenate([[0], np.cumsum([o[-1] for o in r_off])])
        c_base = np.concatenate([[0], np.cumsum([o[-1] for o in c_off])])
        dense = np.zeros((int(r_base[-1]), int(c_base[-1])))
        for s in self.sectors:
            ro, co = r_off[s.subset_row - 1], c_off[s.subset_col - 1]
            rb, cb = r_base[s.subset_row - 1], c_base[s.subset_col - 1]
            rows = s.block_rows()
            for b in range(s.n_blks):
                r, c = int(rows[b]), int(s.col_i[b]) - 1
                m, n = int(s.row_blk_sizes[r]), int(s.col_blk_sizes[c])
                if m * n == 0:
                    continue
                f = int(s.extents[b, 0])
                blk = s.data[f - 1:f - 1 + m * n].reshape(n, m).T
                dense[rb + ro[r]:rb + ro[r] + m, cb + co[c]:cb + co[c] + n] = blk
        return dense

    def block_pattern(self) -> dict:
        """{(subset_row, subset_col): set of (row, col) 1-based} of present blocks."""
        out = {}
        for s in self.sectors:
            rows = s.block_rows() + 1
            out[(s.subset_row, s.subset_col)] = set(zip(rows.tolist(), s.col_i.astype(np.int64).tolist()))
        return out

    def frobenius(self) -> float:
        tot = 0.0
        for s in self.sectors:
            if s.n_blks == 0:
                continue
            used = np.zeros(s.data.shape[0], bool)
            for f, l in s.extents:
                if l >= f:
                    used[f - 1:l] = True
            tot += float(np.sum(s.data[used] ** 2))
        return float(np.sqrt(tot))
