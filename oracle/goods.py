"""LAMB goods messages (one sector on the wire) -- TEST INFRASTRUCTURE ONLY.

Restates, in numpy, the message ``lamb_goods_X_create`` packs and
``lamb_goods_X_unpack`` reads (src/lamb_goods_X_types.F90:79-268,
src/lamb_goods_X_methods.F90:166-218): an int64 word array whose first 12
words are 1-based (offset, size) slots for the index, the data, row_p, col_i,
extents and flags (:79-91), then row_p as int64 words, col_i as int16 values
packed four to a word (TRANSFER, little-endian), extents as int64 pairs and
the flags (zero), each section at least one word long (byte_to_word_count);
the data travel as a separate float64 array (the sector's data store).

Followed by intent, not by bug: row_p carries all n_rows + 1 offsets (the
reference writes n_rows words and size n_rows, :160-162, :196), and col_i is
read back as int16 (the reference's mult sector points at it as int64,
src/lamb_mult_sector_X_types.F90:74-84).  The library's
lamb_gpu_goods_pack / lamb_gpu_goods_unpack are checked against this file.
"""
from __future__ import annotations

import numpy as np

from lamb_b200.matrix import Sector

SLOT_INDEX_OFFSET, SLOT_INDEX_SIZE = 1, 2
SLOT_DATA_OFFSET, SLOT_DATA_SIZE = 3, 4
SLOT_ROW_P_OFFSET, SLOT_ROW_P_SIZE = 5, 6
SLOT_COL_I_OFFSET, SLOT_COL_I_SIZE = 7, 8
SLOT_EXTENTS_OFFSET, SLOT_EXTENTS_SIZE = 9, 10
SLOT_FLAGS_OFFSET, SLOT_FLAGS_SIZE = 11, 12
N_SLOTS = 12


def _words(n_bytes: int) -> int:
    """byte_to_word_count: 8-byte words, at least one."""
    return max(1, (n_bytes + 7) // 8)


def pack(s: Sector):
    """(index int64[n_words], data float64[data_len]) of one sector."""
    n_rows, n_blks = s.n_rows, s.n_blks
    w_rows = _words(8 * (n_rows + 1))
    w_cols = _words(2 * n_blks)
    w_ext = _words(16 * n_blks)
    w_flags = _words(n_blks)
    n_words = N_SLOTS + w_rows + w_cols + w_ext + w_flags
    idx = np.zeros(n_words, np.int64)
    h = {}
    off = 1 + N_SLOTS
    for slot, size, nw in ((SLOT_ROW_P_OFFSET, n_rows + 1, w_rows), (SLOT_COL_I_OFFSET, n_blks, w_cols),
                           (SLOT_EXTENTS_OFFSET, n_blks, w_ext), (SLOT_FLAGS_OFFSET, n_blks, w_flags)):
        h[slot], h[slot + 1] = off, size
        off += nw
    h[SLOT_INDEX_OFFSET], h[SLOT_INDEX_SIZE] = 1, n_words
    h[SLOT_DATA_OFFSET], h[SLOT_DATA_SIZE] = 1, int(s.data.shape[0])
    for k, v in h.items():
        idx[k - 1] = v
    a = h[SLOT_ROW_P_OFFSET] - 1
    idx[a:a + n_rows + 1] = np.asarray(s.row_p, np.int64)
    a = h[SLOT_COL_I_OFFSET] - 1
    raw = np.zeros(w_cols * 4, np.int16)
    raw[:n_blks] = np.asarray(s.col_i, np.int16)
    idx[a:a + w_cols] = raw.view(np.int64)
    a = h[SLOT_EXTENTS_OFFSET] - 1
    idx[a:a + 2 * n_blks] = np.asarray(s.extents, np.int64).reshape(-1)
    return idx, np.asarray(s.data, np.float64).copy()


def unpack(idx: np.ndarray, data: np.ndarray, subset_row: int, subset_col: int, row_blk_sizes, col_blk_sizes) -> Sector:
    idx = np.asarray(idx, np.int64)
    if idx.shape[0] < N_SLOTS or idx[SLOT_INDEX_OFFSET - 1] != 1 or idx[SLOT_INDEX_SIZE - 1] != idx.shape[0]:
        raise ValueError("not a goods index")
    n_rows = int(idx[SLOT_ROW_P_SIZE - 1]) - 1
    n_blks = int(idx[SLOT_COL_I_SIZE - 1])
    if n_rows != len(row_blk_sizes) or int(idx[SLOT_EXTENTS_SIZE - 1]) != n_blks:
        raise ValueError("goods sizes do not match the sector")
    a = int(idx[SLOT_ROW_P_OFFSET - 1]) - 1
    row_p = idx[a:a + n_rows + 1].copy()
    a = int(idx[SLOT_COL_I_OFFSET - 1]) - 1
    col_i = idx[a:a + _words(2 * n_blks)].view(np.int16)[:n_blks].copy()
    a = int(idx[SLOT_EXTENTS_OFFSET - 1]) - 1
    ext = idx[a:a + 2 * n_blks].reshape(n_blks, 2).copy()
    n_data = int(idx[SLOT_DATA_SIZE - 1])
    return Sector(subset_row, subset_col, np.asarray(row_blk_sizes, np.int8), np.asarray(col_blk_sizes, np.int8),
                  row_p, col_i, ext, np.asarray(data, np.float64)[:n_data].copy())
