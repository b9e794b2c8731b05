"""ctypes declarations of the C ABI in include/lamb_gpu.h and include/lamb_gen.h."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .matrix import Sector


class CSector(C.Structure):
    _fields_ = [
        ("subset_row", C.c_int32), ("subset_col", C.c_int32),
        ("n_rows", C.c_int32), ("n_cols", C.c_int32),
        ("row_blk_sizes", C.c_void_p), ("col_blk_sizes", C.c_void_p),
        ("row_p", C.c_void_p), ("col_i", C.c_void_p), ("extents", C.c_void_p), ("data", C.c_void_p),
        ("n_blks", C.c_int64), ("data_len", C.c_int64),
    ]


class CSectorOut(C.Structure):
    _fields_ = CSector._fields_


class CSectorSizes(C.Structure):
    _fields_ = [
        ("subset_row", C.c_int32), ("subset_col", C.c_int32),
        ("n_rows", C.c_int32), ("n_cols", C.c_int32),
        ("n_blks", C.c_int64), ("data_len", C.c_int64),
    ]


class MultStats(C.Structure):
    _fields_ = [
        ("n_products", C.c_int64), ("n_products_skipped", C.c_int64),
        ("n_c_blocks", C.c_int64), ("n_c_blocks_dropped", C.c_int64),
        ("flops", C.c_double), ("ms_symbolic", C.c_double), ("ms_numeric", C.c_double), ("ms_total", C.c_double),
        ("mixed_slices", C.c_int32), ("kernel_launches", C.c_int32),
        ("ms_prepare", C.c_double), ("ms_filter", C.c_double), ("tensor_ops", C.c_double),
        ("ms_kernel", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class PurifyReport(C.Structure):
    _fields_ = [
        ("steps_done", C.c_int32), ("steps_mixed", C.c_int32),
        ("trace", C.c_double), ("idempotency", C.c_double), ("ms_total", C.c_double),
    ]


class DbcsrInfo(C.Structure):
    """lamb_dbcsr_info (include/lamb_gpu.h)."""
    _fields_ = [("name", C.c_char * 81), ("matrix_type", C.c_char), ("n_chunks", C.c_int32),
                ("data_type", C.c_int32), ("n_block_rows", C.c_int32), ("n_block_cols", C.c_int32),
                ("n_blks", C.c_int64), ("data_len", C.c_int64)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["name"] = d["name"].decode("ascii", "replace")
        d["matrix_type"] = d["matrix_type"].decode("ascii", "replace")
        return d


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data if a is not None and a.size else 0


def sector_to_c(s: Sector) -> CSector:
    """Borrowed view of a host sector (the arrays must outlive the call)."""
    for name, dt in (("row_blk_sizes", np.int8), ("col_blk_sizes", np.int8), ("row_p", np.int64),
                     ("col_i", np.int16), ("extents", np.int64), ("data", np.float64)):
        a = getattr(s, name)
        if a.dtype != dt or not a.flags.c_contiguous:
            raise TypeError(f"sector.{name} must be a contiguous {np.dtype(dt).name} array")
    return CSector(s.subset_row, s.subset_col, s.n_rows, s.n_cols,
                   _ptr(s.row_blk_sizes), _ptr(s.col_blk_sizes), _ptr(s.row_p), _ptr(s.col_i),
                   _ptr(s.extents), _ptr(s.data), s.n_blks, int(s.data.shape[0]))


def sector_from_c(c: CSector, copy: bool = True) -> Sector:
    def arr(ptr, n, dt):
        if n == 0 or not ptr:
            return np.zeros(0, dt)
        a = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dt))), shape=(n,))
        return a.copy() if copy else a
    return Sector(c.subset_row, c.subset_col,
                  arr(c.row_blk_sizes, c.n_rows, np.int8), arr(c.col_blk_sizes, c.n_cols, np.int8),
                  arr(c.row_p, c.n_rows + 1, np.int64), arr(c.col_i, c.n_blks, np.int16),
                  arr(c.extents, 2 * c.n_blks, np.int64).reshape(-1, 2), arr(c.data, c.data_len, np.float64))
