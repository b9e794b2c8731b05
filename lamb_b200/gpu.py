"""Python host side of the C ABI (include/lamb_gpu.h), mirroring LAMB's
multiplication interface.

``lamb_multiply(matrix_a, matrix_b, matrix_c)`` keeps the argument meaning of
``lamb_multiply(matrix_a, matrix_b, matrix_c, error)``
(src/lamb_multiplication.F90:116-119): A and B are read, C is replaced by
A.B.  Errors surface as ``LambError`` carrying the LAMB error level and type
(src/lamb_error.F90:120-159) decoded from the C status.

There is no CPU fallback: every call goes through liblamb_b200.so and fails
loudly when the library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from .abi import CSector, CSectorOut, CSectorSizes, DbcsrInfo, MultStats, PurifyReport, sector_to_c
from .matrix import LambMatrix, Sector

FP64 = 0
MIXED = 1
NO_PRODUCT_FILTER = 2
NO_RESULT_FILTER = 4
ASYNC = 8

LEVELS = {1: "note", 2: "warning", 3: "failure", 4: "memory", 5: "fatal"}
TYPES = {1: "caller_error", 100: "wrong_args", 200: "precondition_failed", -1: "internal_error",
         -2: "overflow_error", -100: "invariant_failed", -200: "postcondition_failed", -300: "assertion_failed",
         -1000: "unimplemented", -2000: "external_error"}


class LambError(RuntimeError):
    def __init__(self, status: int, msg: str):
        self.status = status
        self.level = status // 100000 if status else 0
        self.type = status % 100000 - 50000 if status else 0
        super().__init__(f"[{LEVELS.get(self.level, self.level)}/{TYPES.get(self.type, self.type)}] {msg}")


_typed = False


def lib() -> C.CDLL:
    global _typed
    L = _lib.load("liblamb_b200.so")
    if not _typed:
        vp, i32, i64, dbl, u32 = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_uint32
        P = C.POINTER
        sig = {
            "lamb_gpu_ctx_create": [i32, P(vp)],
            "lamb_gpu_ctx_destroy": [vp],
            "lamb_gpu_last_error": [vp, C.c_char_p, i32],
            "lamb_gpu_status_level": [i32],
            "lamb_gpu_status_type": [i32],
            "lamb_gpu_ctx_get_stream": [vp, P(vp)],
            "lamb_gpu_ctx_synchronize": [vp],
            "lamb_gpu_matrix_upload": [vp, P(CSector), i32, P(i64)],
            "lamb_gpu_matrix_from_coo": [vp, i32, i32, vp, vp, vp, vp, i64, vp, vp, vp, vp, i64, P(i64)],
            "lamb_gpu_goods_size": [vp, i64, i32, P(i64), P(i64)],
            "lamb_gpu_goods_pack": [vp, i64, i32, vp, vp],
            "lamb_gpu_goods_unpack": [vp, vp, i64, vp, i32, vp, vp, P(i64)],
            "lamb_gpu_matrix_load_dbcsr": [vp, C.c_char_p, vp, i32, P(i64)],
            "lamb_dbcsr_scan": [C.c_char_p, P(DbcsrInfo), C.c_char_p, i32],
            "lamb_dbcsr_read": [C.c_char_p, vp, vp, vp, vp, vp, vp, i64, C.c_char_p, i32],
            "lamb_gpu_matrix_create_like": [vp, i64, P(i64)],
            "lamb_gpu_matrix_destroy": [vp, i64],
            "lamb_gpu_matrix_n_sectors": [vp, i64, P(i32)],
            "lamb_gpu_matrix_set_positions": [vp, i64, vp, i32, vp],
            "lamb_gpu_matrix_query": [vp, i64, P(CSectorSizes), i32],
            "lamb_gpu_matrix_download": [vp, i64, P(CSectorOut), i32],
            "lamb_gpu_multiply": [vp, i64, i64, i64, dbl, u32, P(MultStats)],
            "lamb_gpu_multiply_stacks": [vp, i64, i64, i64, dbl, u32, vp, P(i64)],
            "lamb_gpu_matrix_axpby": [vp, dbl, i64, dbl, i64],
            "lamb_gpu_matrix_copy": [vp, i64, i64],
            "lamb_gpu_matrix_trace": [vp, i64, P(dbl)],
            "lamb_gpu_matrix_trace_product": [vp, i64, i64, P(dbl)],
            "lamb_gpu_matrix_frobenius": [vp, i64, P(dbl)],
            "lamb_gpu_matrix_diff_frobenius": [vp, i64, i64, P(dbl)],
            "lamb_gpu_matrix_scale_shift": [vp, i64, dbl, dbl],
            "lamb_gpu_purify_mcweeny": [vp, i64, dbl, i32, i32, dbl, i64, P(PurifyReport)],
            "lamb_gpu_multiply_adjoint": [vp, i64, i64, i64, i64, i64],
            "lamb_gpu_batch_create": [vp, P(i64), P(i64), P(i64), i32, dbl, P(vp)],
            "lamb_gpu_batch_execute": [vp, P(MultStats)],
            "lamb_gpu_batch_destroy": [vp],
            "lamb_gpu_batch_config": [vp, P(i32), P(i32), P(i32)],
            "lamb_gpu_batch_run": [vp, u32, P(MultStats)],
            "lamb_gpu_batch_queue_order": [vp, P(i32)],
        }
        for name, args in sig.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.argtypes = args
            f.restype = i32
        _typed = True
    return L


def dbcsr_scan(path: str) -> dict:
    """Sizes and header fields of a DBCSR dump (lamb_dbcsr_scan; host only)."""
    info, msg = DbcsrInfo(), C.create_string_buffer(512)
    st = lib().lamb_dbcsr_scan(path.encode(), C.byref(info), msg, 512)
    if st != 0:
        raise LambError(st, msg.value.decode(errors="replace"))
    return info.as_dict()


def dbcsr_read(path: str) -> dict:
    """A DBCSR dump's blocks in coordinate form (lamb_dbcsr_read; host only)."""
    info = dbcsr_scan(path)
    rbs = np.zeros(info["n_block_rows"], np.int32)
    cbs = np.zeros(info["n_block_cols"], np.int32)
    rows = np.zeros(info["n_blks"], np.int32)
    cols = np.zeros(info["n_blks"], np.int32)
    ext = np.zeros((info["n_blks"], 2), np.int64)
    data = np.zeros(info["data_len"], np.float64)
    msg = C.create_string_buffer(512)
    st = lib().lamb_dbcsr_read(path.encode(), rbs.ctypes.data, cbs.ctypes.data, rows.ctypes.data, cols.ctypes.data,
                               ext.ctypes.data, data.ctypes.data, data.size, msg, 512)
    if st != 0:
        raise LambError(st, msg.value.decode(errors="replace"))
    return dict(info=info, row_blk_size=rbs, col_blk_size=cbs, rows=rows, cols=cols, extents=ext, data=data)


class Context:
    """One CUDA device and stream (lamb_gpu_ctx)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        st = lib().lamb_gpu_ctx_create(device, C.byref(self._h))
        if st != 0:
            raise LambError(st, f"cannot create a context on device {device} (needs an sm_100 GPU)")
        self.device = device

    def check(self, st: int) -> None:
        if st != 0:
            buf = C.create_string_buffer(1024)
            lib().lamb_gpu_last_error(self._h, buf, 1024)
            raise LambError(st, buf.value.decode(errors="replace"))

    @property
    def handle(self):
        return self._h

    def stream_ptr(self) -> int:
        p = C.c_void_p()
        self.check(lib().lamb_gpu_ctx_get_stream(self._h, C.byref(p)))
        return p.value or 0

    def synchronize(self) -> None:
        self.check(lib().lamb_gpu_ctx_synchronize(self._h))

    def close(self) -> None:
        if self._h:
            lib().lamb_gpu_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- matrices ---------------------------------------------------------------
    def upload(self, m: LambMatrix) -> "DeviceMatrix":
        arr = (CSector * len(m.sectors))(*[sector_to_c(s) for s in m.sectors])
        h = C.c_int64()
        self.check(lib().lamb_gpu_matrix_upload(self._h, arr, len(m.sectors), C.byref(h)))
        return DeviceMatrix(self, h.value)

    def from_coo(self, row_blk_sizes, col_blk_sizes, row_subset, col_subset, blk_row, blk_col, extents,
                 data) -> "DeviceMatrix":
        """Device matrix from a coordinate block list (lamb_gpu_matrix_from_coo):
        1-based global atoms per block, 1-based inclusive extents into data."""
        rbs = np.ascontiguousarray(row_blk_sizes, np.int8)
        cbs = np.ascontiguousarray(col_blk_sizes, np.int8)
        rs = np.ascontiguousarray(row_subset, np.int32)
        cs = np.ascontiguousarray(col_subset, np.int32)
        br = np.ascontiguousarray(blk_row, np.int32)
        bc = np.ascontiguousarray(blk_col, np.int32)
        ex = np.ascontiguousarray(extents, np.int64).reshape(-1)
        d = np.ascontiguousarray(data, np.float64)
        h = C.c_int64()
        self.check(lib().lamb_gpu_matrix_from_coo(self._h, rbs.size, cbs.size, rbs.ctypes.data, cbs.ctypes.data,
                                                  rs.ctypes.data, cs.ctypes.data, br.size, br.ctypes.data,
                                                  bc.ctypes.data, ex.ctypes.data, d.ctypes.data, d.size,
                                                  C.byref(h)))
        return DeviceMatrix(self, h.value)

    def load_dbcsr(self, path: str, xyz: Optional[np.ndarray] = None, n_x_cubes: int = 1) -> "DeviceMatrix":
        """lamb_load_dbcsr at one rank (lamb_gpu_matrix_load_dbcsr)."""
        x = None if xyz is None else np.ascontiguousarray(xyz, np.float32).reshape(-1)
        h = C.c_int64()
        self.check(lib().lamb_gpu_matrix_load_dbcsr(self._h, path.encode(), None if x is None else x.ctypes.data,
                                                    n_x_cubes, C.byref(h)))
        return DeviceMatrix(self, h.value)

    def goods_unpack(self, index, data, n_cols: int, row_blk_sizes, col_blk_sizes) -> "DeviceMatrix":
        """A goods message (numpy arrays or CUDA tensors) as a one-sector device
        matrix (lamb_gpu_goods_unpack)."""
        def ptr(x):
            if hasattr(x, "data_ptr"):
                return x.data_ptr() if x.numel() else None
            return x.ctypes.data if x.size else None
        n_idx = int(index.numel() if hasattr(index, "numel") else index.size)
        rbs = np.ascontiguousarray(row_blk_sizes, np.int8)
        cbs = np.ascontiguousarray(col_blk_sizes, np.int8)
        if hasattr(index, "data_ptr") and index.is_cuda:
            import torch
            torch.cuda.synchronize(index.device)
        h = C.c_int64()
        self.check(lib().lamb_gpu_goods_unpack(self._h, ptr(index), n_idx, ptr(data), n_cols,
                                               rbs.ctypes.data if rbs.size else None,
                                               cbs.ctypes.data if cbs.size else None, C.byref(h)))
        return DeviceMatrix(self, h.value)

    def create_like(self, like: "DeviceMatrix") -> "DeviceMatrix":
        h = C.c_int64()
        self.check(lib().lamb_gpu_matrix_create_like(self._h, like.h, C.byref(h)))
        return DeviceMatrix(self, h.value)

    def multiply(self, a: "DeviceMatrix", b: "DeviceMatrix", c: "DeviceMatrix", eps: float = 0.0,
                 flags: int = 0) -> dict:
        st = MultStats()
        self.check(lib().lamb_gpu_multiply(self._h, a.h, b.h, c.h, eps, flags, C.byref(st)))
        return st.as_dict()

    # -- algebra ------------------------------------------------------------------
    def axpby(self, alpha: float, x: "DeviceMatrix", beta: float, y: "DeviceMatrix") -> None:
        """y := alpha*x + beta*y over the union pattern."""
        self.check(lib().lamb_gpu_matrix_axpby(self._h, alpha, x.h, beta, y.h))

    def copy(self, x: "DeviceMatrix", y: "DeviceMatrix") -> None:
        self.check(lib().lamb_gpu_matrix_copy(self._h, x.h, y.h))

    def scale_shift(self, x: "DeviceMatrix", alpha: float, shift: float = 0.0) -> None:
        self.check(lib().lamb_gpu_matrix_scale_shift(self._h, x.h, alpha, shift))

    def _scalar(self, fn, *hs) -> float:
        v = C.c_double()
        self.check(fn(self._h, *[m.h for m in hs], C.byref(v)))
        return v.value

    def trace(self, x: "DeviceMatrix") -> float:
        return self._scalar(lib().lamb_gpu_matrix_trace, x)

    def trace_product(self, x: "DeviceMatrix", y: "DeviceMatrix") -> float:
        return self._scalar(lib().lamb_gpu_matrix_trace_product, x, y)

    def frobenius(self, x: "DeviceMatrix") -> float:
        return self._scalar(lib().lamb_gpu_matrix_frobenius, x)

    def diff_frobenius(self, x: "DeviceMatrix", y: "DeviceMatrix") -> float:
        return self._scalar(lib().lamb_gpu_matrix_diff_frobenius, x, y)

    def purify(self, h: "DeviceMatrix", p: "DeviceMatrix", mu: float = 0.0, steps: int = 30, fp64_tail: int = 5,
               eps: float = 0.0) -> dict:
        """McWeeny purification of h into p (p from create_like(h))."""
        rep = PurifyReport()
        self.check(lib().lamb_gpu_purify_mcweeny(self._h, h.h, mu, steps, fp64_tail, eps, p.h, C.byref(rep)))
        return {k: getattr(rep, k) for k, _ in rep._fields_}

    def adjoint(self, a: "DeviceMatrix", b: "DeviceMatrix", dc: "DeviceMatrix", da: Optional["DeviceMatrix"],
                db: Optional["DeviceMatrix"]) -> None:
        """da := (dc . b^T) on a's pattern, db := (a^T . dc) on b's pattern."""
        self.check(lib().lamb_gpu_multiply_adjoint(self._h, a.h, b.h, dc.h, da.h if da else 0, db.h if db else 0))

    def batch(self, a: Sequence["DeviceMatrix"], b: Sequence["DeviceMatrix"], c: Sequence["DeviceMatrix"],
              eps: float = 0.0) -> "Batch":
        """Independent C_i = A_i . B_i in one persistent launch (graph-replayed)."""
        n = len(a)
        arr = lambda ms: (C.c_int64 * n)(*[m.h for m in ms])
        h = C.c_void_p()
        self.check(lib().lamb_gpu_batch_create(self._h, arr(a), arr(b), arr(c), n, eps, C.byref(h)))
        return Batch(self, h)

    def stacks(self, a: "DeviceMatrix", b: "DeviceMatrix", c: "DeviceMatrix", eps: float = 0.0,
               flags: int = 0) -> np.ndarray:
        n = C.c_int64(0)
        self.check(lib().lamb_gpu_multiply_stacks(self._h, a.h, b.h, c.h, eps, flags, None, C.byref(n)))
        out = np.zeros((max(n.value, 1), 5), np.int64)
        self.check(lib().lamb_gpu_multiply_stacks(self._h, a.h, b.h, c.h, eps, flags, out.ctypes.data, C.byref(n)))
        return out[:n.value]


class Batch:
    """A created batch (lamb_gpu_batch)."""

    def __init__(self, ctx: Context, h):
        self.ctx, self.h = ctx, h

    def execute(self) -> dict:
        """Numeric phase only (graph replay)."""
        st = MultStats()
        self.ctx.check(lib().lamb_gpu_batch_execute(self.h, C.byref(st)))
        return st.as_dict()

    def run_full(self) -> dict:
        """Symbolic phase, graph-replayed numeric launch and result filter of
        every instance (lamb_gpu_batch_run with LAMB_GPU_BATCH_FULL)."""
        st = MultStats()
        self.ctx.check(lib().lamb_gpu_batch_run(self.h, 1, C.byref(st)))
        return st.as_dict()

    def config(self) -> dict:
        w, c, g, o = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        self.ctx.check(lib().lamb_gpu_batch_config(self.h, C.byref(w), C.byref(c), C.byref(g)))
        self.ctx.check(lib().lamb_gpu_batch_queue_order(self.h, C.byref(o)))
        return {"warps": w.value, "cap": c.value, "grab": g.value, "order": "shape" if o.value else "instance"}

    def destroy(self) -> None:
        if self.h:
            lib().lamb_gpu_batch_destroy(self.h)
            self.h = None


class DeviceMatrix:
    """A matrix resident on the GPU (lamb_gpu_matrix handle)."""

    def __init__(self, ctx: Context, h: int):
        self.ctx, self.h = ctx, h

    def sizes(self) -> List[CSectorSizes]:
        n = C.c_int32()
        self.ctx.check(lib().lamb_gpu_matrix_n_sectors(self.ctx.handle, self.h, C.byref(n)))
        arr = (CSectorSizes * n.value)()
        self.ctx.check(lib().lamb_gpu_matrix_query(self.ctx.handle, self.h, arr, n.value))
        return list(arr)

    def download(self, pinned: bool = False, out: Optional[LambMatrix] = None) -> LambMatrix:
        """Two-phase download: query sizes, allocate (or reuse `out`'s arrays
        when they are large enough), fill.  Returned arrays are views trimmed
        to the downloaded sizes."""
        sz = self.sizes()
        secs, outs = [], []
        for i, s in enumerate(sz):
            alloc = _pinned_empty if pinned else np.empty
            old = out.sectors[i] if out is not None and i < len(out.sectors) else None

            def take(a, n, dt, shape=None):
                if a is not None and a.dtype == dt and a.size >= n and a.flags.c_contiguous:
                    v = a.reshape(-1)[:n]
                else:
                    v = (alloc if dt == np.float64 else np.empty)(n, dt)
                return v.reshape(shape) if shape else v

            sec = Sector(s.subset_row, s.subset_col,
                         take(old.row_blk_sizes if old else None, s.n_rows, np.int8),
                         take(old.col_blk_sizes if old else None, s.n_cols, np.int8),
                         take(old.row_p if old else None, s.n_rows + 1, np.int64),
                         take(old.col_i if old else None, s.n_blks, np.int16),
                         take(old.extents if old else None, 2 * s.n_blks, np.int64, (s.n_blks, 2)),
                         take(old.data if old else None, s.data_len, np.float64))
            secs.append(sec)
            o = CSectorOut(s.subset_row, s.subset_col, s.n_rows, s.n_cols,
                           _p(sec.row_blk_sizes), _p(sec.col_blk_sizes), _p(sec.row_p), _p(sec.col_i),
                           _p(sec.extents), _p(sec.data), s.n_blks, s.data_len)
            outs.append(o)
        arr = (CSectorOut * len(outs))(*outs)
        self.ctx.check(lib().lamb_gpu_matrix_download(self.ctx.handle, self.h, arr, len(outs)))
        # after an asynchronous multiply the queried block counts are capacities:
        # keep what the download wrote
        for i, s in enumerate(secs):
            nb = int(arr[i].n_blks)
            if nb != s.col_i.shape[0]:
                secs[i] = Sector(s.subset_row, s.subset_col, s.row_blk_sizes, s.col_blk_sizes, s.row_p,
                                 s.col_i[:nb], s.extents[:nb], s.data)
        return LambMatrix(secs, "C")

    def goods(self, sector: int, device: bool = False):
        """One sector as a goods message (lamb_gpu_goods_pack): (index int64,
        data float64) as numpy arrays, or as CUDA tensors when device=True."""
        nw, nd = C.c_int64(), C.c_int64()
        self.ctx.check(lib().lamb_gpu_goods_size(self.ctx.handle, self.h, sector, C.byref(nw), C.byref(nd)))
        if device:
            import torch
            dev = torch.device("cuda", self.ctx.device)
            idx = torch.empty(nw.value, dtype=torch.int64, device=dev)
            dat = torch.empty(max(nd.value, 1), dtype=torch.float64, device=dev)[:nd.value]
            torch.cuda.synchronize(dev)
            self.ctx.check(lib().lamb_gpu_goods_pack(self.ctx.handle, self.h, sector, idx.data_ptr(),
                                                     dat.data_ptr() if nd.value else None))
            return idx, dat
        idx = np.empty(nw.value, np.int64)
        dat = np.empty(nd.value, np.float64)
        self.ctx.check(lib().lamb_gpu_goods_pack(self.ctx.handle, self.h, sector, idx.ctypes.data,
                                                 dat.ctypes.data if nd.value else None))
        return idx, dat

    def set_positions(self, xyz: np.ndarray, box) -> None:
        """Row-atom coordinates in sector order (locality hint for the multiply)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        bx = np.ascontiguousarray(np.broadcast_to(np.asarray(box, np.float32), (3,)))
        self.ctx.check(lib().lamb_gpu_matrix_set_positions(self.ctx.handle, self.h, xyz.ctypes.data, xyz.shape[0],
                                                           bx.ctypes.data))

    def destroy(self) -> None:
        if self.h:
            lib().lamb_gpu_matrix_destroy(self.ctx.handle, self.h)
            self.h = 0


def _p(a: np.ndarray) -> int:
    return a.ctypes.data if a.size else 0


_pinned_keep = []


def _pinned_empty(n: int, dtype) -> np.ndarray:
    import torch
    t = torch.empty(int(n) * np.dtype(dtype).itemsize, dtype=torch.uint8, pin_memory=True)
    a = t.numpy().view(dtype)
    _pinned_keep.append(t)
    if len(_pinned_keep) > 64:
        del _pinned_keep[:-64]
    return a


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def lamb_multiply(matrix_a: LambMatrix, matrix_b: LambMatrix, matrix_c: Optional[LambMatrix] = None,
                  eps: float = 0.0, flags: int = FP64, ctx: Optional[Context] = None, stats: Optional[dict] = None
                  ) -> LambMatrix:
    """C := A.B on the GPU through the C ABI; returns C (also stored into
    matrix_c's sector list when given, like the reference's intent(inout))."""
    ctx = ctx or default_context()
    da = ctx.upload(matrix_a)
    db = da if matrix_b is matrix_a else ctx.upload(matrix_b)
    dc = ctx.create_like(da)
    try:
        st = ctx.multiply(da, db, dc, eps, flags)
        if stats is not None:
            stats.update(st)
        c = dc.download()
    finally:
        dc.destroy()
        if db is not da:
            db.destroy()
        da.destroy()
    if matrix_c is not None:
        matrix_c.sectors = c.sectors
        return matrix_c
    return c
