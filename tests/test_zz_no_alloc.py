"""lamb_gpu_trace_product_noalloc: the allocation-free Tr(X.Y) for callers
whose device memory is all owned by their own pool (or who must not let a
library allocate between their pre-allocated stages).

The matrices are handed over as device arrays the test owns (torch tensors);
the result is checked against the allocating entry point
lamb_gpu_matrix_trace_product on two calls in a row, and the size limit is
checked to be rejected with a clear status.  This file sorts last so that a
failure here comes after every other test has run."""
import ctypes as C

import numpy as np
import pytest

from lamb_b200 import gpu
from lamb_b200.gen import WaterGeometry

pytestmark = pytest.mark.gpu

TOL = 1e-12


class DCSR(C.Structure):
    _fields_ = [("n_rows", C.c_int32), ("n_cols", C.c_int32), ("nnz", C.c_int64),
                ("row_bs", C.c_void_p), ("col_bs", C.c_void_p), ("row_p", C.c_void_p), ("col", C.c_void_p),
                ("off", C.c_void_p), ("data", C.c_void_p)]


def _device_csr(m):
    """Global sector-order block-CSR of a host LambMatrix, on cuda:0."""
    import torch
    rbs = m.subset_blk_sizes(0)
    cbs = m.subset_blk_sizes(1)
    rbase = np.concatenate([[0], np.cumsum([len(b) for b in rbs])])
    cbase = np.concatenate([[0], np.cumsum([len(b) for b in cbs])])
    n_rows, n_cols = int(rbase[-1]), int(cbase[-1])
    rows = [[] for _ in range(n_rows)]
    data, dpos = [], 0
    for s in m.sectors:
        br = s.block_rows()
        for b in range(s.n_blks):
            r = int(rbase[s.subset_row - 1] + br[b])
            c = int(cbase[s.subset_col - 1] + s.col_i[b] - 1)
            f, l = int(s.extents[b, 0]), int(s.extents[b, 1])
            rows[r].append((c, dpos))
            data.append(s.data[f - 1:l])
            dpos += l - f + 1
    row_p = np.zeros(n_rows + 1, np.int64)
    cols, offs = [], []
    for r in range(n_rows):
        rows[r].sort()
        row_p[r + 1] = row_p[r] + len(rows[r])
        cols += [c for c, _ in rows[r]]
        offs += [o for _, o in rows[r]]
    keep = {}

    def dev(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")
        keep[id(t)] = t
        return t.data_ptr()
    st = DCSR(n_rows, n_cols, len(cols), dev(np.concatenate(rbs).astype(np.int8)),
              dev(np.concatenate(cbs).astype(np.int8)), dev(row_p), dev(np.asarray(cols, np.int32)),
              dev(np.asarray(offs, np.int64)), dev(np.concatenate(data) if data else np.zeros(1)))
    return st, keep


def _noalloc():
    f = gpu.lib().lamb_gpu_trace_product_noalloc
    f.argtypes = [C.POINTER(DCSR), C.POINTER(DCSR), C.c_void_p, C.POINTER(C.c_double)]
    f.restype = C.c_int32
    return f


def test_noalloc_trace_product_matches_allocating_entry_point(gpu_ctx):
    import torch
    g = WaterGeometry(40, None, 5.5, seed=17)
    x, y = g.matrix(3), g.matrix(4)
    dx, dy = gpu_ctx.upload(x), gpu_ctx.upload(y)
    ref = gpu_ctx.trace_product(dx, dy)
    assert abs(ref - np.trace(x.to_dense() @ y.to_dense())) <= TOL * max(1.0, abs(ref))
    sx, kx = _device_csr(x)
    sy, ky = _device_csr(y)
    torch.cuda.synchronize()
    f = _noalloc()
    for _ in range(2):
        out = C.c_double(float("nan"))
        st = f(C.byref(sx), C.byref(sy), None, C.byref(out))
        assert st == 0
        assert abs(out.value - ref) <= TOL * max(1.0, abs(ref))
    dx.destroy()
    dy.destroy()


def test_noalloc_empty_y_with_null_arrays(gpu_ctx):
    """Y without blocks may come with null arrays: the trace is 0."""
    import torch
    g = WaterGeometry(12, None, 4.0, seed=5)
    x = g.matrix(1)
    sx, kx = _device_csr(x)
    y = DCSR(sx.n_cols, sx.n_rows, 0, None, None, None, None, None, None)
    torch.cuda.synchronize()
    out = C.c_double(float("nan"))
    assert _noalloc()(C.byref(sx), C.byref(y), None, C.byref(out)) == 0
    assert out.value == 0.0


def test_noalloc_rejects_mismatched_blocking(gpu_ctx):
    """Same pattern, O blocks of 13 in X and 23 in Y: every Y_ji has the wrong
    shape, so the call skips the blocks and returns lamb_wrong_args."""
    import torch
    x = WaterGeometry(12, None, 4.0, seed=5, blk_o=13).matrix(1)
    y = WaterGeometry(12, None, 4.0, seed=5, blk_o=23).matrix(2)
    sx, kx = _device_csr(x)
    sy, ky = _device_csr(y)
    torch.cuda.synchronize()
    out = C.c_double(0.0)
    st = _noalloc()(C.byref(sx), C.byref(sy), None, C.byref(out))
    assert gpu.lib().lamb_gpu_status_type(st) == 100
    # the flag does not stick: a matching pair right after succeeds
    sy2, ky2 = _device_csr(WaterGeometry(12, None, 4.0, seed=5, blk_o=13).matrix(2))
    torch.cuda.synchronize()
    assert _noalloc()(C.byref(sx), C.byref(sy2), None, C.byref(out)) == 0


def test_noalloc_rejects_oversized_input():
    x = DCSR(1, 1, (1 << 20) + 1, None, None, None, None, None, None)
    out = C.c_double(0.0)
    st = _noalloc()(C.byref(x), C.byref(x), None, C.byref(out))
    assert gpu.lib().lamb_gpu_status_type(st) == 100
    assert gpu.lib().lamb_gpu_status_level(st) == 3
