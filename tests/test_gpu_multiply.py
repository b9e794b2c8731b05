"""GPU multiply against the CPU oracle, through the C ABI (liblamb_b200.so).

Bar: C block pattern and stacks bit-exact, values within 1e-12 relative
Frobenius error of the oracle (FP64 path)."""
import numpy as np
import pytest

import oracle
from lamb_b200 import gpu
from lamb_b200.gen import WATER_192, WATER_6144, WaterGeometry, random_fill_matrix
from lamb_b200.matrix import LambMatrix, Sector
from tests.helpers import assert_same_pattern, block_values, rel_frobenius_error

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def _gpu_mult(ctx, a, b, eps, flags=0):
    da = ctx.upload(a)
    db = da if b is a else ctx.upload(b)
    dc = ctx.create_like(da)
    st = ctx.multiply(da, db, dc, eps, flags)
    c = dc.download()
    for m in (dc, db, da):
        m.destroy()
    return c, st


def _no_borderline(c_ref, eps):
    if eps <= 0:
        return
    for v in block_values(c_ref).values():
        n = float(np.sqrt(np.sum(v ** 2)))
        assert abs(n - eps) > 1e-9 * eps, "a C block norm sits on the filter threshold"


def _with_values(a, seed):
    rng = np.random.default_rng(seed)
    return LambMatrix([Sector(s.subset_row, s.subset_col, s.row_blk_sizes, s.col_blk_sizes, s.row_p, s.col_i,
                              s.extents, rng.random(s.data.shape[0])) for s in a.sectors])


def test_water192_cut6_parity(gpu_ctx):
    g, a, b = WATER_192.build()
    c_ref, st_ref = oracle.multiply(a, b, WATER_192.eps)
    _no_borderline(c_ref, WATER_192.eps)
    c, st = _gpu_mult(gpu_ctx, a, b, WATER_192.eps)
    c.validate()
    assert_same_pattern(c, c_ref)
    assert rel_frobenius_error(c, c_ref) <= TOL_FP64
    assert st["n_products"] == st_ref["n_products"]
    assert st["n_products_skipped"] == st_ref["n_products_skipped"]
    assert st["flops"] == st_ref["flops"]


@pytest.mark.parametrize("seed", [0, 1, 2, 3, 4, 7])
def test_random_fill_parity(gpu_ctx, seed):
    a = random_fill_matrix(seed)
    b = _with_values(a, seed + 50)
    c_ref, st_ref = oracle.multiply(a, b, 0.0)
    c, st = _gpu_mult(gpu_ctx, a, b, 0.0)
    assert_same_pattern(c, c_ref)
    assert rel_frobenius_error(c, c_ref) <= TOL_FP64


def test_empty_and_tiny(gpu_ctx):
    a = random_fill_matrix(0, n_atoms=0)
    c, st = _gpu_mult(gpu_ctx, a, a, 0.0)
    assert all(s.n_blks == 0 for s in c.sectors)
    a = random_fill_matrix(3, n_atoms=1)
    c_ref, _ = oracle.multiply(a, a, 0.0)
    c, _ = _gpu_mult(gpu_ctx, a, a, 0.0)
    assert_same_pattern(c, c_ref)


def _sector_from_blocks(rb, cb, blocks, rng):
    """One sector (1, 1) whose blocks, given as 1-based (row, col) keys, get random values."""
    rows = sorted(blocks)
    row_p = np.zeros(len(rb) + 1, np.int64)
    col_i, ext, data, pos = [], [], [], 1
    for r, c in rows:
        row_p[r] += 1
        n = int(rb[r - 1]) * int(cb[c - 1])
        col_i.append(c)
        ext.append((pos, pos + n - 1))
        data.append(rng.standard_normal(n))
        pos += n
    row_p = np.concatenate([[0], np.cumsum(row_p[1:])]).astype(np.int64)
    return Sector(1, 1, np.asarray(rb, np.int8), np.asarray(cb, np.int8), row_p, np.asarray(col_i, np.int16),
                  np.asarray(ext, np.int64).reshape(-1, 2), np.concatenate(data) if data else np.zeros(0))


def test_largest_local_index_and_block_size(gpu_ctx):
    """A subset of 32767 atoms (the largest 1-based int16 local column) and
    127-row blocks (the largest int8 block size) on the inner dimension, with a
    zero-size row; 32768 atoms are refused at upload."""
    rng = np.random.default_rng(11)
    nk = 32767
    kb = np.ones(nk, np.int8)
    kb[0], kb[nk // 2], kb[nk - 1] = 2, 0, 127
    ab = np.array([127, 1, 0], np.int8)
    bb = np.array([127, 3], np.int8)
    a = LambMatrix([_sector_from_blocks(ab, kb, {(1, 1): 0, (1, nk // 2 + 1): 0, (1, nk): 0, (2, nk): 0,
                                                (2, 7): 0, (3, 1): 0}, rng)])
    b = LambMatrix([_sector_from_blocks(kb, bb, {(1, 1): 0, (1, 2): 0, (7, 2): 0, (nk // 2 + 1, 1): 0,
                                                (nk, 1): 0, (nk, 2): 0}, rng)])
    a.validate()
    b.validate()
    c_ref, st_ref = oracle.multiply(a, b, 0.0)
    c, st = _gpu_mult(gpu_ctx, a, b, 0.0)
    assert_same_pattern(c, c_ref)
    assert rel_frobenius_error(c, c_ref) <= TOL_FP64
    assert st["flops"] == st_ref["flops"]
    too_wide = LambMatrix([_sector_from_blocks(np.ones(1, np.int8), np.ones(nk + 1, np.int8), {(1, 1): 0}, rng)])
    with pytest.raises(gpu.LambError) as ei:
        gpu_ctx.upload(too_wide)
    assert ei.value.type == 100 and "32767" in str(ei.value)


@pytest.mark.parametrize("flags", [0, gpu.MIXED])
def test_long_stack_of_full_digits(gpu_ctx, flags):
    """One 1 x 1 C block whose stack has 4,200 products over 127-wide inner
    blocks (533,400 inner indices), every entry 0.999: the leading int8 digit
    is 64 everywhere, so one int32 sum over the whole stack would exceed 2^31."""
    rng = np.random.default_rng(3)
    nk = 4200
    kb = np.full(nk, 127, np.int8)
    one = np.ones(1, np.int8)
    a = LambMatrix([_sector_from_blocks(one, kb, {(1, k): 0 for k in range(1, nk + 1)}, rng)])
    b = LambMatrix([_sector_from_blocks(kb, one, {(k, 1): 0 for k in range(1, nk + 1)}, rng)])
    for m in (a, b):
        m.sectors[0].data[:] = 0.999
    c, st = _gpu_mult(gpu_ctx, a, b, 0.0, flags)
    assert st["n_products"] == nk
    assert_same_pattern(c, oracle.multiply(a, b, 0.0)[0])
    if flags & gpu.MIXED:  # against the long-double oracle, like the other mixed tests
        assert rel_frobenius_error(c, oracle.multiply(a, b, 0.0, oracle.LONG_DOUBLE)[0]) <= 1e-11
    else:  # FP64 sums over 533,400 terms drift 1.5e-11 from the exact value; the oracle sums alike
        assert rel_frobenius_error(c, oracle.multiply(a, b, 0.0)[0]) <= TOL_FP64


@pytest.mark.parametrize("seed", [0, 5])
def test_stacks_bit_exact(gpu_ctx, seed):
    g = WaterGeometry(48, None, 6.0, seed=seed)
    a, b = g.matrix(seed + 1), g.matrix(seed + 2)
    _, _, stk_ref = oracle.multiply(a, b, 0.0, want_stacks=True)
    da, db = gpu_ctx.upload(a), gpu_ctx.upload(b)
    dc = gpu_ctx.create_like(da)
    stk = gpu_ctx.stacks(da, db, dc, 0.0)
    assert np.array_equal(stk, stk_ref)
    for m in (dc, db, da):
        m.destroy()


def test_stacks_random_fill_zero_size_blocks(gpu_ctx):
    a = random_fill_matrix(9)
    b = _with_values(a, 3)
    _, _, stk_ref = oracle.multiply(a, b, 0.0, want_stacks=True)
    da, db = gpu_ctx.upload(a), gpu_ctx.upload(b)
    dc = gpu_ctx.create_like(da)
    assert np.array_equal(gpu_ctx.stacks(da, db, dc, 0.0), stk_ref)


def test_product_filter_parity(gpu_ctx):
    g = WaterGeometry(64, None, 7.0, seed=8)
    a, b = g.matrix(3), g.matrix(4)
    # eps near the middle of the product-norm distribution: many products drop
    eps = 2e-3
    c_ref, st_ref, stk_ref = oracle.multiply(a, b, eps, oracle.NO_RESULT_FILTER, want_stacks=True)
    assert st_ref["n_products_skipped"] > 0
    c, st = _gpu_mult(gpu_ctx, a, b, eps, gpu.NO_RESULT_FILTER)
    assert st["n_products_skipped"] == st_ref["n_products_skipped"]
    assert_same_pattern(c, c_ref)
    assert rel_frobenius_error(c, c_ref) <= TOL_FP64
    da, db = gpu_ctx.upload(a), gpu_ctx.upload(b)
    dc = gpu_ctx.create_like(da)
    assert np.array_equal(gpu_ctx.stacks(da, db, dc, eps, gpu.NO_RESULT_FILTER), stk_ref)


def test_result_filter_parity(gpu_ctx):
    g = WaterGeometry(64, None, 7.0, seed=8)
    a, b = g.matrix(5), g.matrix(6)
    eps = 0.3
    c_ref, st_ref = oracle.multiply(a, b, eps, oracle.NO_PRODUCT_FILTER)
    assert st_ref["n_c_blocks_dropped"] > 0
    _no_borderline(c_ref, eps)
    c, st = _gpu_mult(gpu_ctx, a, b, eps, gpu.NO_PRODUCT_FILTER)
    assert st["n_c_blocks_dropped"] == st_ref["n_c_blocks_dropped"]
    assert_same_pattern(c, c_ref)
    assert rel_frobenius_error(c, c_ref) <= TOL_FP64


def test_async_multiply_overlapped_download(gpu_ctx):
    """LAMB_GPU_ASYNC: the multiply returns after queueing its numeric row
    chunks and the device-side result filter; query gives capacities (block
    counts before the filter, exact data lengths) and download copies C chunk
    by chunk, then reports the filtered counts.  Same C as the synchronous call
    and as the oracle."""
    g = WaterGeometry(256, None, 7.0, seed=8)
    a, b = g.matrix(5), g.matrix(6)
    eps = 0.3
    c_ref, st_ref = oracle.multiply(a, b, eps, oracle.NO_PRODUCT_FILTER)
    assert st_ref["n_c_blocks_dropped"] > 0
    _no_borderline(c_ref, eps)
    da, db = gpu_ctx.upload(a), gpu_ctx.upload(b)
    da.set_positions(g.sector_positions(), g.box)
    for rep in range(2):
        dc = gpu_ctx.create_like(da)
        gpu_ctx.multiply(da, db, dc, eps, gpu.NO_PRODUCT_FILTER | gpu.ASYNC)
        caps = dc.sizes()
        c = dc.download()
        assert sum(s.n_blks for s in caps) >= sum(s.n_blks for s in c.sectors)
        assert sum(s.n_blks for s in c.sectors) == sum(s.n_blks for s in c_ref.sectors)
        assert_same_pattern(c, c_ref)
        assert rel_frobenius_error(c, c_ref) <= TOL_FP64
        # the synchronous call on the same handles gives identical values
        gpu_ctx.multiply(da, db, dc, eps, gpu.NO_PRODUCT_FILTER)
        c2 = dc.download()
        assert_same_pattern(c2, c)
        assert np.array_equal(c2.to_dense(), c.to_dense())
        dc.destroy()
    db.destroy()
    da.destroy()


def test_python_lamb_multiply_api(gpu_ctx):
    g = WaterGeometry(32, None, 6.0, seed=1)
    a = g.matrix(1)
    c_ref, _ = oracle.multiply(a, a, 1e-8)
    holder = LambMatrix([], "C")
    out = gpu.lamb_multiply(a, a, holder, eps=1e-8, ctx=gpu_ctx)
    assert out is holder
    assert rel_frobenius_error(holder, c_ref) <= TOL_FP64


def test_errors_are_reported_not_raised_through_abi(gpu_ctx):
    a = WaterGeometry(16, None, 5.0, seed=1).matrix(1)
    b = WaterGeometry(20, None, 5.0, seed=2).matrix(1)
    da, db = gpu_ctx.upload(a), gpu_ctx.upload(b)
    dc = gpu_ctx.create_like(da)
    with pytest.raises(gpu.LambError) as ei:
        gpu_ctx.multiply(da, db, dc, 0.0)
    assert ei.value.type == 100 and ei.value.level == 3
    with pytest.raises(gpu.LambError):
        gpu_ctx.multiply(da, da, da, 0.0)  # C aliases A
    bad = WaterGeometry(16, None, 5.0, seed=1).matrix(1)
    bad.sectors[0].col_i[0] = 32000
    with pytest.raises(gpu.LambError) as ei:
        gpu_ctx.upload(bad)
    assert ei.value.type == 100


def _rows_of(m: LambMatrix, stride: int):
    out = {}
    for s in m.sectors:
        rows = s.block_rows()
        for b in range(s.n_blks):
            r = int(rows[b])
            if r % stride == 0:
                c = int(s.col_i[b]) - 1
                f, l = int(s.extents[b, 0]), int(s.extents[b, 1])
                out[(s.subset_row, s.subset_col, r, c)] = s.data[f - 1:l]
    return out


def test_water6144_cut8_whole_product(gpu_ctx):
    """Full-size workload (6,144 waters, cutoff 8 A, eps 1e-10), every row:
    the GPU C (both filters on) against the oracle's whole product.  The
    oracle computes C without the result filter and applies the filter rule
    while comparing, so the check also shows how close any block norm comes
    to eps (a block within rounding of eps could flip either way)."""
    g, a, b = WATER_6144.build()
    c, st = _gpu_mult(gpu_ctx, a, b, WATER_6144.eps)
    r = oracle.check_product(a, b, WATER_6144.eps, c)
    assert r["min_rel_gap_to_eps"] > 1e-9
    assert r["pattern_mismatches"] == 0
    assert r["rel_frobenius_err"] <= TOL_FP64
    assert st["n_products"] == r["n_products"]
    assert st["n_products_skipped"] == r["n_products_skipped"]
    assert st["flops"] == r["flops"]
    assert st["n_c_blocks"] == sum(s.n_blks for s in c.sectors)


def test_positions_hint_does_not_change_results(gpu_ctx):
    """The work order (Morton from coordinates vs Cuthill-McKee) leaves every C
    block bit-identical; only where the blocks sit in a sector's data store
    follows the work order (the extents say where)."""
    g = WaterGeometry(96, None, 7.0, seed=12)
    a, b = g.matrix(1), g.matrix(2)
    outs = []
    for use_pos in (False, True):
        da, db = gpu_ctx.upload(a), gpu_ctx.upload(b)
        if use_pos:
            da.set_positions(g.sector_positions(), g.box)
        dc = gpu_ctx.create_like(da)
        gpu_ctx.multiply(da, db, dc, 1e-10)
        outs.append(dc.download())
        for m in (dc, db, da):
            m.destroy()
    for s1, s2 in zip(outs[0].sectors, outs[1].sectors):
        assert np.array_equal(s1.row_p, s2.row_p) and np.array_equal(s1.col_i, s2.col_i)
        assert s1.data.size == s2.data.size
        for k in range(s1.n_blks):
            assert np.array_equal(s1.block(k), s2.block(k))


@pytest.mark.parametrize("blk_o,blk_h", [(23, 5), (13, 5), (3, 1), (40, 7)])
def test_block_size_classes(gpu_ctx, blk_o, blk_h):
    """m8n8k4 (<= 8 rows), m16n8k16 slabs (9..32 rows) and the generic path (> 24 columns)."""
    g = WaterGeometry(40, None, 6.0, blk_o=blk_o, blk_h=blk_h, seed=3)
    a, b = g.matrix(1), g.matrix(2)
    c_ref, _ = oracle.multiply(a, b, 0.0)
    c, _ = _gpu_mult(gpu_ctx, a, b, 0.0)
    assert_same_pattern(c, c_ref)
    assert rel_frobenius_error(c, c_ref) <= TOL_FP64


@pytest.mark.parametrize("slices,tol", [(7, 1e-11), (6, 1e-9)])
def test_mixed_mma_sync_precision_error(gpu_ctx, monkeypatch, slices, tol):
    """The mma.sync digit kernel (kept for shapes the tensor-core path does
    not take): same pattern as FP64, error against the long-double oracle
    within the stated bound."""
    monkeypatch.setenv("LAMB_GPU_MIXED_MMA_SYNC", "1")
    monkeypatch.setenv("LAMB_GPU_MIXED_SLICES", str(slices))
    g = WaterGeometry(96, None, 7.0, seed=21)
    a, b = g.matrix(1), g.matrix(2)
    c_ld, _ = oracle.multiply(a, b, 1e-10, oracle.LONG_DOUBLE)
    c, st = _gpu_mult(gpu_ctx, a, b, 1e-10, gpu.MIXED)
    assert st["mixed_slices"] == slices
    assert_same_pattern(c, c_ld)
    err = rel_frobenius_error(c, c_ld)
    assert err <= tol, err


# Tensor-core path (tcgen05 kind::i8 on cluster tiles, six base-254 digits):
# the bound the configuration states for the mixed multiply.
TOL_MIXED = 1e-11


@pytest.mark.parametrize("n_mol,cutoff,blk_o,blk_h", [(96, 7.0, 13, 5), (64, 6.0, 23, 5), (40, 6.0, 40, 7),
                                                      (30, 5.0, 3, 1), (200, 8.0, 13, 5)])
def test_mixed_tensor_core_error(gpu_ctx, n_mol, cutoff, blk_o, blk_h):
    """Same C pattern as the oracle, error against the long-double oracle
    within 1e-11, over block-size classes (1 to 40 rows) and box sizes."""
    g = WaterGeometry(n_mol, None, cutoff, blk_o=blk_o, blk_h=blk_h, seed=21)
    a, b = g.matrix(1), g.matrix(2)
    c_ld, _ = oracle.multiply(a, b, 1e-10, oracle.LONG_DOUBLE)
    _no_borderline(c_ld, 1e-10)
    c, st = _gpu_mult(gpu_ctx, a, b, 1e-10, gpu.MIXED)
    assert st["mixed_slices"] == 6
    c.validate()
    assert_same_pattern(c, c_ld)
    err = rel_frobenius_error(c, c_ld)
    assert err <= TOL_MIXED, err


def test_mixed_tensor_core_dense_tiles(gpu_ctx):
    """A dense product (352 waters, cutoff across the box): every tile couples
    to all 1,056 inner atoms, more entries than the tile kernel holds unless
    consecutive atoms merge into entries of contiguous panel rows.  The
    tensor-core kernel must run (tensor_ops > 0) and match the FP64 product
    within 1e-11."""
    g = WaterGeometry(352, None, 30.0, seed=3)
    a, b = g.matrix(1), g.matrix(2)
    da, db = gpu_ctx.upload(a), gpu_ctx.upload(b)
    da.set_positions(g.sector_positions(), g.box)
    c64, cm = gpu_ctx.create_like(da), gpu_ctx.create_like(da)
    st64 = gpu_ctx.multiply(da, db, c64, 1e-10)
    stm = gpu_ctx.multiply(da, db, cm, 1e-10, gpu.MIXED)
    assert stm["tensor_ops"] > 0
    assert stm["n_c_blocks"] == st64["n_c_blocks"] == (3 * 352) ** 2
    err = gpu_ctx.diff_frobenius(cm, c64) / gpu_ctx.frobenius(c64)
    assert err <= TOL_MIXED, err
    for m in (cm, c64, db, da):
        m.destroy()


def test_mixed_tensor_core_keeps_filtered_pattern(gpu_ctx):
    """With an eps that filters products, C's pattern is the filtered one
    (bit-exact with the oracle); its blocks carry every product, the
    filtered ones included (each below eps), so the values are checked
    against the unfiltered product on that pattern."""
    g = WaterGeometry(48, None, 6.0, seed=8)
    a, b = g.matrix(1), g.matrix(2)
    eps = 1e-2  # about 13 % of the products fall below it
    c_ref, st_ref = oracle.multiply(a, b, eps, oracle.NO_RESULT_FILTER)
    assert st_ref["n_products_skipped"] > 0
    c, st = _gpu_mult(gpu_ctx, a, b, eps, gpu.MIXED | gpu.NO_RESULT_FILTER)
    assert_same_pattern(c, c_ref)
    assert st["n_products"] == st_ref["n_products"] and st["flops"] == st_ref["flops"]
    full, _ = oracle.multiply(a, b, 0.0, oracle.LONG_DOUBLE)
    fv, cv = block_values(full), block_values(c)
    num = sum(float(np.sum((cv[k] - fv[k]) ** 2)) for k in cv)
    den = sum(float(np.sum(fv[k] ** 2)) for k in cv)
    assert np.sqrt(num / den) <= TOL_MIXED


def test_mixed_precision_random_fill(gpu_ctx):
    """Zero-size and 1-3 element blocks, fill 0.7, no filter."""
    a = random_fill_matrix(5)
    b = _with_values(a, 9)
    c_ld, _ = oracle.multiply(a, b, 0.0, oracle.LONG_DOUBLE)
    c, _ = _gpu_mult(gpu_ctx, a, b, 0.0, gpu.MIXED)
    assert_same_pattern(c, c_ld)
    assert rel_frobenius_error(c, c_ld) <= 1e-11
