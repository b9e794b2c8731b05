"""Goods messages from device matrices (lamb_gpu_goods_pack / _unpack) against
the oracle's restatement of the reference's wire format."""
import numpy as np
import pytest
import torch

from oracle import goods as og
from lamb_b200.gen import WaterGeometry

pytestmark = pytest.mark.gpu


def test_goods_pack_matches_oracle_and_round_trips(gpu_ctx):
    g = WaterGeometry(48, None, 5.5, seed=7)
    a = g.matrix(3)
    da = gpu_ctx.upload(a)
    dl = da.download()  # the device's own layout of every sector (same blocks as a)
    for k, s in enumerate(dl.sectors):
        idx, data = da.goods(k)
        ref_idx, ref_data = og.pack(s)
        assert np.array_equal(idx, ref_idx) and np.array_equal(data, ref_data)
        # device buffers in, device matrix out
        tidx, tdat = da.goods(k, device=True)
        assert torch.equal(tidx.cpu(), torch.from_numpy(ref_idx))
        one = gpu_ctx.goods_unpack(tidx, tdat, s.n_cols, s.row_blk_sizes, s.col_blk_sizes)
        back = one.download().sectors[0]
        assert np.array_equal(back.row_p, s.row_p) and np.array_equal(back.col_i, s.col_i)
        for b in range(s.n_blks):
            assert np.array_equal(back.block(b), s.block(b))
        one.destroy()
    da.destroy()


def test_goods_unpack_rejects_a_damaged_index(gpu_ctx):
    g = WaterGeometry(16, None, 5.0, seed=1)
    da = gpu_ctx.upload(g.matrix(1))
    idx, data = da.goods(0)
    s = da.download().sectors[0]
    bad = idx.copy()
    bad[1] += 1  # index size
    with pytest.raises(Exception):
        gpu_ctx.goods_unpack(bad, data, s.n_cols, s.row_blk_sizes, s.col_blk_sizes)
    da.destroy()
