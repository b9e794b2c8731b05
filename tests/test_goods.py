"""Goods messages (one sector on the wire, src/lamb_goods_X_types.F90:79-268):
the oracle's restatement pinned on a hand-checked message, and the exchange
of messages between two gloo ranks on CPU (the transport the NCCL path uses
between GPUs)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from lamb_b200.matrix import Sector
from oracle import goods as og


def _small_sector():
    # 3 rows (sizes 2, 1, 2) x 4 columns (sizes 1, 2, 1, 2); blocks (0,1), (0,3), (2,0)
    rbs, cbs = np.array([2, 1, 2], np.int8), np.array([1, 2, 1, 2], np.int8)
    row_p = np.array([0, 2, 2, 3], np.int64)
    col_i = np.array([2, 4, 1], np.int16)
    ext = np.array([[1, 4], [5, 8], [9, 10]], np.int64)
    data = np.arange(1.0, 11.0)
    return Sector(1, 2, rbs, cbs, row_p, col_i, ext, data)


def test_oracle_goods_pinned():
    s = _small_sector()
    idx, data = og.pack(s)
    # 12 header words, row_p 4 words (13-16), col_i 6 bytes -> 1 word (17),
    # extents 6 words (18-23), flags 3 bytes -> 1 word (24): 24 words
    assert idx[:12].tolist() == [1, 24, 1, 10, 13, 4, 17, 3, 18, 3, 24, 3]
    assert idx[12:16].tolist() == [0, 2, 2, 3]
    # col_i 2, 4, 1 as little-endian int16 in one word
    assert int(idx[16]) == 2 | (4 << 16) | (1 << 32)
    assert idx[17:23].tolist() == [1, 4, 5, 8, 9, 10]
    assert int(idx[23]) == 0 and idx.shape[0] == 24
    assert np.array_equal(data, s.data)
    t = og.unpack(idx, data, 1, 2, s.row_blk_sizes, s.col_blk_sizes)
    for f in ("row_p", "col_i", "extents", "data"):
        assert np.array_equal(getattr(t, f), getattr(s, f))


def test_oracle_goods_empty_sector():
    s = Sector(2, 1, np.array([3, 3], np.int8), np.array([1], np.int8), np.zeros(3, np.int64),
               np.zeros(0, np.int16), np.zeros((0, 2), np.int64), np.zeros(0))
    idx, data = og.pack(s)
    # row_p 3 words (13-15); col_i, extents and flags still take one word each
    assert idx[:12].tolist() == [1, 18, 1, 0, 13, 3, 16, 0, 17, 0, 18, 0]
    t = og.unpack(idx, data, 2, 1, s.row_blk_sizes, s.col_blk_sizes)
    assert t.n_blks == 0 and np.array_equal(t.row_p, s.row_p)


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from lamb_b200.exchange import recv_goods, send_goods
    from lamb_b200.gen import WaterGeometry
    g = WaterGeometry(24, None, 5.0, seed=2)
    a = g.matrix(1)
    ok = True
    for k, s in enumerate(a.sectors):  # rank 0 sends every sector, rank 1 checks it
        if rank == 0:
            idx, data = og.pack(s)
            send_goods(torch.from_numpy(idx), torch.from_numpy(data), 1)
        else:
            idx, data = recv_goods(0, torch.device("cpu"))
            t = og.unpack(idx.numpy(), data.numpy(), s.subset_row, s.subset_col, s.row_blk_sizes, s.col_blk_sizes)
            ok &= all(np.array_equal(getattr(t, f), getattr(s, f)) for f in ("row_p", "col_i", "extents", "data"))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ok))


def test_goods_exchange_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == {0: True, 1: True}
