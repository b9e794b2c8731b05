"""Sector exchange between ranks: goods messages over torch.distributed.

The reference moves remote sectors with its market/window layer
(lamb_market_X_*, src/lamb_market_X_methods.F90:94-415; service_schedule,
src/lamb_multiplication.F90:227-320): a rank requests sector (m, k) of A or
(k, n) of B from its owner and receives it as goods (an int64 index and a
float64 data array, lamb_goods_X_types.F90:79-268).  Here one rank per GPU
sends the two arrays point to point: with the NCCL backend straight from one
GPU's memory to another's over NVLink (packed on the device by
lamb_gpu_goods_pack, unpacked by lamb_gpu_goods_unpack), with gloo through
host tensors.  A message is preceded by its two lengths.
"""
from __future__ import annotations

from typing import Optional, Tuple

import torch
import torch.distributed as dist


def send_goods(index: torch.Tensor, data: torch.Tensor, dst: int, group: Optional[dist.ProcessGroup] = None) -> None:
    sizes = torch.tensor([index.numel(), data.numel()], dtype=torch.int64, device=index.device)
    dist.send(sizes, dst, group=group)
    dist.send(index.contiguous(), dst, group=group)
    if data.numel():
        dist.send(data.contiguous(), dst, group=group)


def recv_goods(src: int, device: torch.device, group: Optional[dist.ProcessGroup] = None
               ) -> Tuple[torch.Tensor, torch.Tensor]:
    sizes = torch.empty(2, dtype=torch.int64, device=device)
    dist.recv(sizes, src, group=group)
    n_idx, n_data = int(sizes[0]), int(sizes[1])
    index = torch.empty(n_idx, dtype=torch.int64, device=device)
    dist.recv(index, src, group=group)
    data = torch.empty(n_data, dtype=torch.float64, device=device)
    if n_data:
        dist.recv(data, src, group=group)
    return index, data


def send_sector(matrix, sector: int, dst: int, group: Optional[dist.ProcessGroup] = None) -> None:
    """Packs sector `sector` of a device matrix on its GPU and sends it (NCCL)."""
    index, data = matrix.goods(sector, device=True)
    send_goods(index, data, dst, group)


def recv_sector(ctx, src: int, n_cols: int, row_blk_sizes, col_blk_sizes,
                group: Optional[dist.ProcessGroup] = None):
    """Receives a sector into this rank's GPU and returns it as a device matrix."""
    index, data = recv_goods(src, torch.device("cuda", ctx.device), group)
    return ctx.goods_unpack(index, data, n_cols, row_blk_sizes, col_blk_sizes)
