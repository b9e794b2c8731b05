"""Differentiation through the C ABI: the block-sparse matmul Function and
Tr(P_K H) through K McWeeny steps with checkpointed recomputation, against
dense torch autograd (FP64 reference gradient) and central differences."""
import numpy as np
import pytest
import torch

from lamb_b200 import autograd as AG
from lamb_b200.gen import WaterGeometry, gapped_hamiltonian

pytestmark = pytest.mark.gpu


def _flat(m):
    return torch.from_numpy(np.concatenate([s.data for s in m.sectors]))


def _dense_index(m):
    """For every value of m's flat vector, its (row, col) in m.to_dense()."""
    rbs, cbs = m.subset_blk_sizes(0), m.subset_blk_sizes(1)
    ro = [np.concatenate([[0], np.cumsum(b.astype(np.int64))]) for b in rbs]
    co = [np.concatenate([[0], np.cumsum(b.astype(np.int64))]) for b in cbs]
    rb = np.concatenate([[0], np.cumsum([o[-1] for o in ro])])
    cb = np.concatenate([[0], np.cumsum([o[-1] for o in co])])
    idx_r, idx_c = [], []
    for s in m.sectors:
        r_ = np.full(s.data.shape[0], -1, np.int64)
        c_ = np.full(s.data.shape[0], -1, np.int64)
        rows = s.block_rows()
        for b in range(s.n_blks):
            r, c = int(rows[b]), int(s.col_i[b]) - 1
            mm, nn = int(s.row_blk_sizes[r]), int(s.col_blk_sizes[c])
            f = int(s.extents[b, 0]) - 1
            for q in range(nn):
                for p in range(mm):
                    r_[f + q * mm + p] = rb[s.subset_row - 1] + ro[s.subset_row - 1][r] + p
                    c_[f + q * mm + p] = cb[s.subset_col - 1] + co[s.subset_col - 1][c] + q
        idx_r.append(r_)
        idx_c.append(c_)
    return np.concatenate(idx_r), np.concatenate(idx_c)


def test_block_sparse_matmul_function(gpu_ctx):
    g = WaterGeometry(20, None, 5.0, seed=4)
    a, b = g.matrix(1), g.matrix(2)
    av, bv = _flat(a).requires_grad_(True), _flat(b).requires_grad_(True)
    cv = AG.BlockSparseMatmul.apply(av, bv, a, b, gpu_ctx)
    w = torch.randn(cv.shape[0], dtype=torch.float64, generator=torch.Generator().manual_seed(0))
    (cv * w).sum().backward()
    # dense reference: C = A.B, loss = sum(W * C) over C's pattern
    ra, ca = _dense_index(a)
    rb, cb = _dense_index(b)
    n = a.to_dense().shape[0]
    Ad = torch.zeros(n, n, dtype=torch.float64)
    Bd = torch.zeros(n, n, dtype=torch.float64)
    av2, bv2 = _flat(a).requires_grad_(True), _flat(b).requires_grad_(True)
    Ad = Ad.index_put((torch.from_numpy(ra), torch.from_numpy(ca)), av2)
    Bd = Bd.index_put((torch.from_numpy(rb), torch.from_numpy(cb)), bv2)
    Cd = Ad @ Bd
    # place W on C's pattern through the layout the Function returned (its saved C)
    c_host = AG._with_values(cv.grad_fn.c_pat, w.numpy())
    rc, cc = _dense_index(c_host)
    Wd = torch.zeros(n, n, dtype=torch.float64).index_put((torch.from_numpy(rc), torch.from_numpy(cc)), w)
    ref_loss = (Cd * Wd).sum()
    ref_loss.backward()
    assert torch.allclose(av.grad, av2.grad, rtol=1e-12, atol=1e-12)
    assert torch.allclose(bv.grad, bv2.grad, rtol=1e-12, atol=1e-12)


def _dense_purify_loss(hv, ra, ca, n, lam, K, mu=0.0):
    H = torch.zeros(n, n, dtype=torch.float64).index_put((torch.from_numpy(ra), torch.from_numpy(ca)), hv)
    P = 0.5 * lam * (mu * torch.eye(n, dtype=torch.float64) - H) + 0.5 * torch.eye(n, dtype=torch.float64)
    for _ in range(K):
        P2 = P @ P
        P = 3 * P2 - 2 * P2 @ P
    return torch.trace(P @ H)


def test_purification_gradient_checkpointed(gpu_ctx):
    g = WaterGeometry(16, None, 4.5, seed=6)
    h = gapped_hamiltonian(g, 3, coupling=0.05)
    K, cp = 6, 2
    lam = AG.gershgorin_lambda(h)
    eng = AG.PurifyEngine(gpu_ctx, K, lam, checkpoint=cp)
    hv = _flat(h).requires_grad_(True)
    loss = AG.PurifyTrace.apply(hv, h, eng)
    loss.backward()
    ra, ca = _dense_index(h)
    n = h.to_dense().shape[0]
    hv2 = _flat(h).requires_grad_(True)
    ref = _dense_purify_loss(hv2, ra, ca, n, lam, K)
    ref.backward()
    assert abs(loss.item() - ref.item()) <= 1e-10 * abs(ref.item())
    err = torch.linalg.norm(hv.grad - hv2.grad) / torch.linalg.norm(hv2.grad)
    assert err.item() <= 1e-10
    # central differences, step 1e-6.  FD resolves a derivative only down to
    # its roundoff floor ~ eps_mach |L| / h, so: relative 1e-6 on entries whose
    # gradient is well above that floor, and the floor itself on uniformly
    # random entries.
    h_fd = 1e-6
    floor = 8 * np.finfo(np.float64).eps * abs(loss.item()) / h_fd
    rng = np.random.default_rng(1)
    g = hv.grad.numpy()
    big = np.nonzero(np.abs(g) >= floor / 1e-6)[0]
    picks = [(i, True) for i in rng.choice(big, min(12, len(big)), replace=False)]
    picks += [(i, False) for i in rng.choice(hv.shape[0], 12, replace=False)]
    assert len(picks) >= 18
    for i, rel in picks:
        e = torch.zeros_like(hv)
        e[i] = h_fd
        with torch.no_grad():
            lp = AG.PurifyTrace.apply(_flat(h) + e, h, eng).item()
            lm = AG.PurifyTrace.apply(_flat(h) - e, h, eng).item()
        fd = (lp - lm) / (2 * h_fd)
        if rel:
            assert abs(fd - g[i]) <= 1e-6 * abs(g[i]), (i, fd, g[i])
        else:
            assert abs(fd - g[i]) <= floor + 1e-6 * abs(g[i]), (i, fd, g[i])
