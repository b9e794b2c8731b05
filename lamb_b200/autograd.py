"""Differentiation harness over the C ABI (checks only, not a training stack).

* ``BlockSparseMatmul``: torch.autograd.Function for the pattern-fixed
  product C = A.B of block-sparse matrices whose values are torch float64
  vectors in the sector data layout of fixed host patterns.  Backward calls
  lamb_gpu_multiply_adjoint: dA = (dC.B^T) on A's pattern, dB = (A^T.dC) on
  B's pattern.
* ``PurifyTrace``: L(H) = Tr(P_K(H) . H) after K McWeeny steps
  P <- 3P^2 - 2P^3 from P_0 = lam/2 (mu I - H) + I/2, with lam held fixed
  (it comes from Gershgorin bounds of the unperturbed H).  The forward keeps
  every `checkpoint`-th P_k on the device; the backward recomputes the P_k of
  each segment from its checkpoint and walks the steps in reverse with the
  adjoint kernel:
      G_P2 = 3 G, G_P3 = -2 G (G = dL/dP_{k+1})
      P3 = P2.P  ->  G_P2 += (G_P3.P^T)|P2,  G_P += (P2^T.G_P3)|P
      P2 = P.P   ->  G_P  += (G_P2.P^T)|P + (P^T.G_P2)|P
  and finally dL/dH = P_K^T + (-lam/2) G_P0.  Products may use a result
  filter (C blocks below eps dropped; a locally constant mask, so the masked
  adjoint is the exact gradient); the product filter is off.
"""
from __future__ import annotations

from typing import List, Optional

import numpy as np
import torch

from . import gpu as G
from .matrix import LambMatrix, Sector


def _with_values(pattern: LambMatrix, vals: np.ndarray) -> LambMatrix:
    """Copy of `pattern` whose data arrays are taken from one flat vector
    (sectors concatenated in order)."""
    secs, pos = [], 0
    for s in pattern.sectors:
        n = s.data.shape[0]
        secs.append(Sector(s.subset_row, s.subset_col, s.row_blk_sizes, s.col_blk_sizes, s.row_p, s.col_i,
                           s.extents, np.ascontiguousarray(vals[pos:pos + n], dtype=np.float64)))
        pos += n
    return LambMatrix(secs, pattern.name)


def _flat_on(pattern: LambMatrix, m: LambMatrix) -> np.ndarray:
    """Values of m (a matrix whose blocks include pattern's blocks) in
    pattern's data layout; blocks absent from m are zero."""
    out = []
    for ps, ms in zip(pattern.sectors, m.sectors):
        v = np.zeros(ps.data.shape[0])
        rows = ps.block_rows()
        for b in range(ps.n_blks):
            r, c = int(rows[b]) + 1, int(ps.col_i[b])
            mb = ms.get_blk_n(r, c)
            f, l = int(ps.extents[b, 0]), int(ps.extents[b, 1])
            if mb >= 0 and l >= f:
                g0, g1 = int(ms.extents[mb, 0]), int(ms.extents[mb, 1])
                v[f - 1:l] = ms.data[g0 - 1:g1]
        out.append(v)
    return np.concatenate(out) if out else np.zeros(0)


class BlockSparseMatmul(torch.autograd.Function):
    """C = A.B with fixed patterns; values are flat float64 tensors."""

    @staticmethod
    def forward(fctx, a_vals, b_vals, a_pat: LambMatrix, b_pat: LambMatrix, ctx: G.Context):
        A = _with_values(a_pat, a_vals.detach().cpu().numpy())
        B = _with_values(b_pat, b_vals.detach().cpu().numpy())
        da, db = ctx.upload(A), ctx.upload(B)
        dc = ctx.create_like(da)
        ctx.multiply(da, db, dc, 0.0)
        c = dc.download()
        fctx.save_for_backward(a_vals, b_vals)
        fctx.pats = (a_pat, b_pat, c, ctx)
        for m in (dc, db, da):
            m.destroy()
        c_vals = torch.from_numpy(np.concatenate([s.data for s in c.sectors]) if c.sectors else np.zeros(0))
        fctx.c_pat = c
        return c_vals

    @staticmethod
    def backward(fctx, dc_vals):
        a_vals, b_vals = fctx.saved_tensors
        a_pat, b_pat, c_pat, ctx = fctx.pats
        A = _with_values(a_pat, a_vals.detach().cpu().numpy())
        B = _with_values(b_pat, b_vals.detach().cpu().numpy())
        dC = _with_values(c_pat, dc_vals.detach().cpu().numpy())
        da, db, ddc = ctx.upload(A), ctx.upload(B), ctx.upload(dC)
        ga, gb = ctx.create_like(da), ctx.create_like(db)
        ctx.adjoint(da, db, ddc, ga, gb)
        ga_h, gb_h = ga.download(), gb.download()
        for m in (ga, gb, ddc, db, da):
            m.destroy()
        return (torch.from_numpy(_flat_on(a_pat, ga_h)), torch.from_numpy(_flat_on(b_pat, gb_h)), None, None, None)


def gershgorin_lambda(h: LambMatrix, mu: float = 0.0) -> float:
    """lam = min(1/(emax - mu), 1/(mu - emin)) from Gershgorin discs of h's element rows."""
    rs = {m: np.zeros(int(b.astype(np.int64).sum())) for m, b in enumerate(h.subset_blk_sizes(0), start=1)}
    dg = {m: np.zeros_like(v) for m, v in rs.items()}
    for s in h.sectors:
        roff = np.concatenate([[0], np.cumsum(s.row_blk_sizes.astype(np.int64))])
        rows = s.block_rows()
        for b in range(s.n_blks):
            r, c = int(rows[b]), int(s.col_i[b]) - 1
            mm, nn = int(s.row_blk_sizes[r]), int(s.col_blk_sizes[c])
            if mm * nn == 0:
                continue
            f = int(s.extents[b, 0])
            x = s.data[f - 1:f - 1 + mm * nn].reshape(nn, mm).T
            rs[s.subset_row][roff[r]:roff[r] + mm] += np.abs(x).sum(axis=1)
            if s.subset_row == s.subset_col and r == c:
                dg[s.subset_row][roff[r]:roff[r] + mm] += np.diag(x)
    lo = min(float(np.min(dg[m] - (rs[m] - np.abs(dg[m])))) for m in rs if rs[m].size)
    hi = max(float(np.max(dg[m] + (rs[m] - np.abs(dg[m])))) for m in rs if rs[m].size)
    return min(1.0 / (hi - mu), 1.0 / (mu - lo))


class PurifyEngine:
    """Forward and checkpointed reverse pass of L(H) = Tr(P_K H) on device handles."""

    def __init__(self, ctx: G.Context, steps: int, lam: float, mu: float = 0.0, eps: float = 0.0,
                 checkpoint: int = 4):
        self.ctx, self.K, self.lam, self.mu, self.eps, self.cp = ctx, steps, lam, mu, eps, max(1, checkpoint)
        self.flags = G.NO_PRODUCT_FILTER

    def _p0(self, dh: G.DeviceMatrix) -> G.DeviceMatrix:
        p = self.ctx.create_like(dh)
        self.ctx.copy(dh, p)
        self.ctx.scale_shift(p, -0.5 * self.lam, 0.5 * self.lam * self.mu + 0.5)
        return p

    def _step(self, p: G.DeviceMatrix, keep: bool = False):
        c = self.ctx
        p2, p3 = c.create_like(p), c.create_like(p)
        c.multiply(p, p, p2, self.eps, self.flags)
        c.multiply(p2, p, p3, self.eps, self.flags)
        nxt = c.create_like(p)
        c.copy(p2, nxt)
        c.axpby(-2.0, p3, 3.0, nxt)
        if keep:
            return nxt, p2, p3
        p2.destroy()
        p3.destroy()
        return nxt

    def forward(self, dh: G.DeviceMatrix, keep_checkpoints: bool = True):
        c = self.ctx
        p = self._p0(dh)
        cps = {0: p}
        for k in range(self.K):
            nxt = self._step(p)
            if keep_checkpoints and (k + 1) % self.cp == 0 and k + 1 < self.K:
                cps[k + 1] = nxt
            if p is not cps.get(k):
                p.destroy()
            p = nxt
        loss = c.trace_product(p, dh)
        return loss, p, cps

    def backward(self, dh: G.DeviceMatrix, pk: G.DeviceMatrix, cps: dict) -> G.DeviceMatrix:
        """dL/dH as a device matrix on H's pattern union P_K's pattern."""
        c = self.ctx
        # G = dL/dP_K = H^T (H is used as given; its transpose pattern equals its pattern for water boxes)
        g = self._transpose(dh)
        k = self.K
        starts = sorted(cps)
        for s in reversed(starts):
            if s >= k:
                continue
            # recompute P_s .. P_{k-1} from the checkpoint
            seg = [cps[s]]
            for _ in range(s, k - 1):
                seg.append(self._step(seg[-1]))
            for j in range(k - 1, s - 1, -1):
                p = seg[j - s]
                p2 = c.create_like(p)
                c.multiply(p, p, p2, self.eps, self.flags)
                p3 = c.create_like(p)
                c.multiply(p2, p, p3, self.eps, self.flags)
                g3 = c.create_like(p)
                c.copy(g, g3)
                c.scale_shift(g3, -2.0)
                g2 = c.create_like(p)
                c.copy(g, g2)
                c.scale_shift(g2, 3.0)
                # P3 = P2.P
                da2, dp = c.create_like(p), c.create_like(p)
                c.adjoint(p2, p, g3, da2, dp)
                c.axpby(1.0, da2, 1.0, g2)
                # P2 = P.P
                dpa, dpb = c.create_like(p), c.create_like(p)
                c.adjoint(p, p, g2, dpa, dpb)
                c.axpby(1.0, dpa, 1.0, dp)
                c.axpby(1.0, dpb, 1.0, dp)
                for m in (p2, p3, g3, g2, da2, dpa, dpb, g):
                    m.destroy()
                g = dp
            for m in seg[1:]:
                m.destroy()
            k = s
        # P_0 = -lam/2 H + const I
        c.scale_shift(g, -0.5 * self.lam)
        pt = self._transpose(pk)
        c.axpby(1.0, pt, 1.0, g)
        pt.destroy()
        return g

    def _transpose(self, m: G.DeviceMatrix) -> G.DeviceMatrix:
        """Block transpose through the host (test harness only; matrices here are square)."""
        host = m.download()
        secs = []
        # transpose sector (m,n) into (n,m): blocks (i,j) -> (j,i) with transposed data
        by = {(s.subset_row, s.subset_col): s for s in host.sectors}
        for s in host.sectors:
            src = by[(s.subset_col, s.subset_row)]
            rows = src.block_rows()
            entries = []
            for b in range(src.n_blks):
                i, j = int(rows[b]), int(src.col_i[b]) - 1
                mm, nn = int(src.row_blk_sizes[i]), int(src.col_blk_sizes[j])
                f = int(src.extents[b, 0])
                blk = src.data[f - 1:f - 1 + mm * nn].reshape(nn, mm).T  # (mm x nn)
                entries.append((j, i, blk.T))                            # (nn x mm) at (j, i)
            entries.sort(key=lambda e: (e[0], e[1]))
            nr = src.n_cols
            row_p = np.zeros(nr + 1, np.int64)
            for e in entries:
                row_p[e[0] + 1] += 1
            row_p = np.cumsum(row_p)
            col_i = np.array([e[1] + 1 for e in entries], np.int16)
            data = np.concatenate([e[2].T.ravel() for e in entries]) if entries else np.zeros(0)
            sizes = np.array([e[2].size for e in entries], np.int64)
            ends = np.cumsum(sizes)
            ext = np.stack([ends - sizes + 1, ends], axis=1) if entries else np.zeros((0, 2), np.int64)
            secs.append(Sector(s.subset_row, s.subset_col, src.col_blk_sizes.copy(), src.row_blk_sizes.copy(), row_p,
                               col_i, ext.astype(np.int64), data))
        return self.ctx.upload(LambMatrix(secs, "T"))


class PurifyTrace(torch.autograd.Function):
    """L(h_vals) = Tr(P_K H) with H = h_pat carrying the values h_vals."""

    @staticmethod
    def forward(fctx, h_vals, h_pat: LambMatrix, engine: PurifyEngine):
        H = _with_values(h_pat, h_vals.detach().cpu().numpy())
        dh = engine.ctx.upload(H)
        need = bool(fctx.needs_input_grad[0])
        loss, pk, cps = engine.forward(dh, keep_checkpoints=need)
        if need:
            fctx.state = (h_pat, engine, dh, pk, cps)
        else:
            for m in [pk, dh] + list(cps.values()):
                m.destroy()
        return torch.tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(fctx, gl):
        h_pat, engine, dh, pk, cps = fctx.state
        g = engine.backward(dh, pk, cps)
        gh = g.download()
        for m in [g, pk, dh] + list(cps.values()):
            m.destroy()
        return torch.from_numpy(_flat_on(h_pat, gh)) * gl, None, None


def dense_index(m: LambMatrix):
    """(row, col) in m.to_dense() of every value of m's concatenated sector data
    (-1 for values outside any block)."""
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
            pp, qq = np.meshgrid(np.arange(mm), np.arange(nn), indexing="ij")
            r_[f + qq.ravel() * mm + pp.ravel()] = rb[s.subset_row - 1] + ro[s.subset_row - 1][r] + pp.ravel()
            c_[f + qq.ravel() * mm + pp.ravel()] = cb[s.subset_col - 1] + co[s.subset_col - 1][c] + qq.ravel()
        idx_r.append(r_)
        idx_c.append(c_)
    return np.concatenate(idx_r), np.concatenate(idx_c)


def dense_purify_loss(h_vals: torch.Tensor, ri, ci, n: int, lam: float, steps: int, mu: float = 0.0) -> torch.Tensor:
    """The same L(H) = Tr(P_K H) with dense torch matrices (FP64 reference gradient)."""
    dev = h_vals.device
    eye = torch.eye(n, dtype=torch.float64, device=dev)
    H = torch.zeros(n, n, dtype=torch.float64, device=dev).index_put(
        (torch.as_tensor(ri, device=dev), torch.as_tensor(ci, device=dev)), h_vals)
    P = 0.5 * lam * (mu * eye - H) + 0.5 * eye
    for _ in range(steps):
        P2 = P @ P
        P = 3 * P2 - 2 * P2 @ P
    return torch.trace(P @ H)
