"""Block-sparse algebra, McWeeny purification and the masked adjoint on the
GPU against dense numpy references (small systems)."""
import numpy as np
import pytest

from lamb_b200 import gpu
from lamb_b200.gen import WaterGeometry, gapped_hamiltonian

pytestmark = pytest.mark.gpu


def _pair(ctx, seed=1, n=32, cut1=5.0, cut2=6.5):
    g1 = WaterGeometry(n, None, cut1, seed=seed)
    g2 = WaterGeometry(n, None, cut2, seed=seed)  # same atoms, wider pattern
    x, y = g1.matrix(3), g2.matrix(4)
    return x, y, ctx.upload(x), ctx.upload(y)


def test_axpby_union_pattern(gpu_ctx):
    x, y, dx, dy = _pair(gpu_ctx)
    gpu_ctx.axpby(2.5, dx, -0.75, dy)
    ref = 2.5 * x.to_dense() - 0.75 * y.to_dense()
    got = dy.download()
    got.validate()
    assert np.allclose(got.to_dense(), ref, rtol=0, atol=1e-14)


def test_copy_scale_shift_trace(gpu_ctx):
    x, y, dx, dy = _pair(gpu_ctx, seed=2)
    dz = gpu_ctx.create_like(dx)
    gpu_ctx.copy(dx, dz)
    gpu_ctx.scale_shift(dz, -0.5, 0.25)
    ref = -0.5 * x.to_dense() + 0.25 * np.eye(x.to_dense().shape[0])
    assert np.allclose(dz.download().to_dense(), ref, atol=1e-14)
    assert abs(gpu_ctx.trace(dz) - np.trace(ref)) < 1e-10
    assert abs(gpu_ctx.trace_product(dx, dy) - np.trace(x.to_dense() @ y.to_dense())) < 1e-9
    assert abs(gpu_ctx.frobenius(dx) - np.linalg.norm(x.to_dense())) < 1e-10
    assert abs(gpu_ctx.diff_frobenius(dx, dy) - np.linalg.norm(x.to_dense() - y.to_dense())) < 1e-10


def _mcweeny_dense(h, mu, steps):
    d = np.diag(h)
    rad = np.sum(np.abs(h), axis=1) - np.abs(d)
    emin, emax = np.min(d - rad), np.max(d + rad)
    lam = min(1.0 / (emax - mu), 1.0 / (mu - emin))
    p = 0.5 * lam * (mu * np.eye(len(h)) - h) + 0.5 * np.eye(len(h))
    for _ in range(steps):
        p2 = p @ p
        p = 3 * p2 - 2 * p2 @ p
    return p


def test_mcweeny_fp64_matches_dense(gpu_ctx):
    g = WaterGeometry(24, None, 5.0, seed=5)
    h = gapped_hamiltonian(g, 7)
    hd = h.to_dense()
    assert np.allclose(hd, hd.T)
    dh = gpu_ctx.upload(h)
    dp = gpu_ctx.create_like(dh)
    rep = gpu_ctx.purify(dh, dp, mu=0.0, steps=30, fp64_tail=30, eps=0.0)
    ref = _mcweeny_dense(hd, 0.0, 30)
    got = dp.download().to_dense()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-10
    n_occ = np.sum(np.linalg.eigvalsh(hd) < 0)
    assert abs(rep["trace"] - n_occ) < 1e-6
    assert rep["idempotency"] < 1e-8


def test_masked_adjoint_matches_dense(gpu_ctx):
    g = WaterGeometry(28, None, 5.5, seed=9)
    a, b = g.matrix(1), g.matrix(2)
    da_, db_ = gpu_ctx.upload(a), gpu_ctx.upload(b)
    dc_ = gpu_ctx.create_like(da_)
    gpu_ctx.multiply(da_, db_, dc_, 0.0)
    # dC with C's pattern and random values
    dcm = dc_.download()
    rng = np.random.default_rng(0)
    for s in dcm.sectors:
        s.data[:] = rng.standard_normal(s.data.shape[0])
    ddc = gpu_ctx.upload(dcm)
    gA, gB = gpu_ctx.create_like(da_), gpu_ctx.create_like(db_)
    gpu_ctx.adjoint(da_, db_, ddc, gA, gB)
    A, B, dC = a.to_dense(), b.to_dense(), dcm.to_dense()
    mask_a, mask_b = (A != 0), (B != 0)
    ref_a = (dC @ B.T) * mask_a
    ref_b = (A.T @ dC) * mask_b
    got_a, got_b = gA.download(), gB.download()
    got_a.validate(); got_b.validate()
    assert [s.n_blks for s in got_a.sectors] == [s.n_blks for s in a.sectors]
    assert np.linalg.norm(got_a.to_dense() - ref_a) / np.linalg.norm(ref_a) < 1e-13
    assert np.linalg.norm(got_b.to_dense() - ref_b) / np.linalg.norm(ref_b) < 1e-13


def test_mcweeny_mixed_early_steps_match_fp64(gpu_ctx):
    """Purification with int8-slice products in the early steps and an FP64
    tail reaches the all-FP64 density matrix and band energy Tr(P.H).

    Both runs filter products and C blocks at eps = 1e-10, but not the same
    ones: the tensor-core mixed products keep every product (also those below
    eps), the FP64 products skip them, so the two truncated iterations end a
    few 1e-9 apart.  Against an unfiltered FP64 run (eps = 0) the mixed run
    is as close as the filtered FP64 run."""
    g = WaterGeometry(48, None, 5.5, seed=6)
    h = gapped_hamiltonian(g, 3)
    dh = gpu_ctx.upload(h)
    p64, pmx, pex = gpu_ctx.create_like(dh), gpu_ctx.create_like(dh), gpu_ctx.create_like(dh)
    r64 = gpu_ctx.purify(dh, p64, mu=0.0, steps=30, fp64_tail=30, eps=1e-10)
    rmx = gpu_ctx.purify(dh, pmx, mu=0.0, steps=30, fp64_tail=5, eps=1e-10)
    gpu_ctx.purify(dh, pex, mu=0.0, steps=30, fp64_tail=30, eps=0.0)
    assert rmx["steps_mixed"] == 25 and r64["steps_mixed"] == 0
    nrm = gpu_ctx.frobenius(pex)
    rel = gpu_ctx.diff_frobenius(pmx, p64) / nrm
    rel_mx, rel_64 = gpu_ctx.diff_frobenius(pmx, pex) / nrm, gpu_ctx.diff_frobenius(p64, pex) / nrm
    e64, emx = gpu_ctx.trace_product(p64, dh), gpu_ctx.trace_product(pmx, dh)
    assert rel < 5e-9
    assert rel_mx <= max(2 * rel_64, 1e-10), (rel_mx, rel_64)
    assert abs(emx - e64) <= 1e-9 * abs(e64)
    assert abs(rmx["trace"] - r64["trace"]) < 1e-8
    assert rmx["idempotency"] < 1e-8
    for m in (pex, pmx, p64, dh):
        m.destroy()
