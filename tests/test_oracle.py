"""The CPU oracle against an independent dense product, and its filter rules.

The reference's own multiply is a stub and ships no golden vectors, so the
oracle is pinned to the mathematical definition (a dense numpy product on the
same inputs) and to the committed fixtures in tests/golden/ (made by
tests/golden/make_golden.py from that dense product)."""
import os

import numpy as np
import pytest

import oracle
from lamb_b200.gen import WaterGeometry, random_fill_matrix
from lamb_b200.matrix import LambMatrix, Sector
from tests.helpers import block_values

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _dense_check(a, b, eps=0.0, flags=oracle.NO_PRODUCT_FILTER | oracle.NO_RESULT_FILTER):
    c, st = oracle.multiply(a, b, eps, flags)
    c.validate()
    ref = a.to_dense() @ b.to_dense()
    got = c.to_dense()
    den = np.linalg.norm(ref)
    err = np.linalg.norm(got - ref) / (den if den > 0 else 1.0)
    return c, st, err


def test_water_box_matches_dense_product():
    g = WaterGeometry(48, None, 5.0, seed=11)
    a = g.matrix(1)
    b = g.matrix(2)
    c, st, err = _dense_check(a, b)
    assert err < 1e-14
    assert st["n_products_skipped"] == 0


@pytest.mark.parametrize("seed", [0, 1, 2, 3, 5, 8])
def test_random_fill_patterns_match_dense(seed):
    a = random_fill_matrix(seed)
    b = random_fill_matrix(seed, n_atoms=None) if False else None
    # B must share A's atoms (same distribution): reuse A's pattern with new values
    b = LambMatrix([Sector(s.subset_row, s.subset_col, s.row_blk_sizes, s.col_blk_sizes, s.row_p, s.col_i,
                           s.extents, np.random.default_rng(seed + 100).random(s.data.shape[0]))
                    for s in a.sectors])
    c, st, err = _dense_check(a, b)
    assert err < 1e-14


def test_empty_matrix():
    a = random_fill_matrix(0, n_atoms=0)
    c, st, err = _dense_check(a, a)
    assert all(s.n_blks == 0 for s in c.sectors)
    assert st["n_products"] == 0


def test_long_double_mode_close():
    g = WaterGeometry(32, None, 5.0, seed=3)
    a = g.matrix(4)
    c1, _ = oracle.multiply(a, a, 0.0)
    c2, _ = oracle.multiply(a, a, 0.0, oracle.LONG_DOUBLE)
    d1, d2 = c1.to_dense(), c2.to_dense()
    assert np.linalg.norm(d1 - d2) / np.linalg.norm(d2) < 1e-14


def test_product_filter_rule():
    g = WaterGeometry(48, None, 6.0, seed=5)
    a = g.matrix(6)
    # pick eps at the median of |A_ik||A_kj| so about half the products drop
    norms = {}
    for k, v in block_values(a).items():
        norms[k] = float(np.sqrt(np.sum(v ** 2)))
    vals = np.sort(np.array(list(norms.values())))
    eps = float(vals[len(vals) // 2] ** 2)
    c, st = oracle.multiply(a, a, eps, oracle.NO_RESULT_FILTER)
    assert st["n_products_skipped"] > 0
    # recompute the kept product count by brute force over the dense block pattern
    c_all, st_all = oracle.multiply(a, a, 0.0)
    assert st["n_products"] + st["n_products_skipped"] == st_all["n_products"]


def test_result_filter_drops_small_blocks():
    g = WaterGeometry(48, None, 6.0, seed=5)
    a = g.matrix(7)
    c0, _ = oracle.multiply(a, a, 0.0)
    bn = sorted(float(np.sqrt(np.sum(v ** 2))) for v in block_values(c0).values())
    eps = bn[len(bn) // 4]
    c, st = oracle.multiply(a, a, eps, oracle.NO_PRODUCT_FILTER)
    assert st["n_c_blocks_dropped"] > 0
    kept = [float(np.sqrt(np.sum(v ** 2))) for v in block_values(c).values()]
    assert min(kept) >= eps
    assert sum(s.n_blks for s in c.sectors) + st["n_c_blocks_dropped"] == sum(s.n_blks for s in c0.sectors)


def test_stacks_canonical_order():
    g = WaterGeometry(24, None, 5.0, seed=2)
    a = g.matrix(1)
    c, st, stk = oracle.multiply(a, a, 0.0, want_stacks=True)
    assert stk.shape == (st["n_products"], 5)
    # every C block (c_blk within its sector) is covered; sector ids in range
    assert stk[:, 0].max() < len(a.sectors) and stk[:, 2].max() < len(a.sectors)


def test_block_norm_fixed_order():
    x = np.random.default_rng(0).standard_normal(169)
    s = 0.0
    for v in x:
        s = np.fma(v, v, s) if hasattr(np, "fma") else s + v * v
    assert abs(oracle.block_norm(x) - np.sqrt(np.sum(x * x))) < 1e-13


@pytest.mark.parametrize("name", ["water8_cut3p5", "random_fill_seed4"])
def test_golden_fixtures(name):
    path = os.path.join(GOLDEN, name + ".npz")
    z = np.load(path)
    a = _from_npz(z, "a")
    b = _from_npz(z, "b")
    c, st = oracle.multiply(a, b, float(z["eps"]), int(z["flags"]))
    d = c.to_dense()
    ref = z["c_dense"]
    assert d.shape == ref.shape
    assert np.linalg.norm(d - ref) <= 1e-14 * max(np.linalg.norm(ref), 1.0)
    pat = np.array(sorted(tuple(k) for k in block_values(c).keys()), dtype=np.int64).reshape(-1, 4)
    assert np.array_equal(pat, z["c_pattern"])


def _from_npz(z, p):
    secs = []
    n = int(z[p + "_n"])
    for i in range(n):
        q = f"{p}{i}_"
        secs.append(Sector(int(z[q + "sr"]), int(z[q + "sc"]), z[q + "rbs"], z[q + "cbs"], z[q + "row_p"],
                           z[q + "col_i"], z[q + "extents"], z[q + "data"]))
    return LambMatrix(secs)


def test_whole_product_check_accepts_itself_and_catches_planted_mistakes():
    """oracle.check_product (used for the whole 6,144-water comparison on the
    GPU): the oracle's own filtered result passes; a changed value, a dropped
    block and an extra block are each caught.  The mistakes are planted in a
    copy of the oracle's result, on the CPU."""
    g = WaterGeometry(40, None, 5.0, seed=21)
    a, b = g.matrix(1), g.matrix(2)
    eps = 0.1
    c, st = oracle.multiply(a, b, eps)
    assert st["n_c_blocks_dropped"] > 0  # the filter rule is exercised
    ok = oracle.check_product(a, b, eps, c)
    assert ok["pattern_mismatches"] == 0 and ok["rel_frobenius_err"] == 0.0
    assert ok["n_products"] == st["n_products"] and ok["min_rel_gap_to_eps"] > 0

    def copy(m):
        return LambMatrix([Sector(s.subset_row, s.subset_col, s.row_blk_sizes.copy(), s.col_blk_sizes.copy(),
                                  s.row_p.copy(), s.col_i.copy(), s.extents.copy(), s.data.copy())
                           for s in m.sectors])
    bad = copy(c)
    bad.sectors[0].data[5] += 1e-6
    r = oracle.check_product(a, b, eps, bad)
    assert r["pattern_mismatches"] == 0 and r["rel_frobenius_err"] > 1e-12
    # drop the first block of sector 0 (row_p shifts down by one after row 0's first block)
    s0 = c.sectors[0]
    bad = copy(c)
    t = bad.sectors[0]
    bad.sectors[0] = Sector(t.subset_row, t.subset_col, t.row_blk_sizes, t.col_blk_sizes,
                            np.maximum(t.row_p - 1, 0), t.col_i[1:], t.extents[1:], t.data)
    assert oracle.check_product(a, b, eps, bad)["pattern_mismatches"] >= 1
    assert s0.n_blks > 1
