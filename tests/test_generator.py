"""Water-box generator: LAMB sector layout invariants and determinism."""
import numpy as np

from lamb_b200.gen import WATER_192, WaterGeometry, box_side, random_fill_matrix


def test_sector_layout_invariants():
    g = WaterGeometry(64, None, 6.0, seed=3)
    a = g.matrix(1)
    a.validate()
    assert [(s.subset_row, s.subset_col) for s in a.sectors] == [(1, 1), (1, 2), (2, 1), (2, 2)]
    for s in a.sectors:
        # blocks contiguous in row-major order, 1-based inclusive extents
        assert s.extents[0, 0] == 1 if s.n_blks else True
        assert np.all(s.extents[1:, 0] == s.extents[:-1, 1] + 1)
        assert s.extents[-1, 1] == s.data.shape[0] if s.n_blks else True


def test_subset_rule_float32():
    g = WaterGeometry(200, None, 6.0, seed=4)
    x = g.positions[:, 0].astype(np.float32)
    mult = np.float32(2.0) / np.float32(g.box)
    sub = (x * mult).astype(np.int32) % 2 + 1
    assert np.array_equal(sub, g.subset)
    for s in (1, 2):
        idx = np.nonzero(g.subset == s)[0]
        assert np.array_equal(g.local[idx], np.arange(len(idx)))


def test_geometry_constraints():
    g = WaterGeometry(192, 17.9, 6.0, seed=0)
    L = g.box
    O = g.positions[0::3]
    H1, H2 = g.positions[1::3], g.positions[2::3]
    mi = lambda d: d - L * np.round(d / L)
    d1 = np.linalg.norm(mi(H1 - O), axis=1)
    d2 = np.linalg.norm(mi(H2 - O), axis=1)
    assert np.allclose(d1, 0.96) and np.allclose(d2, 0.96)
    ang = np.degrees(np.arccos(np.sum(mi(H1 - O) * mi(H2 - O), axis=1) / (d1 * d2)))
    assert np.allclose(ang, 104.5)
    dd = mi(O[:, None, :] - O[None, :, :])
    r = np.linalg.norm(dd, axis=2) + np.eye(len(O)) * 100
    assert r.min() >= 2.5


def test_pattern_is_cutoff_and_values_decay():
    g = WaterGeometry(40, None, 5.0, seed=6)
    a = g.matrix(2)
    d = a.to_dense()
    assert np.allclose(d.shape, (40 * 23, 40 * 23))
    total = sum(s.n_blks for s in a.sectors)
    assert total == g.n_pairs


def test_deterministic_and_symmetric():
    g1 = WaterGeometry(30, None, 5.0, seed=9)
    g2 = WaterGeometry(30, None, 5.0, seed=9)
    assert np.array_equal(g1.positions, g2.positions)
    a1, a2 = g1.matrix(5), g2.matrix(5)
    for s1, s2 in zip(a1.sectors, a2.sectors):
        assert np.array_equal(s1.data, s2.data)
    h = g1.matrix(7, symmetric=True).to_dense()
    assert np.array_equal(h, h.T)
    x = g1.matrix(7).to_dense()
    # diagonal blocks symmetric with +1 on the diagonal
    assert not np.array_equal(x, x.T)


def test_named_workload_sizes():
    assert abs(box_side(192) - 17.9) < 0.05
    assert abs(box_side(6144) - 56.8) < 0.1
    g, a, b = WATER_192.build()
    assert g.n_atoms == 576 and a is b
    assert sum(int(s.row_blk_sizes.astype(np.int64).sum()) for s in a.sectors if s.subset_col == 1) == 4416


def test_random_fill_has_zero_size_blocks():
    a = random_fill_matrix(4)
    a.validate()
    sizes = np.concatenate([s.row_blk_sizes for s in a.sectors])
    assert (sizes == 0).any()
