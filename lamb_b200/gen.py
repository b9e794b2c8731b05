"""Synthetic inputs: water boxes in LAMB's single-rank sector layout.

Thin ctypes wrapper of liblamb_gen.so (include/lamb_gen.h) plus the named
workloads used by tests and the benchmark.  The geometry and value rules are
documented in include/lamb_gen.h.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
from typing import Optional

import numpy as np

from . import _lib
from .abi import CSector, sector_from_c
from .matrix import LambMatrix

MOLECULES_PER_A3 = 0.0335  # 192 / 17.9^3 and 6144 / 56.8^3


def box_side(n_mol: int) -> float:
    """Side of a cubic box holding n_mol waters at 0.0335 molecules per cubic angstrom."""
    return (n_mol / MOLECULES_PER_A3) ** (1.0 / 3.0)


def _gen():
    lib = _lib.load("liblamb_gen.so")
    if not getattr(lib, "_typed", False):
        lib.lamb_gen_water_geometry.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                                C.c_uint64, C.c_double, C.c_int32, C.POINTER(C.c_void_p)]
        lib.lamb_gen_geom_free.argtypes = [C.c_void_p]
        lib.lamb_gen_geom_n_atoms.argtypes = [C.c_void_p]
        lib.lamb_gen_geom_n_pairs.argtypes = [C.c_void_p]
        lib.lamb_gen_geom_n_pairs.restype = C.c_int64
        lib.lamb_gen_geom_atoms.argtypes = [C.c_void_p] + [C.c_void_p] * 4
        lib.lamb_gen_water_matrix.argtypes = [C.c_void_p, C.c_uint64, C.c_double, C.c_int32, C.POINTER(C.c_void_p)]
        lib.lamb_gen_matrix_free.argtypes = [C.c_void_p]
        lib.lamb_gen_matrix_n_sectors.argtypes = [C.c_void_p]
        lib.lamb_gen_matrix_sector.argtypes = [C.c_void_p, C.c_int32, C.POINTER(CSector)]
        lib.lamb_gen_last_error.restype = C.c_char_p
        lib._typed = True
    return lib


class WaterGeometry:
    """Water box geometry with its neighbour pattern; owns the C object."""

    def __init__(self, n_mol: int, box: Optional[float] = None, cutoff: float = 6.0, blk_o: int = 13,
                 blk_h: int = 5, seed: int = 0, min_oo: float = 2.5, n_x_cubes: int = 2):
        self.n_mol, self.box = n_mol, float(box if box is not None else box_side(n_mol))
        self.cutoff, self.blk_o, self.blk_h, self.seed = cutoff, blk_o, blk_h, seed
        lib = _gen()
        h = C.c_void_p()
        rc = lib.lamb_gen_water_geometry(n_mol, self.box, cutoff, blk_o, blk_h, seed, min_oo, n_x_cubes,
                                         C.byref(h))
        if rc != 0:
            raise RuntimeError(lib.lamb_gen_last_error().decode())
        self._h = h
        self.n_atoms = lib.lamb_gen_geom_n_atoms(h)
        self.n_pairs = lib.lamb_gen_geom_n_pairs(h)
        self.positions = np.zeros((self.n_atoms, 3))
        self.blk = np.zeros(self.n_atoms, np.int8)
        self.subset = np.zeros(self.n_atoms, np.int32)
        self.local = np.zeros(self.n_atoms, np.int32)
        lib.lamb_gen_geom_atoms(h, self.positions.ctypes.data, self.blk.ctypes.data, self.subset.ctypes.data,
                                self.local.ctypes.data)

    def sector_positions(self) -> np.ndarray:
        """Atom coordinates in sector order (subset 1's atoms first, local order)."""
        counts = np.bincount(self.subset, minlength=int(self.subset.max(initial=0)) + 1)[1:]
        base = np.concatenate([[0], np.cumsum(counts)])
        out = np.zeros((self.n_atoms, 3), np.float32)
        out[base[self.subset - 1] + self.local] = self.positions
        return out

    def matrix(self, seed: int, decay: float = 1.5, symmetric: bool = False, name: str = "matrix") -> LambMatrix:
        lib = _gen()
        m = C.c_void_p()
        rc = lib.lamb_gen_water_matrix(self._h, seed, decay, int(symmetric), C.byref(m))
        if rc != 0:
            raise RuntimeError(lib.lamb_gen_last_error().decode())
        try:
            secs = []
            for s in range(lib.lamb_gen_matrix_n_sectors(m)):
                cs = CSector()
                if lib.lamb_gen_matrix_sector(m, s, C.byref(cs)) != 0:
                    raise RuntimeError(lib.lamb_gen_last_error().decode())
                secs.append(sector_from_c(cs, copy=True))
        finally:
            lib.lamb_gen_matrix_free(m)
        return LambMatrix(secs, name)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _gen().lamb_gen_geom_free(h)
            except Exception:
                pass
            self._h = None


@dataclasses.dataclass(frozen=True)
class WaterWorkload:
    """One multiply C = A.B on a water box."""
    name: str
    n_mol: int
    box: float
    cutoff: float
    eps: float
    geom_seed: int
    seed_a: int
    seed_b: int
    blk_o: int = 13
    blk_h: int = 5

    def build(self):
        g = WaterGeometry(self.n_mol, self.box, self.cutoff, self.blk_o, self.blk_h, seed=self.geom_seed)
        a = g.matrix(self.seed_a, name="A")
        b = a if self.seed_b == self.seed_a else g.matrix(self.seed_b, name="B")
        return g, a, b


# 192 waters in a 17.9 A box, cutoff 6 A, A = B from seed 0, eps 1e-8.
WATER_192 = WaterWorkload("water192_cut6", 192, 17.9, 6.0, 1e-8, 0, 0, 0)
# 6144 waters in a 56.8 A box, cutoff 8 A, A and B from seeds 1 and 2, eps 1e-10.
WATER_6144 = WaterWorkload("water6144_cut8", 6144, 56.8, 8.0, 1e-10, 1, 1, 2)
# 1536 waters at the same density, cutoff 7 A, seed 4 (the purification-adjoint geometry).
WATER_1536 = WaterWorkload("water1536_cut7", 1536, box_side(1536), 7.0, 1e-10, 4, 4, 5)
# A profiling size of the same family: small enough for multi-pass ncu
# captures (a few GB on the device), larger than L2.
WATER_768 = WaterWorkload("water768_cut7", 768, box_side(768), 7.0, 1e-10, 11, 11, 12)


def batch_instances(n: int = 64, seed: int = 3, mol_range=(96, 1536), cut_range=(5.0, 9.0)):
    """Uneven independent instances: molecule counts log-uniform in mol_range,
    cutoffs uniform in cut_range, O basis 23 for half of them and 13 for the rest."""
    rng = np.random.default_rng(seed)
    lo, hi = math.log(mol_range[0]), math.log(mol_range[1])
    out = []
    for b in range(n):
        nm = int(round(math.exp(rng.uniform(lo, hi))))
        cut = float(rng.uniform(*cut_range))
        blk_o = 23 if b % 2 == 0 else 13
        out.append(WaterWorkload(f"batch{b}", nm, box_side(nm), cut, 1e-10, 1000 + b, 2000 + b, 3000 + b,
                                 blk_o=blk_o))
    return out


def random_fill_matrix(seed: int, n_atoms: Optional[int] = None, max_atoms: int = 100, fill: float = 0.7,
                       max_blk: int = 4, n_x_cubes: int = 2, name: str = "random") -> LambMatrix:
    """Random sparse matrix with the semantics of the reference's test fixture
    (lamb_matrix_X_create_random / fill_sector, src/lamb_matrix_X_tests.F90:89-250):
    n_atoms = int(U*max_atoms), block sizes int(U*4) in {0..3} (zero-size
    blocks included), random positions in the unit box split into subsets by
    the float32 cube rule, each (i,j) present with probability `fill`,
    values U[0,1), blocks stored contiguously in row-major (i,j) order.
    Extents are 1-based inclusive (the reference's fill_sector writes a
    0-based start there, inconsistent with its 1-based data stores)."""
    rng = np.random.default_rng(seed)
    if n_atoms is None:
        n_atoms = int(rng.random() * max_atoms)
    blk = (rng.random(n_atoms) * max_blk).astype(np.int8)
    x = rng.random(n_atoms).astype(np.float32)
    mult = np.float32(n_x_cubes) / np.float32(1.0)
    sub = ((x * mult).astype(np.int32) % n_x_cubes) + 1
    atoms = [np.nonzero(sub == s + 1)[0] for s in range(n_x_cubes)]
    secs = []
    from .matrix import Sector
    for m in range(n_x_cubes):
        for n in range(n_x_cubes):
            ra, ca = atoms[m], atoms[n]
            rbs, cbs = blk[ra].copy(), blk[ca].copy()
            present = rng.random((len(ra), len(ca))) < fill
            rows, cols = np.nonzero(present)
            sizes = rbs[rows].astype(np.int64) * cbs[cols].astype(np.int64)
            ends = np.cumsum(sizes)
            starts = ends - sizes
            row_p = np.zeros(len(ra) + 1, np.int64)
            np.add.at(row_p, rows + 1, 1)
            row_p = np.cumsum(row_p)
            data = rng.random(int(ends[-1]) if len(ends) else 0)
            secs.append(Sector(m + 1, n + 1, rbs, cbs, row_p, (cols + 1).astype(np.int16),
                               np.stack([starts + 1, ends], axis=1).astype(np.int64).reshape(-1, 2), data))
    return LambMatrix(secs, name)


def gapped_hamiltonian(geom: "WaterGeometry", seed: int, gap: float = 0.2, occ_fraction: float = 0.3,
                       decay: float = 1.5, coupling: float = 1.0) -> LambMatrix:
    """Symmetric block-sparse H on the geometry's pattern with a spectral gap
    of at least `gap` around mu = 0.

    H = s*V + D: V is the symmetric water matrix (entries u*exp(-r/decay),
    diagonal blocks (X+X^T)/2 + I), s = `coupling`; D is diagonal with
    d_p = -(gap/2 + R_p) for the first round(occ_fraction*b) functions of
    every atom (occupied) and +(gap/2 + R_p) for the rest,
    R_p = sum_q |s*V_pq| (row p of s*V).  Every Gershgorin disc of H then lies
    outside (-gap/2, gap/2)."""
    v = geom.matrix(seed, decay, symmetric=True, name="H")
    if coupling != 1.0:
        for s_ in v.sectors:
            s_.data *= coupling
    # row sums of |V| per element row, per subset
    sub_sizes = v.subset_blk_sizes(0)
    offs = [np.concatenate([[0], np.cumsum(b.astype(np.int64))]) for b in sub_sizes]
    rsum = [np.zeros(int(o[-1])) for o in offs]
    for s in v.sectors:
        rows = s.block_rows()
        for blk in range(s.n_blks):
            r, c = int(rows[blk]), int(s.col_i[blk]) - 1
            m, n = int(s.row_blk_sizes[r]), int(s.col_blk_sizes[c])
            f = int(s.extents[blk, 0])
            x = s.data[f - 1:f - 1 + m * n].reshape(n, m).T
            rsum[s.subset_row - 1][offs[s.subset_row - 1][r]:offs[s.subset_row - 1][r] + m] += np.abs(x).sum(axis=1)
    for s in v.sectors:
        if s.subset_row != s.subset_col:
            continue
        rows = s.block_rows()
        o = offs[s.subset_row - 1]
        rs = rsum[s.subset_row - 1]
        for blk in range(s.n_blks):
            r, c = int(rows[blk]), int(s.col_i[blk]) - 1
            if r != c:
                continue
            m = int(s.row_blk_sizes[r])
            f = int(s.extents[blk, 0])
            n_occ = int(round(occ_fraction * m))
            for p in range(m):
                sign = -1.0 if p < n_occ else 1.0
                s.data[f - 1 + p * m + p] += sign * (0.5 * gap + rs[o[r] + p])
    return v
