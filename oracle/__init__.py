"""CPU oracle for LAMB's sector multiply -- TEST INFRASTRUCTURE ONLY.

Only the tests, the smoke check and the benchmark's CPU-baseline leg use this
package, as the checker.  PARITY UNPINNED: the reference's sector_multiply is
a stub (src/lamb_multiplication.F90:206-225) and ships no golden vectors, so
the C restatement in lamb_oracle.c (rules in lamb_oracle.h) is pinned against
an independent dense product in the tests instead.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from lamb_b200.abi import CSector, sector_from_c, sector_to_c
from lamb_b200.matrix import LambMatrix

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liblamb_oracle.so")
LONG_DOUBLE = 0x100
NO_STACKS = 0x200
NO_PRODUCT_FILTER = 2
NO_RESULT_FILTER = 4

_lib = None


def build() -> str:
    subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.lamb_oracle_multiply.argtypes = [C.POINTER(CSector), C.c_int32, C.POINTER(CSector), C.c_int32, C.c_double,
                                           C.c_uint32, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
        L.lamb_oracle_n_sectors.argtypes = [C.c_void_p]
        L.lamb_oracle_sector.argtypes = [C.c_void_p, C.c_int32, C.POINTER(CSector)]
        L.lamb_oracle_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                        C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        L.lamb_oracle_stacks.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]
        L.lamb_oracle_free.argtypes = [C.c_void_p]
        L.lamb_oracle_compare.argtypes = [C.c_void_p, C.POINTER(CSector), C.c_int32, C.c_double, C.c_int32,
                                          C.POINTER(C.c_int64), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double)]
        L.lamb_oracle_block_norm.argtypes = [C.c_void_p, C.c_int64]
        L.lamb_oracle_block_norm.restype = C.c_double
        _lib = L
    return _lib


def _arr(m: LambMatrix):
    arr = (CSector * len(m.sectors))(*[sector_to_c(s) for s in m.sectors])
    return arr


def multiply(a: LambMatrix, b: LambMatrix, eps: float = 0.0, flags: int = 0, threads: int = 0,
             row_stride: int = 1, want_stacks: bool = False):
    """C = A.B on the CPU.  Returns (C, stats dict[, stacks int64 (n,5)])."""
    L = lib()
    ca, cb = _arr(a), _arr(b)
    h = C.c_void_p()
    rc = L.lamb_oracle_multiply(ca, len(a.sectors), cb, len(b.sectors), eps, flags, threads, row_stride, C.byref(h))
    if rc != 0:
        raise RuntimeError(f"oracle multiply failed ({rc})")
    try:
        secs = []
        for s in range(L.lamb_oracle_n_sectors(h)):
            cs = CSector()
            L.lamb_oracle_sector(h, s, C.byref(cs))
            secs.append(sector_from_c(cs, copy=True))
        npr, nsk, ndr = C.c_int64(), C.c_int64(), C.c_int64()
        fl = C.c_double()
        L.lamb_oracle_stats(h, C.byref(npr), C.byref(nsk), C.byref(fl), C.byref(ndr))
        stats = {"n_products": npr.value, "n_products_skipped": nsk.value, "flops": fl.value,
                 "n_c_blocks_dropped": ndr.value}
        out = [LambMatrix(secs, "C"), stats]
        if want_stacks:
            n = C.c_int64(0)
            if L.lamb_oracle_stacks(h, None, C.byref(n)) != 0:
                raise RuntimeError("oracle stacks unavailable")
            ent = np.zeros((max(n.value, 1), 5), np.int64)
            L.lamb_oracle_stacks(h, ent.ctypes.data, C.byref(n))
            out.append(ent[:n.value])
        return tuple(out)
    finally:
        L.lamb_oracle_free(h)


def check_product(a: LambMatrix, b: LambMatrix, eps: float, got: LambMatrix, flags: int = 0,
                  threads: int = 0) -> dict:
    """Whole-product check of a device result `got` (computed with the result
    filter at eps) without copying the oracle's C into Python: the oracle
    computes C = A.B without the result filter, then counts pattern
    mismatches under the filter rule and the relative Frobenius error over the
    kept blocks (lamb_oracle_compare)."""
    L = lib()
    ca, cb, cg = _arr(a), _arr(b), _arr(got)
    h = C.c_void_p()
    rc = L.lamb_oracle_multiply(ca, len(a.sectors), cb, len(b.sectors), eps, flags | NO_RESULT_FILTER | NO_STACKS,
                                threads, 1, C.byref(h))
    if rc != 0:
        raise RuntimeError(f"oracle multiply failed ({rc})")
    try:
        mis, num, den, gap = C.c_int64(), C.c_double(), C.c_double(), C.c_double()
        if L.lamb_oracle_compare(h, cg, len(got.sectors), eps, threads, C.byref(mis), C.byref(num), C.byref(den),
                                 C.byref(gap)) != 0:
            raise RuntimeError("oracle compare failed")
        npr, nsk, ndr = C.c_int64(), C.c_int64(), C.c_int64()
        fl = C.c_double()
        L.lamb_oracle_stats(h, C.byref(npr), C.byref(nsk), C.byref(fl), C.byref(ndr))
        rel = float(np.sqrt(num.value / den.value)) if den.value > 0 else float(np.sqrt(num.value))
        return {"pattern_mismatches": mis.value, "rel_frobenius_err": rel, "min_rel_gap_to_eps": gap.value,
                "n_products": npr.value, "n_products_skipped": nsk.value, "flops": fl.value}
    finally:
        L.lamb_oracle_free(h)


def block_norm(x: np.ndarray) -> float:
    x = np.ascontiguousarray(x, dtype=np.float64).ravel()
    return lib().lamb_oracle_block_norm(x.ctypes.data, x.size)
