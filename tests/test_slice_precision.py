"""Why the mixed-precision multiply slices operands into int8 digits with exact
int32 accumulation instead of bf16 slices with FP32 accumulation.

Both schemes write each operand as a sum of low-precision slices and
recombine the slice products in FP64 (Ozaki, Ogita, Oishi and Rump, Numer.
Algorithms 59 (2012)).  With FP32 accumulators every slice product is rounded
to 24 bits while it is summed over the inner dimension, so the leading slice
pair alone limits the result to about 1e-7 relative, whatever the number of
slices.  Digits of at most 7 bits on a power-of-two scale per element row of A
(column of B) make every slice product an exact integer sum, and the error
falls by about 2^7 per digit.  This is the scheme of lamb_b200/csrc/mixed.cu
(its header states the digit weights w_p = 2^(-6-7(p-1)) and the dropped pairs
p + q > s + 1).  Inner length 256 is that of a typical C block's stack at
6,144 waters (31.5 products of 7.7 inner columns on average).
"""
import numpy as np
import pytest

M, K, N = 64, 256, 64
BOUND = 1e-11  # error bound of the mixed-precision multiply against FP64


@pytest.fixture(scope="module")
def operands():
    rng = np.random.default_rng(0)
    # entries spread over three decades inside a row, like exp(-r/1.5) within a cutoff
    a = rng.uniform(-1, 1, (M, K)) * 10.0 ** rng.uniform(-3, 0, (M, K))
    b = rng.uniform(-1, 1, (K, N)) * 10.0 ** rng.uniform(-3, 0, (K, N))
    return a, b, a @ b


def _bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float32."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def _bf16_fp32(a, b, s):
    def split(x):
        out, r = [], x.copy()
        for _ in range(s):
            p = _bf16(r).astype(np.float64)
            out.append(p)
            r = r - p
        return out
    sa, sb = split(a), split(b)
    c = np.zeros((a.shape[0], b.shape[1]))
    for p in range(s):
        for q in range(s - p):
            c += (sa[p].astype(np.float32) @ sb[q].astype(np.float32)).astype(np.float64)
    return c


def _int8_digits(a, b, s):
    def digits(x, axis):
        e = np.ceil(np.log2(np.abs(x).max(axis=axis, keepdims=True)))
        r, ds = x / 2.0 ** e, []
        for p in range(s):
            w = 2.0 ** (-6 - 7 * p)
            d = np.rint(r / w)
            assert np.abs(d).max() <= 64
            ds.append(d.astype(np.int64))
            r = r - d * w
        return ds, e
    da, ea = digits(a, 1)
    db, eb = digits(b, 0)
    c = np.zeros((a.shape[0], b.shape[1]))
    for p in range(s):
        for q in range(s - p):
            c += (da[p] @ db[q]).astype(np.float64) * 2.0 ** (-12 - 7 * (p + q))  # exact integer products
    return c * 2.0 ** ea * 2.0 ** eb


def _err(c, ref):
    return float(np.linalg.norm(c - ref) / np.linalg.norm(ref))


def test_bf16_slices_with_fp32_accumulation_stall_above_the_bound(operands):
    a, b, ref = operands
    errs = [_err(_bf16_fp32(a, b, s), ref) for s in (3, 4, 6)]
    assert min(errs) > 1e3 * BOUND
    assert errs[2] > 0.5 * errs[0]  # more slices do not help: the FP32 sums limit the result


def test_int8_digits_with_exact_accumulation_reach_the_bound(operands):
    a, b, ref = operands
    errs = {s: _err(_int8_digits(a, b, s), ref) for s in (5, 6, 7)}
    assert errs[5] > BOUND
    assert errs[7] <= BOUND / 10
    assert errs[5] > 30 * errs[6] > 900 * errs[7]  # about 2^7 per added digit
