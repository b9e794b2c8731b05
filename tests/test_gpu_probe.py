"""The tensor-core throughput probe behind the mixed path's roofline: the
tile kernel's own nine-MMA stage (n = 0) and the single-width forms run and
report a throughput between the mma.sync int8 rate (about 1,140 TOP/s) and
a little above the nominal dense int8 peak of a B200 (4,500 TOP/s)."""
import ctypes

import pytest

from lamb_b200 import gpu

pytestmark = pytest.mark.gpu


def test_tcgen05_stage_probe(gpu_ctx):
    f = gpu.lib().lamb_probe_int8_tcgen05_tops
    f.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]
    f.restype = ctypes.c_int32
    tops = {}
    for n in (0, 64, 256):
        out = ctypes.c_double(0.0)
        assert f(0, n, 2, ctypes.byref(out)) == 0
        tops[n] = out.value
        assert 1000.0 < out.value < 5000.0, (n, out.value)
    # nine MMAs of N up to 256 per stage beat 21 of N = 64
    assert tops[0] > tops[64]
