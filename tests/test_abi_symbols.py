"""The C-ABI libraries load and export every function their headers declare
(no compute calls: these run without a GPU)."""
import ctypes
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    txt = open(os.path.join(REPO, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*LAMB_API\s+[\w\s\*]+?\b(lamb_\w+)\s*\(", txt, flags=re.M)))


def test_gpu_library_exports_header():
    from lamb_b200 import build
    path = build.build_cuda()
    lib = ctypes.CDLL(path)
    names = _declared("lamb_gpu.h")
    assert "lamb_gpu_multiply" in names and "lamb_gpu_matrix_upload" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_gen_library_exports_header():
    from lamb_b200 import build
    lib = ctypes.CDLL(build.build_gen())
    missing = [n for n in _declared("lamb_gen.h") if not hasattr(lib, n)]
    assert not missing, missing


def test_status_decoding_without_gpu():
    from lamb_b200 import build
    lib = ctypes.CDLL(build.build_cuda())
    st = 3 * 100000 + (100 + 50000)
    assert lib.lamb_gpu_status_level(st) == 3
    assert lib.lamb_gpu_status_type(st) == 100
    st = 5 * 100000 + (-2000 + 50000)
    assert lib.lamb_gpu_status_type(st) == -2000


def test_context_creation_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from lamb_b200 import gpu
    with pytest.raises(gpu.LambError):
        gpu.Context(0)


def test_probe_library_exports_header_and_refuses_bad_arguments():
    """Every probe declared in lamb_probe.h is exported; the tcgen05 probe
    refuses an unknown instruction width or a null output before it touches
    a device."""
    from lamb_b200 import build
    lib = ctypes.CDLL(build.build_cuda())
    names = _declared("lamb_probe.h")
    assert "lamb_probe_int8_tcgen05_tops" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    f = lib.lamb_probe_int8_tcgen05_tops
    f.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]
    f.restype = ctypes.c_int32
    out = ctypes.c_double(-1.0)
    for n in (7, 128, -1):
        assert lib.lamb_gpu_status_type(f(0, n, 1, ctypes.byref(out))) == 100
    assert lib.lamb_gpu_status_type(f(0, 0, 1, None)) == 100
