"""The C ABI from a plain C99 program (tests/abi_caller.c).

The CPU test compiles the caller with strict warnings against
include/lamb_gpu.h, links it to liblamb_b200.so and runs it: without a device
lamb_gpu_ctx_create must fail with a decodable status (exit code 3).  The GPU
test runs the same binary on a water system and checks its C, read back from
the file the program wrote, against the oracle: block pattern bit-exact,
values within 1e-12 relative Frobenius error."""
import os
import subprocess

import numpy as np
import pytest

from lamb_b200.matrix import LambMatrix, Sector

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(REPO, "tests", "abi_caller.c")


def _compile(tmp_path):
    from lamb_b200 import build
    lib = build.build_cuda()
    libdir = os.path.dirname(lib)
    exe = str(tmp_path / "abi_caller")
    subprocess.check_call(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror", "-O1",
                           "-I", os.path.join(REPO, "include"), SRC, "-o", exe, "-L", libdir, "-llamb_b200",
                           "-Wl,-rpath," + libdir])
    return exe


def _write_matrix(f, m: LambMatrix):
    f.write(np.int64(len(m.sectors)).tobytes())
    for s in m.sectors:
        f.write(np.array([s.subset_row, s.subset_col, s.n_rows, s.n_cols, s.n_blks, s.data.shape[0]],
                         np.int64).tobytes())
        f.write(np.asarray(s.row_blk_sizes, np.int8).tobytes())
        f.write(np.asarray(s.col_blk_sizes, np.int8).tobytes())
        f.write(np.asarray(s.row_p, np.int64).tobytes())
        f.write(np.asarray(s.col_i, np.int16).tobytes())
        f.write(np.asarray(s.extents, np.int64).reshape(-1).tobytes())
        f.write(np.asarray(s.data, np.float64).tobytes())


def _read_matrix(buf: bytes) -> LambMatrix:
    pos = 0

    def take(dtype, n):
        nonlocal pos
        a = np.frombuffer(buf, dtype, count=n, offset=pos).copy()
        pos += a.nbytes
        return a

    n = int(take(np.int64, 1)[0])
    sectors = []
    for _ in range(n):
        sr, sc, nr, nc, nb, dl = (int(v) for v in take(np.int64, 6))
        rb, cb = take(np.int8, nr), take(np.int8, nc)
        row_p, col_i = take(np.int64, nr + 1), take(np.int16, nb)
        ext = take(np.int64, 2 * nb).reshape(nb, 2)
        sectors.append(Sector(sr, sc, rb, cb, row_p, col_i, ext, take(np.float64, dl)))
    assert pos == len(buf)
    return LambMatrix(sectors)


def _inputs(tmp_path, a, b):
    path = str(tmp_path / "in.bin")
    with open(path, "wb") as f:
        _write_matrix(f, a)
        _write_matrix(f, b)
    return path


def test_c_caller_builds_and_reports_no_device(tmp_path):
    import torch
    exe = _compile(tmp_path)
    from lamb_b200.gen import random_fill_matrix
    a = random_fill_matrix(0)
    inp = _inputs(tmp_path, a, a)
    r = subprocess.run([exe, inp, str(tmp_path / "out.bin"), "0", "0"], capture_output=True, text=True, timeout=120)
    if torch.cuda.is_available():
        pytest.skip("a device is present: the no-device path is not reachable")
    assert r.returncode == 3, r.stderr
    assert "ctx_create: status" in r.stderr and "level 3" in r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "usage" in r.stderr


def test_read_write_round_trip(tmp_path):
    from lamb_b200.gen import random_fill_matrix
    a = random_fill_matrix(3)
    p = tmp_path / "m.bin"
    with open(p, "wb") as f:
        _write_matrix(f, a)
    b = _read_matrix(p.read_bytes())
    for x, y in zip(a.sectors, b.sectors):
        for k in ("row_blk_sizes", "col_blk_sizes", "row_p", "col_i", "extents", "data"):
            assert np.array_equal(getattr(x, k), getattr(y, k)), k


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [0, 8])
def test_c_caller_multiply_parity(tmp_path, flags):
    import oracle
    from lamb_b200.gen import WATER_192
    from tests.helpers import assert_same_pattern, rel_frobenius_error
    exe = _compile(tmp_path)
    g, a, b = WATER_192.build()
    inp = _inputs(tmp_path, a, b)
    out = tmp_path / "out.bin"
    r = subprocess.run([exe, inp, str(out), repr(WATER_192.eps), str(flags)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "bad handle (expected)" in r.stderr and "invalid handle" in r.stderr
    c = _read_matrix(out.read_bytes())
    c.validate()
    c_ref, st_ref = oracle.multiply(a, b, WATER_192.eps)
    assert_same_pattern(c, c_ref)
    assert rel_frobenius_error(c, c_ref) <= 1e-12
    fields = dict(zip(r.stdout.split()[0::2], r.stdout.split()[1::2]))
    assert int(fields["products"]) == st_ref["n_products"]
    assert int(fields["skipped"]) == st_ref["n_products_skipped"]
    assert int(fields["launches"]) > 0
