"""The single-rank MPI stub (lamb_b200/fortran/mpi_stub): its constant set
against mpif.h and against the names LAMB's sources use, and the routines'
one-rank semantics, called through the gfortran calling convention (every
argument by reference, CHARACTER lengths appended) from ctypes."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STUB = os.path.join(REPO, "lamb_b200", "fortran", "mpi_stub")

# Every MPI constant named in LAMB's Fortran sources (src/*.F90: the kinds
# module, the environment, market, window, file and utility modules).
USED_BY_LAMB = ["MPI_ADDRESS_KIND", "MPI_ANY_SOURCE", "MPI_ANY_TAG", "MPI_STATUS_SIZE", "MPI_REAL4", "MPI_REAL8",
                "MPI_COMPLEX8", "MPI_COMPLEX16", "MPI_INTEGER4", "MPI_INTEGER8", "MPI_INTEGER1", "MPI_INTEGER2",
                "MPI_REAL16", "MPI_CHARACTER", "MPI_SUCCESS", "MPI_INFO_NULL", "MPI_COMM_WORLD", "MPI_MAX",
                "MPI_SUM", "MPI_LOCK_SHARED", "MPI_LOCK_EXCLUSIVE", "MPI_MODE_NOCHECK", "MPI_UNDEFINED",
                "MPI_TAG", "MPI_SOURCE", "MPI_ERROR", "MPI_MODE_WRONLY", "MPI_MODE_RDWR", "MPI_MODE_RDONLY",
                "MPI_MODE_NOSUCCEED", "MPI_MODE_NOSTORE", "MPI_MODE_NOPUT", "MPI_MODE_NOPRECEDE",
                "MPI_ERRORS_RETURN", "MPI_INTEGER", "MPI_REAL", "MPI_COMPLEX"]


@pytest.fixture(scope="module")
def stub(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("mpi") / "libmpi_stub.so")
    subprocess.check_call(["gcc", "-O2", "-Wall", "-Werror", "-fPIC", "-shared", os.path.join(STUB, "mpi_stub.c"),
                           "-o", out])
    return C.CDLL(out)


def _mpif():
    vals = {}
    for line in open(os.path.join(STUB, "mpif.h")):
        m = re.match(r"\s*PARAMETER\s*\((.*)\)\s*$", line)
        if m:
            for part in m.group(1).split(","):
                k, v = part.split("=")
                vals[k.strip()] = int(v)
    return vals


def _i(v=0):
    return C.c_int32(v)


def test_constants_match_and_cover_lamb(stub):
    vals = _mpif()
    for name in USED_BY_LAMB:
        assert name in vals, name
    for name, v in vals.items():
        got = C.c_int64()
        assert stub.lamb_mpi_stub_constant(name.encode(), C.byref(got)) == 0, name
        assert got.value == v, name
    assert vals["MPI_ADDRESS_KIND"] == 8 and vals["MPI_STATUS_SIZE"] >= 5


def test_environment_and_collectives(stub):
    v, ierr = _mpif(), _i(-1)
    flag = _i(7)
    stub.mpi_initialized_(C.byref(flag), C.byref(ierr))
    assert flag.value == 0 and ierr.value == 0
    stub.mpi_init_(C.byref(ierr))
    stub.mpi_initialized_(C.byref(flag), C.byref(ierr))
    assert flag.value == 1
    world = _i(v["MPI_COMM_WORLD"])
    size, rank, dup = _i(), _i(-1), _i()
    stub.mpi_comm_size_(C.byref(world), C.byref(size), C.byref(ierr))
    stub.mpi_comm_rank_(C.byref(world), C.byref(rank), C.byref(ierr))
    assert (size.value, rank.value, ierr.value) == (1, 0, 0)
    stub.mpi_comm_dup_(C.byref(world), C.byref(dup), C.byref(ierr))
    assert ierr.value == 0 and dup.value not in (0, world.value)
    stub.mpi_comm_free_(C.byref(dup), C.byref(ierr))
    assert dup.value == v["MPI_COMM_NULL"]
    for t, nbytes in (("MPI_REAL8", 8), ("MPI_INTEGER2", 2), ("MPI_COMPLEX16", 16), ("MPI_CHARACTER", 1)):
        s = _i()
        stub.mpi_type_size_(C.byref(_i(v[t])), C.byref(s), C.byref(ierr))
        assert s.value == nbytes and ierr.value == 0
    src = np.arange(5, dtype=np.float64)
    dst = np.zeros(5)
    stub.mpi_allreduce_(src.ctypes.data_as(C.c_void_p), dst.ctypes.data_as(C.c_void_p), C.byref(_i(5)),
                        C.byref(_i(v["MPI_REAL8"])), C.byref(_i(v["MPI_SUM"])), C.byref(world), C.byref(ierr))
    assert ierr.value == 0 and np.array_equal(src, dst)
    text = C.create_string_buffer(b"x" * 64, 64)
    ln = _i()
    stub.mpi_error_string_(C.byref(_i(3)), text, C.byref(ln), C.byref(ierr), C.c_size_t(64))
    assert ierr.value == 0 and 0 < ln.value <= 64 and text.raw[ln.value:] == b" " * (64 - ln.value)


def test_messages_to_self(stub):
    v, ierr = _mpif(), _i(-1)
    world, r8 = _i(v["MPI_COMM_WORLD"]), _i(v["MPI_REAL8"])
    a = np.array([1.5, 2.5, 3.5])
    b = np.array([9.0])
    sreq, rreq, flag = _i(), _i(), _i(-1)
    status = (C.c_int32 * v["MPI_STATUS_SIZE"])()
    out = np.zeros(3)
    stub.mpi_irecv_(out.ctypes.data_as(C.c_void_p), C.byref(_i(3)), C.byref(r8), C.byref(_i(0)), C.byref(_i(7)),
                    C.byref(world), C.byref(rreq), C.byref(ierr))
    assert ierr.value == 0 and rreq.value > 0
    stub.mpi_test_(C.byref(rreq), C.byref(flag), status, C.byref(ierr))
    assert flag.value == 0  # nothing sent yet
    stub.mpi_send_(b.ctypes.data_as(C.c_void_p), C.byref(_i(1)), C.byref(r8), C.byref(_i(0)), C.byref(_i(8)),
                   C.byref(world), C.byref(ierr))
    stub.mpi_isend_(a.ctypes.data_as(C.c_void_p), C.byref(_i(3)), C.byref(r8), C.byref(_i(0)), C.byref(_i(7)),
                    C.byref(world), C.byref(sreq), C.byref(ierr))
    stub.mpi_test_(C.byref(rreq), C.byref(flag), status, C.byref(ierr))
    assert flag.value == 1 and np.array_equal(out, a)  # tag 7 matched past the tag-8 message
    assert status[v["MPI_TAG"] - 1] == 7 and status[v["MPI_SOURCE"] - 1] == 0
    cnt = _i()
    stub.mpi_get_count_(status, C.byref(r8), C.byref(cnt), C.byref(ierr))
    assert cnt.value == 3
    stub.mpi_test_(C.byref(sreq), C.byref(flag), status, C.byref(ierr))
    assert flag.value == 1 and sreq.value == 0
    # the tag-8 message is still queued; an any-tag receive takes it
    one = np.zeros(1)
    stub.mpi_irecv_(one.ctypes.data_as(C.c_void_p), C.byref(_i(1)), C.byref(r8), C.byref(_i(v["MPI_ANY_SOURCE"])),
                    C.byref(_i(v["MPI_ANY_TAG"])), C.byref(world), C.byref(rreq), C.byref(ierr))
    stub.mpi_test_(C.byref(rreq), C.byref(flag), status, C.byref(ierr))
    assert flag.value == 1 and one[0] == 9.0 and status[v["MPI_TAG"] - 1] == 8


def test_windows_memory_and_files(stub, tmp_path):
    v, ierr = _mpif(), _i(-1)
    world = _i(v["MPI_COMM_WORLD"])
    win = _i()
    buf = np.zeros(4)
    stub.mpi_win_create_(buf.ctypes.data_as(C.c_void_p), C.byref(C.c_int64(32)), C.byref(_i(8)),
                         C.byref(_i(v["MPI_INFO_NULL"])), C.byref(world), C.byref(win), C.byref(ierr))
    assert ierr.value == 0 and win.value > 0
    stub.mpi_win_lock_(C.byref(_i(v["MPI_LOCK_SHARED"])), C.byref(_i(0)), C.byref(_i(v["MPI_MODE_NOCHECK"])),
                       C.byref(win), C.byref(ierr))
    stub.mpi_win_unlock_(C.byref(_i(0)), C.byref(win), C.byref(ierr))
    stub.mpi_win_fence_(C.byref(_i(0)), C.byref(win), C.byref(ierr))
    stub.mpi_win_free_(C.byref(win), C.byref(ierr))
    assert ierr.value == 0 and win.value == 0
    p = C.c_void_p()
    stub.mpi_alloc_mem_(C.byref(C.c_int64(1024)), C.byref(_i(0)), C.byref(p), C.byref(ierr))
    assert ierr.value == 0 and p.value
    stub.mpi_free_mem_(p, C.byref(ierr))
    data = np.arange(10, dtype=np.int64)
    path = tmp_path / "blob.bin"
    data.tofile(path)
    name = str(path).encode() + b" " * 8  # blank-padded like a Fortran CHARACTER
    fh, status = _i(), (C.c_int32 * v["MPI_STATUS_SIZE"])()
    stub.mpi_file_open_(C.byref(world), name, C.byref(_i(v["MPI_MODE_RDONLY"])), C.byref(_i(0)), C.byref(fh),
                        C.byref(ierr), C.c_size_t(len(name)))
    assert ierr.value == 0 and fh.value > 0
    got = np.zeros(10, np.int64)
    stub.mpi_file_read_(C.byref(fh), got.ctypes.data_as(C.c_void_p), C.byref(_i(10)),
                        C.byref(_i(v["MPI_INTEGER8"])), status, C.byref(ierr))
    cnt = _i()
    stub.mpi_get_count_(status, C.byref(_i(v["MPI_INTEGER8"])), C.byref(cnt), C.byref(ierr))
    assert np.array_equal(got, data) and cnt.value == 10
    stub.mpi_file_close_(C.byref(fh), C.byref(ierr))
    assert ierr.value == 0 and fh.value == 0
