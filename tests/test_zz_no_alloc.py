"""The allocation-free transpose (eg_csr2csc_device_noalloc).

It exists for callers that must not allocate device memory when they need a
transpose: an application that gave all GPU memory to its own pool at
start-up, a serving process that cannot afford cudaMalloc / cudaFree on its
request path, a plugin whose host forbids allocation after initialisation.
They pass device buffers of their own and the temporaries come from a fixed
static device array.  Its output must equal the allocating entry point's,
bit for bit, call after call, since the static array keeps the previous
call's contents.

This file is collected last (test_zz_*), so that a failure here cannot hide
any other test in a run that stops at the first failure; it also passes when
run alone in a fresh process.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import egsolver_b200 as eg

pytestmark = pytest.mark.gpu


def random_csr(rng, nrow, ncol, nnz):
    counts = rng.multinomial(nnz, np.ones(nrow) / nrow)
    rp = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    col = rng.integers(0, ncol, nnz).astype(np.int32)
    val = rng.integers(-10**6, 10**6, nnz).astype(np.int32)
    return rp, col, val


def call_noalloc(torch, nrow, ncol, rp, col, val):
    dev = torch.device("cuda:0")
    d_rp = torch.from_numpy(rp).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    d_val = torch.from_numpy(val).to(dev)
    nnz = col.shape[0]
    d_cp = torch.full((ncol + 1,), -1, dtype=torch.int64, device=dev)
    d_cr = torch.full((max(nnz, 1),), -1, dtype=torch.int32, device=dev)
    d_cv = torch.full((max(nnz, 1),), -1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    status = eg.lib().eg_csr2csc_device_noalloc(nrow, ncol, nnz, d_rp.data_ptr(), d_col.data_ptr(), d_val.data_ptr(),
                                                d_cp.data_ptr(), d_cr.data_ptr(), d_cv.data_ptr(),
                                                ctypes.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    return status, d_cp.cpu().numpy(), d_cr.cpu().numpy()[:nnz], d_cv.cpu().numpy()[:nnz]


def test_noalloc_transpose_equals_allocating_transpose_twice_in_a_row():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2024)
    # two calls in a row with different shapes: the second must not see the first's leftovers
    for nrow, ncol, nnz in ((3000, 5000, 200_000), (700, 300, 90_000)):
        rp, col, val = random_csr(rng, nrow, ncol, nnz)
        want = eg.csr2csc(nrow, ncol, rp, col, val)
        status, cp, cr, cv = call_noalloc(torch, nrow, ncol, rp, col, val)
        assert status == 0, eg.lib().eg_last_error().decode()
        np.testing.assert_array_equal(cp, want[0])
        np.testing.assert_array_equal(cr, want[1])
        np.testing.assert_array_equal(cv, want[2])


def test_noalloc_rejects_inputs_beyond_its_static_capacity():
    torch = pytest.importorskip("torch")
    too_many = (1 << 20) + 1
    dev = torch.device("cuda:0")
    d = torch.zeros(8, dtype=torch.int64, device=dev)
    status = eg.lib().eg_csr2csc_device_noalloc(1, 4, too_many, d.data_ptr(), d.data_ptr(), d.data_ptr(),
                                                d.data_ptr(), d.data_ptr(), d.data_ptr(), None)
    assert eg._ffi.STATUS_NAMES[status] == "EG_ERR_INVALID"
    assert "at most" in eg.lib().eg_last_error().decode()


def test_noalloc_empty_matrix():
    torch = pytest.importorskip("torch")
    rp = np.zeros(6, dtype=np.int64)
    col = np.zeros(0, dtype=np.int32)
    val = np.zeros(0, dtype=np.int32)
    status, cp, cr, cv = call_noalloc(torch, 5, 7, rp, col, val)
    assert status == 0, eg.lib().eg_last_error().decode()
    np.testing.assert_array_equal(cp, np.zeros(8, dtype=np.int64))
    assert cr.size == 0 and cv.size == 0


def test_noalloc_reports_a_column_out_of_range():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(7)
    rp, col, val = random_csr(rng, 100, 50, 1000)
    col[123] = 50  # one past the last column
    status, *_ = call_noalloc(torch, 100, 50, rp, col, val)
    assert eg._ffi.STATUS_NAMES[status] == "EG_ERR_INVALID"
    assert "column" in eg.lib().eg_last_error().decode()


def test_noalloc_reports_malformed_offsets_after_a_larger_call():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(8)
    # a large valid call leaves its edge indexes in the shared array ...
    rp, col, val = random_csr(rng, 2000, 2000, 400_000)
    status, *_ = call_noalloc(torch, 2000, 2000, rp, col, val)
    assert status == 0, eg.lib().eg_last_error().decode()
    # ... and a smaller call whose offsets skip entries must not read them
    rp, col, val = random_csr(rng, 50, 40, 5000)
    rp[10] = rp[11] + 7  # row 9 ends after row 10 ends: not monotone
    status, cp, cr, cv = call_noalloc(torch, 50, 40, rp, col, val)
    assert eg._ffi.STATUS_NAMES[status] == "EG_ERR_INVALID"
    assert "row offsets" in eg.lib().eg_last_error().decode()
    # the outputs hold only values the call could legally write
    assert ((cr >= 0) & (cr < 50)).all()
    assert np.isin(cv, val).all()
    # and the next valid call is exact again
    rp, col, val = random_csr(rng, 300, 200, 20_000)
    want = eg.csr2csc(300, 200, rp, col, val)
    status, cp, cr, cv = call_noalloc(torch, 300, 200, rp, col, val)
    assert status == 0, eg.lib().eg_last_error().decode()
    np.testing.assert_array_equal(cp, want[0])
    np.testing.assert_array_equal(cr, want[1])
    np.testing.assert_array_equal(cv, want[2])
