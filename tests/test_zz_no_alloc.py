"""The allocation-free transpose (eg_csr2csc_device_noalloc).

It exists for callers that cannot allocate device memory when they need a
transpose (inside CUDA stream capture, under a runtime that owns all device
memory, after start-up in hosts that forbid allocation): they pass device
buffers of their own and the temporaries come from a fixed static device
array.  Its output must equal the allocating entry point's, bit for bit, call
after call, since the static array keeps the previous call's contents.

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
