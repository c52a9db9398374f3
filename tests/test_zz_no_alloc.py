"""The allocation-free filter entry point against the FP32 oracle.

spx_filter_noalloc exists for callers that cannot call cudaMalloc (a host loop
that must not synchronize the device, a framework with its own memory pool, a
driver that forbids allocation after start-up).  It works on device buffers the
caller owns and keeps its scratch in a fixed device array.  This file is named
to be collected last, so a run that stops at the first failure has run every
other test first; it also passes alone in a fresh process.

The filter is bit-exact with the reference's FP32 arithmetic, so results are
compared with array_equal against the oracle's binomial_filter_2_d passes.
The argument checks run before any CUDA call, so they are tested on the CPU.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as orc

SPX_ERR_ARG = 1
MAX_CELLS = 4 * 1024 * 1024


def _lib():
    from spectral_rs_b200 import _lib
    return _lib.load()


def _call(lib, nx, ny, n_pass, d_in, d_out):
    import torch
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.spx_filter_noalloc(nx, ny, n_pass, ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(d_out.data_ptr()),
                                ctypes.c_void_p(st))
    assert rc == 0, lib.spx_noalloc_last_error()
    torch.cuda.synchronize()


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,n_pass", [(24, 12, 4), (64, 32, 3), (512, 128, 8), (40, 20, 1), (32, 16, 0)])
def test_filter_noalloc_matches_oracle(nx, ny, n_pass):
    import torch
    lib = _lib()
    rng = np.random.default_rng(nx + ny + n_pass)
    for call in range(2):  # two calls in a row share the one scratch array
        x = rng.standard_normal((ny + 2) * (nx + 2)).astype(np.float32)
        ref = orc.field_op(nx, ny, 2, x, n_pass=n_pass, dtype=np.float32)
        d_in = torch.from_numpy(x).cuda()
        d_out = torch.full_like(d_in, float("nan"))
        _call(lib, nx, ny, n_pass, d_in, d_out)
        assert np.array_equal(d_out.cpu().numpy(), ref), (call, "out of place")
        assert np.array_equal(d_in.cpu().numpy(), x)  # input untouched
        # in place on the same buffer
        d_io = torch.from_numpy(x).cuda()
        _call(lib, nx, ny, n_pass, d_io, d_io)
        assert np.array_equal(d_io.cpu().numpy(), ref), (call, "in place")


@pytest.mark.gpu
def test_filter_noalloc_rejects_oversize_grid():
    import torch
    lib = _lib()
    d = torch.zeros(8, device="cuda")
    rc = lib.spx_filter_noalloc(4096, 4096, 1, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                                ctypes.c_void_p(0))
    assert rc == SPX_ERR_ARG
    assert b"exceeds the fixed scratch" in lib.spx_noalloc_last_error()


# Argument checks: each returns before any CUDA call, so these run on the CPU
# with addresses that are never dereferenced.
FAKE_IN, FAKE_OUT = 0x10000000, 0x20000000


@pytest.mark.parametrize("nx,ny,expect", [
    (2 ** 62, 2, b"must each be at most"),      # would wrap (nx+2)*(ny+2) to 8 cells
    (2, 2 ** 62, b"must each be at most"),
    (MAX_CELLS + 1, 2, b"must each be at most"),
    (2 ** 32 + 6, 2, b"must each be at most"),  # would truncate to a small int grid
    (4096, 4096, b"exceeds the fixed scratch"),
    (1, 64, b"smaller than 2 x 2"),
    (64, 1, b"smaller than 2 x 2"),
])
def test_filter_noalloc_rejects_bad_sizes_without_launching(nx, ny, expect):
    lib = _lib()
    rc = lib.spx_filter_noalloc(nx, ny, 4, ctypes.c_void_p(FAKE_IN), ctypes.c_void_p(FAKE_OUT), None)
    assert rc == SPX_ERR_ARG
    assert expect in lib.spx_noalloc_last_error()


def test_filter_noalloc_rejects_null_and_partial_overlap():
    lib = _lib()
    assert lib.spx_filter_noalloc(64, 32, 4, None, ctypes.c_void_p(FAKE_OUT), None) == SPX_ERR_ARG
    assert lib.spx_filter_noalloc(64, 32, 4, ctypes.c_void_p(FAKE_IN), None, None) == SPX_ERR_ARG
    assert b"null buffer" in lib.spx_noalloc_last_error()
    # d_out starts inside d_in's (66*34 floats) range: partial overlap
    rc = lib.spx_filter_noalloc(64, 32, 4, ctypes.c_void_p(FAKE_IN), ctypes.c_void_p(FAKE_IN + 4 * 100), None)
    assert rc == SPX_ERR_ARG
    assert b"overlap" in lib.spx_noalloc_last_error()
    rc = lib.spx_filter_noalloc(64, 32, 0, ctypes.c_void_p(FAKE_IN + 4 * 100), ctypes.c_void_p(FAKE_IN), None)
    assert rc == SPX_ERR_ARG


def test_filter_noalloc_error_message_is_per_thread():
    import threading
    lib = _lib()
    lib.spx_filter_noalloc(1, 64, 4, ctypes.c_void_p(FAKE_IN), ctypes.c_void_p(FAKE_OUT), None)
    mine = lib.spx_noalloc_last_error()
    seen = []

    def other():
        seen.append(lib.spx_noalloc_last_error())  # nothing failed on this thread yet
        lib.spx_filter_noalloc(4096, 4096, 4, ctypes.c_void_p(FAKE_IN), ctypes.c_void_p(FAKE_OUT), None)
        seen.append(lib.spx_noalloc_last_error())

    t = threading.Thread(target=other)
    t.start()
    t.join()
    assert seen[0] == b"" and b"exceeds" in seen[1]
    assert lib.spx_noalloc_last_error() == mine
