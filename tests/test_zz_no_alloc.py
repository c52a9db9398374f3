"""The allocation-free filter entry point against the allocating one.

spx_filter_noalloc exists for callers that cannot call cudaMalloc (a host loop
that must not synchronize the device, a framework with its own memory pool, a
driver that forbids allocation after start-up).  It works on device buffers the
caller owns and keeps its scratch in a fixed device array.  This file is named
to be collected last, so a run that stops at the first failure has run every
other test first; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(lib, nx, ny, n_pass, d_in, d_out):
    import torch
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.spx_filter_noalloc(nx, ny, n_pass, ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(d_out.data_ptr()),
                                ctypes.c_void_p(st))
    assert rc == 0, lib.spx_noalloc_last_error()
    torch.cuda.synchronize()


@pytest.mark.parametrize("nx,ny,n_pass", [(24, 12, 4), (64, 32, 3), (512, 128, 8)])
def test_filter_noalloc_matches_allocating_entry_point(nx, ny, n_pass):
    import torch
    from spectral_rs_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(nx + ny + n_pass)
    for call in range(2):  # two calls in a row share the one scratch array
        x = rng.standard_normal((ny + 2) * (nx + 2)).astype(np.float32)
        ref = _lib.field_op(nx, ny, 2, x, n_pass=n_pass)
        d_in = torch.from_numpy(x).cuda()
        d_out = torch.empty_like(d_in)
        _call(lib, nx, ny, n_pass, d_in, d_out)
        out = d_out.cpu().numpy()
        assert np.max(np.abs(out - ref)) <= 1e-6 * max(1.0, float(np.max(np.abs(ref)))), call
        assert np.array_equal(d_in.cpu().numpy(), x)  # input untouched
        # in place on the same buffer
        d_io = torch.from_numpy(x).cuda()
        _call(lib, nx, ny, n_pass, d_io, d_io)
        assert np.max(np.abs(d_io.cpu().numpy() - ref)) <= 1e-6 * max(1.0, float(np.max(np.abs(ref)))), call


def test_filter_noalloc_rejects_oversize_grid():
    import torch
    from spectral_rs_b200 import _lib
    lib = _lib.load()
    d = torch.zeros(8, device="cuda")
    rc = lib.spx_filter_noalloc(4096, 4096, 1, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                                ctypes.c_void_p(0))
    assert rc == 1
    assert b"exceeds the fixed scratch" in lib.spx_noalloc_last_error()
