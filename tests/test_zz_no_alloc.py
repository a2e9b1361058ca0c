"""The allocation-free template-norm entry point (gwb_sigma2_noalloc), through the C ABI.

Some callers cannot let a library allocate device memory (a host program whose own pool owns the device, code
running inside a stream capture, latency-bound loops where cudaMalloc would synchronise); this entry keeps its
scratch in a static device array instead of asking for a workspace. Checked: two calls in a row give the same norms
as the allocating entry point gwb_sigma2 (float64, relative 1e-12, the tolerance of the other sigma^2 tests), and a
shape beyond the static scratch is refused before any device work. Collected last so that a failure here comes after
every other test has run."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _norms_with_workspace(lib, H, IP, kmin, df):
    n, flen = H.shape
    nseg = IP.shape[0]
    part_elems = n * nseg * 64
    part = torch.empty(part_elems, dtype=torch.float64, device='cuda')
    sig = torch.empty((n, nseg), dtype=torch.float64, device='cuda')
    lib.call('gwb_sigma2', lib.ptr(H), H.stride(0), n, lib.ptr(IP), IP.stride(0), nseg, kmin, flen, df,
             lib.ptr(part), part_elems, lib.ptr(sig), sig.stride(0), lib.stream_ptr())
    return sig


def test_sigma2_noalloc_matches_the_allocating_entry_point():
    from gwb200 import _lib
    rng = np.random.default_rng(31)
    n, nseg, flen, kmin, df = 300, 9, 65537, 1280, 1 / 64.
    H = torch.from_numpy((rng.standard_normal((n, flen)) + 1j * rng.standard_normal((n, flen))).astype(np.complex64)).cuda()
    ip = rng.uniform(0.1, 2.0, (nseg, flen)).astype(np.float32)
    ip[:, :kmin] = 0
    IP = torch.from_numpy(ip).cuda()
    ref = _norms_with_workspace(_lib, H, IP, kmin, df).cpu().numpy()
    for _ in range(2):
        sig = torch.full((n, nseg), np.nan, dtype=torch.float64, device='cuda')
        _lib.call('gwb_sigma2_noalloc', _lib.ptr(H), H.stride(0), n, _lib.ptr(IP), IP.stride(0), nseg, kmin, flen, df,
                  _lib.ptr(sig), sig.stride(0), _lib.stream_ptr())
        torch.cuda.synchronize()
        np.testing.assert_allclose(sig.cpu().numpy(), ref, rtol=1e-12)


def test_sigma2_noalloc_refuses_shapes_beyond_its_scratch():
    from gwb200 import _lib
    lib = _lib.load()
    n, nseg = 1 << 12, 1 << 8            # n * nseg = 2^20 > 2^19 partial sums
    st = lib.gwb_sigma2_noalloc(ctypes.c_void_p(16), 1024, n, ctypes.c_void_p(16), 1024, nseg, 10, 1024, 1.0,
                                ctypes.c_void_p(16), nseg, None)
    assert st == _lib.GWB_ERR_CAPACITY
    assert b'static scratch' in lib.gwb_last_error()
