"""GPU test of jsvd_plain_svd_noalloc, the entry point for callers that cannot
call cudaMalloc (a framework owning the whole device pool, latency-critical code
that cannot take the device synchronisation of cudaMalloc/cudaFree, plugin hosts
that forbid allocation).  It must give the same results as the allocating entry
point jsvd_plain_svd_device - the tolerance of the plain-path tests is
bit-for-bit equality - on two calls in a row (the second call reuses the shared
scratch array that the first one left dirty), it must leave the device's free
memory unchanged once a warm-up call has loaded it, and it must refuse requests
larger than its fixed scratch with a clear error.

Kept in its own file, collected last, so a run that stops at the first failure
has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import jsvd
import workloads as W

pytestmark = pytest.mark.gpu


def _bind():
    lib = jsvd.lib()
    fn = lib.jsvd_plain_svd_noalloc
    P, S = ctypes.c_void_p, ctypes.c_size_t
    fn.argtypes = [P, S, S, ctypes.POINTER(jsvd.Config), P, P, P, P, P]
    fn.restype = ctypes.c_int
    return fn


def _solve(fn, a, cfg, device):
    import torch

    m, n = a.shape
    da = torch.from_numpy(a).to(device)
    du = torch.full((m, n), np.nan, dtype=torch.float64, device=device)
    ds = torch.full((n,), np.nan, dtype=torch.float64, device=device)
    dv = torch.full((n, n), np.nan, dtype=torch.float64, device=device)
    torch.cuda.synchronize(device)
    sw = ctypes.c_int(0)
    if fn is None:
        sweeps = jsvd.plain_svd_device(da.data_ptr(), m, n, du.data_ptr(), ds.data_ptr(), dv.data_ptr(), cfg)
    else:
        rc = fn(da.data_ptr(), m, n, ctypes.byref(cfg), du.data_ptr(), ds.data_ptr(), dv.data_ptr(),
                ctypes.byref(sw), None)
        jsvd.check(rc)
        sweeps = sw.value
    torch.cuda.synchronize(device)
    return du.cpu().numpy(), ds.cpu().numpy(), dv.cpu().numpy(), sweeps


def test_noalloc_matches_allocating_entry_on_two_calls(cuda_device):
    fn = _bind()
    cfg = jsvd.default_config(epsilon=1e-13)
    # Two calls in a row with different shapes: the second must not see the
    # first one's leftovers in the shared scratch array.
    for m, n, seed in [(400, 301, 41), (512, 512, 1)]:
        a = W.gaussian_splitmix(m, n, seed)
        got = _solve(fn, a, cfg, cuda_device)
        exp = _solve(None, a, cfg, cuda_device)
        assert got[3] == exp[3]
        for x, y in zip(got[:3], exp[:3]):
            assert np.array_equal(x, y)


def test_noalloc_allocates_nothing_after_warm_up(cuda_device):
    """After one warm-up call (module loaded, scratch committed, kernels of
    this reduction width loaded), a call of a new shape must leave the device's
    free memory exactly as it was.  Every buffer the call touches is made
    before the first reading of free memory."""
    import torch

    fn = _bind()
    cfg = jsvd.default_config(epsilon=1e-12)
    _solve(fn, W.gaussian_splitmix(96, 64, 5), cfg, cuda_device)  # warm-up
    m, n = 300, 200
    a = W.gaussian_splitmix(m, n, 6)
    da = torch.from_numpy(a).to(cuda_device)
    du = torch.empty((m, n), dtype=torch.float64, device=cuda_device)
    ds = torch.empty((n,), dtype=torch.float64, device=cuda_device)
    dv = torch.empty((n, n), dtype=torch.float64, device=cuda_device)
    sw = ctypes.c_int(0)
    torch.cuda.synchronize(cuda_device)
    free_before, _ = torch.cuda.mem_get_info(cuda_device)
    rc = fn(da.data_ptr(), m, n, ctypes.byref(cfg), du.data_ptr(), ds.data_ptr(), dv.data_ptr(), ctypes.byref(sw),
            None)
    torch.cuda.synchronize(cuda_device)
    free_after, _ = torch.cuda.mem_get_info(cuda_device)
    jsvd.check(rc)
    assert sw.value >= 1
    assert free_after == free_before


def test_noalloc_rejects_requests_beyond_its_scratch(cuda_device):
    import torch

    fn = _bind()
    m, n = 4096, 1024  # 4M + 1M doubles > 2M
    da = torch.zeros((m, n), dtype=torch.float64, device=cuda_device)
    rc = fn(da.data_ptr(), m, n, ctypes.byref(jsvd.default_config()), None, None, None, None, None)
    assert rc == jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert "exceeds the fixed scratch" in jsvd.last_error()[1]
