"""Device-buffer entry points called without a stream (stream 0) on buffers
the caller filled on the legacy default stream.

The library then runs on its own non-blocking stream, made to wait on the
device for everything queued on the legacy stream so far; the host never
synchronises.  The input copy here is queued behind about ten milliseconds of
FP64 GEMMs, so a solve that did not wait would read the zeros the buffer held
before the copy.  The result must equal the host-buffer entry's bit for bit.
"""
import numpy as np
import pytest

import jsvd
import workloads as W

pytestmark = pytest.mark.gpu

ENTRIES = {
    "plain": jsvd.plain_svd_device,
    "precond": jsvd.precond_svd_device,
    "blocked": jsvd.blocked_svd_device,
    "blockpair": jsvd.blockpair_svd_device,
}


@pytest.mark.parametrize("solver", sorted(ENTRIES))
def test_null_stream_waits_for_legacy_stream_work(cuda_device, solver):
    import torch

    legacy = torch.cuda.default_stream(cuda_device)
    assert legacy.cuda_stream == 0, "torch's default stream is the legacy default stream"
    m, n = 300, 96
    a = W.gaussian_splitmix(m, n, seed=77)
    cfg = jsvd.default_config(epsilon=1e-13)
    ref = jsvd.svd(a, solver, cfg)
    host_a = torch.from_numpy(a).pin_memory()
    torch.cuda.synchronize(cuda_device)
    with torch.cuda.stream(legacy):
        da = torch.zeros((m, n), dtype=torch.float64, device=cuda_device)
        du = torch.empty((m, n), dtype=torch.float64, device=cuda_device)
        ds = torch.empty(n, dtype=torch.float64, device=cuda_device)
        dv = torch.empty((n, n), dtype=torch.float64, device=cuda_device)
        busy = torch.randn((4096, 4096), dtype=torch.float64, device=cuda_device)
        for _ in range(4):
            busy = busy @ busy / 64.0
        da.copy_(host_a, non_blocking=True)
    sw = ENTRIES[solver](da.data_ptr(), m, n, du.data_ptr(), ds.data_ptr(), dv.data_ptr(), cfg)
    torch.cuda.synchronize(cuda_device)
    assert sw == ref.sweeps
    assert np.array_equal(ds.cpu().numpy(), ref.sigma)
    assert np.array_equal(du.cpu().numpy(), ref.u)
    assert np.array_equal(dv.cpu().numpy(), ref.v)
    assert torch.isfinite(busy).all()
