"""Blocked FP64 one-sided Jacobi (32-column blocks, two-sided Jacobi on the
64 x 64 panel Gram) on the GPU, within tolerance of LAPACK and of the plain
path: sigma normwise error <= 1e-15 * max(n, 100), per-value relative error
<= 1e-13 * n * max(1, kappa * 1e-6), rho_A <= 1e-13 * n, ||V^T V - I||_F and
||U^T U - I||_F <= 1e-12 * n.  Two FP64 algorithms each carry a normwise
error of order n u, so blocked vs plain is held to 4e-15 * n."""
import numpy as np
import pytest

import jsvd
import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu

CASES = [
    ("square_gauss_256", lambda: W.gaussian_splitmix(256, 256, 61), 1e3),
    ("tall_1024x200_k1e6", lambda: W.spectrum_matrix(1024, 200, W.geometric_sigma(200, 1e-6), 62), 1e6),
    ("odd_blocks_300x161", lambda: W.gaussian_splitmix(300, 161, 63), 1e3),
    ("exact_2_blocks", lambda: W.gaussian_splitmix(100, 64, 64), 1e2),
    ("narrow_40", lambda: W.gaussian_splitmix(90, 40, 65), 1e2),
    ("rank_deficient", lambda: np.hstack([W.gaussian_splitmix(200, 50, 66)] * 2), 1e16),
]


def _solve(a, device, eps=1e-14):
    import torch

    m, n = a.shape
    da = torch.from_numpy(a).to(device)
    du = torch.empty((m, n), dtype=torch.float64, device=device)
    ds = torch.empty(n, dtype=torch.float64, device=device)
    dv = torch.empty((n, n), dtype=torch.float64, device=device)
    sw = jsvd.blocked_svd_device(da.data_ptr(), m, n, du.data_ptr(), ds.data_ptr(), dv.data_ptr(),
                                 jsvd.default_config(epsilon=eps))
    return du.cpu().numpy(), ds.cpu().numpy(), dv.cpu().numpy(), sw


@pytest.mark.parametrize("name,make,kappa", CASES, ids=[c[0] for c in CASES])
def test_blocked_accuracy(cuda_device, name, make, kappa):
    a = make()
    m, n = a.shape
    u, s, v, sw = _solve(a, cuda_device)
    ref = np.linalg.svd(a, compute_uv=False)
    e = O.sigma_errors(s, ref)
    assert e["normwise"] <= 1e-15 * max(n, 100), e
    if kappa < 1e12:
        assert e["max_rel"] <= 1e-13 * n * max(1.0, kappa * 1e-6), e
    r = O.residuals(a, u, s, v)
    assert r["rho_A"] <= 1e-13 * n and r["rho_V"] <= 1e-12 * n, r
    if kappa < 1e12:
        assert r["rho_U"] <= 1e-12 * n, r
    assert 1 <= sw < 128


def test_blocked_deterministic_and_close_to_plain(cuda_device):
    a = W.spectrum_matrix(512, 256, W.geometric_sigma(256, 1e-5), 67)
    x = _solve(a, cuda_device)
    y = _solve(a, cuda_device)
    for p, q in zip(x[:3], y[:3]):
        assert np.array_equal(p, q)
    pu, ps, pv, _ = jsvd.plain_svd(a, jsvd.default_config(epsilon=1e-14))
    assert O.sigma_errors(x[1], ps)["normwise"] <= 4e-15 * 256


@pytest.mark.parametrize("entry", ["jsvd_blocked_svd", "jsvd_blockpair_svd"])
def test_host_buffer_entries_match_device(cuda_device, entry):
    """The host-buffer entry points return the device entry points' bytes."""
    import ctypes

    a = W.gaussian_splitmix(300, 161, 67)
    m, n = a.shape
    cfg = jsvd.default_config(epsilon=1e-14)
    u, s, v = np.empty((m, n)), np.empty(n), np.empty((n, n))
    sw = ctypes.c_int(0)
    jsvd.check(getattr(jsvd.lib(), entry)(a.ctypes.data, m, n, ctypes.byref(cfg), u.ctypes.data, s.ctypes.data,
                                          v.ctypes.data, ctypes.byref(sw)))
    if entry == "jsvd_blocked_svd":
        du, ds, dv, dsw = _solve(a, cuda_device)
    else:
        du, ds, dv, dsw = jsvd.blockpair_svd(a, cfg)
    assert sw.value == dsw and np.array_equal(s, ds) and np.array_equal(u, du) and np.array_equal(v, dv)
