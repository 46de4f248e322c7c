"""QR-preconditioned path (shifted CholeskyQR3 + Jacobi on R^T) on the GPU.

Not bit-identical to the reference (different algorithm), so checked within
tolerance against LAPACK on the same input and against the plain path:
sigma normwise error |d sigma_i| / sigma_max <= 1e-15 * n (LAPACK's own error
is of that order), per-value relative error <= 1e-13 * n * max(1, kappa * 1e-6),
rho_A <= 1e-13 * n, ||U^T U - I||_F and ||V^T V - I||_F <= 1e-12 * n.
"""
import numpy as np
import pytest

import jsvd
import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu

CASES = [
    ("tall_k1e6", lambda: W.spectrum_matrix(2048, 512, W.geometric_sigma(512, 1e-6), 41), 1e6),
    ("square_gauss", lambda: W.gaussian_splitmix(300, 300, 42), 1e4),
    ("tall_k1e8", lambda: W.spectrum_matrix(1000, 200, W.geometric_sigma(200, 1e-8), 43), 1e8),
    ("tall_k1e10_graded", lambda: W.spectrum_matrix(1200, 300, W.graded_clustered_sigma(300, 2, 16), 44), 1e10),
    ("odd_cols", lambda: W.gaussian_splitmix(257, 129, 45), 1e3),
    ("one_col", lambda: W.gaussian_splitmix(50, 1, 46), 1.0),
    ("two_cols", lambda: W.gaussian_splitmix(3, 2, 47), 10.0),
]


@pytest.mark.parametrize("name,make,kappa", CASES, ids=[c[0] for c in CASES])
def test_precond_accuracy(cuda_device, name, make, kappa):
    a = make()
    m, n = a.shape
    u, s, v, sw = jsvd.precond_svd(a, jsvd.default_config(epsilon=1e-14))
    ref = np.linalg.svd(a, compute_uv=False)
    e = O.sigma_errors(s, ref)
    assert e["normwise"] <= 1e-15 * max(n, 100), e
    assert e["max_rel"] <= 1e-13 * n * max(1.0, kappa * 1e-6), e
    r = O.residuals(a, u, s, v)
    assert r["rho_A"] <= 1e-13 * n and r["rho_V"] <= 1e-12 * n and r["rho_U"] <= 1e-12 * n, r
    assert 1 <= sw < 128


def test_precond_agrees_with_plain(cuda_device):
    a = W.spectrum_matrix(1024, 256, W.geometric_sigma(256, 1e-6), 48)
    cfg = jsvd.default_config(epsilon=1e-14)
    pu, ps, pv, psw = jsvd.precond_svd(a, cfg)
    qu, qs, qv, qsw = jsvd.plain_svd(a, cfg)
    assert O.sigma_errors(ps, qs)["normwise"] <= 4e-15 * 256
    # the two paths order sigma differently; match columns by sigma
    ip, iq = np.argsort(-ps), np.argsort(-qs)
    big = ps[ip] > 1e-3  # well-separated part of the spectrum
    assert O.columns_match_up_to_sign(pv[:, ip][:, big], qv[:, iq][:, big], 1e-8) <= 1e-8


def test_precond_device_entry(cuda_device):
    import torch

    a = W.spectrum_matrix(600, 300, W.geometric_sigma(300, 1e-4), 49)
    da = torch.from_numpy(a).to(cuda_device)
    du = torch.empty((600, 300), dtype=torch.float64, device=cuda_device)
    ds = torch.empty(300, dtype=torch.float64, device=cuda_device)
    dv = torch.empty((300, 300), dtype=torch.float64, device=cuda_device)
    jsvd.precond_stats_reset()
    sw = jsvd.precond_svd_device(da.data_ptr(), 600, 300, du.data_ptr(), ds.data_ptr(), dv.data_ptr(),
                                 jsvd.default_config(epsilon=1e-14))
    host = jsvd.precond_svd(a, jsvd.default_config(epsilon=1e-14))
    assert sw == host[3]
    assert np.array_equal(ds.cpu().numpy(), host[1])
    st = jsvd.precond_stats()
    assert st.solves >= 1 and st.fallbacks == 0 and st.qr_ms > 0 and st.jacobi_ms > 0


@pytest.mark.parametrize("name,make,kappa", [CASES[0], CASES[3], CASES[4]], ids=[CASES[0][0], CASES[3][0], CASES[4][0]])
def test_precond_gram_stop_matches_full_sweeps(cuda_device, name, make, kappa):
    """At epsilon 1e-10 the final rotation-free sweep is replaced by the Gram
    test: same sweep count, results within the precond tolerance of the run
    that executes every sweep."""
    a = make()
    n = a.shape[1]
    cfg = jsvd.default_config(epsilon=1e-10)
    jsvd.plain_stats_reset()
    gu, gs, gv, gsw = jsvd.precond_svd(a, cfg)
    checks = jsvd.plain_stats().gram_checks
    jsvd.plain_stats_reset()
    jsvd.precond_set_gram_stop(False)
    try:
        fu, fs, fv, fsw = jsvd.precond_svd(a, cfg)
    finally:
        jsvd.precond_set_gram_stop(True)
    assert jsvd.plain_stats().gram_checks == 0
    if name == CASES[0][0]:
        assert checks >= 1  # the 2048 x 512 graded case reaches the test before converging
    assert gsw == fsw
    assert O.sigma_errors(gs, fs)["normwise"] <= 1e-15 * max(n, 100)
    r = O.residuals(a, gu, gs, gv)
    assert r["rho_A"] <= 1e-11 * n and r["rho_V"] <= 1e-12 * n and r["rho_U"] <= 1e-10 * n, r


def test_precond_graph_replay_identical(cuda_device):
    """The QR stage runs directly on a shape's first solve and from captured
    graphs afterwards: the results are the same bytes."""
    a = W.spectrum_matrix(1500, 400, W.geometric_sigma(400, 1e-6), 77)
    cfg = jsvd.default_config(epsilon=1e-14)
    runs = [jsvd.precond_svd(a, cfg) for _ in range(3)]
    for r in runs[1:]:
        assert r[3] == runs[0][3]
        for x, y in zip(r[:3], runs[0][:3]):
            assert np.array_equal(x, y)


def test_precond_cluster_subspaces_agree_with_lapack(cuda_device):
    """Graded spectrum 1 .. 1e-10 with runs of 8 singular values 1e-10 apart
    (the 16384 x 8192 workload's shape of spectrum, at 300 x 160): cluster
    subspaces of V with sigma >= 1e-3 sigma_max agree with LAPACK's to
    sin(theta) <= 1e-10 (single vectors are not defined inside a cluster)."""
    n, m = 160, 300
    s = W.graded_clustered_sigma(n, clusters=4, size=8, gap=1e-10)
    a = W.spectrum_matrix(m, n, s, 77)
    _, sp, vp, _ = jsvd.precond_svd(a, jsvd.default_config(epsilon=1e-14))
    _, sl, vt = np.linalg.svd(a, full_matrices=False)
    r = O.cluster_subspace_sines(vp, sp, vt.T, sl, floor=1e-3)
    assert r["largest_cluster"] == 8 and r["max_sine"] <= 1e-10, r
