"""Blocked mixed-precision path on the GPU (tcgen05 3xTF32 phase, FP64 block
eigen-solves, FP64 DMMA refinement).

Kernel level (jsvd_mixed_test_round), against numpy's FP64 products of the
same block pairs:
  * FP64 Gram: |error| <= 8 m u (|P|^T |P|) elementwise; FP64 rotation:
    ||dP||_F <= 512 u ||P||_F;
  * tensor-core Gram: |g - g_ref|_ij <= 2e-6 sqrt(g_ii g_jj) (3xTF32 operands
    keep about 21 bits, accumulation is FP32);
  * tensor-core rotation: ||dP||_F <= 2e-6 ||P||_F.
End to end, not bit-identical to the plain path (another algorithm), held to
the QR-preconditioned path's tolerances against LAPACK on the same input:
sigma normwise |d sigma_i| / sigma_max <= 1e-15 max(n, 100), per-value
relative <= 1e-13 n max(1, kappa 1e-6), rho_A <= 1e-13 n, ||U^T U - I||_F and
||V^T V - I||_F <= 1e-12 n.
"""
import numpy as np
import pytest

import jsvd
import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu

U53 = 2.0 ** -53


def block_pair(nb, r, k):
    """Pair k of round r of the fixed-head circle over nb (even) blocks."""
    L = nb - 1
    i, i2 = k, nb - 1 - k
    p = 0 if i == 0 else 1 + ((i - 1 - r) % L)
    q = 1 + ((i2 - 1 - r) % L)
    return p, q


def pair_cols(p, q):
    return np.r_[p * 32:(p + 1) * 32, q * 32:(q + 1) * 32]


def _dev(x, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x)).to(dev)


@pytest.mark.parametrize("rows,cols,rnd", [(256, 256, 0), (384, 256, 3), (1024, 512, 7)])
def test_gram_kernels(cuda_device, rows, cols, rnd):
    import torch

    rng = np.random.default_rng(rows + cols + rnd)
    # graded columns: the scaled off-diagonal bound must hold for small columns too
    X = rng.standard_normal((rows, cols)) * np.logspace(0, -3, cols)
    nb = cols // 32
    dX = _dev(X.T, cuda_device)  # column-major
    for kind in (0, 1):
        g = torch.zeros((nb // 2, 64, 64), dtype=torch.float64, device=cuda_device)
        jsvd.mixed_test_round(kind, dX.data_ptr(), rows, cols, rnd, g.data_ptr())
        G = g.cpu().numpy().transpose(0, 2, 1)  # column-major 64 x 64 per pair
        for k in range(nb // 2):
            P = X[:, pair_cols(*block_pair(nb, rnd, k))]
            ref = P.T @ P
            if kind == 1:
                bound = 8 * rows * U53 * (np.abs(P).T @ np.abs(P))
                assert np.all(np.abs(G[k] - ref) <= bound), (k, np.max(np.abs(G[k] - ref) / bound))
            else:
                d = np.sqrt(np.outer(np.diag(ref), np.diag(ref)))
                err = np.max(np.abs(G[k] - ref) / d)
                assert err <= 2e-6, (k, err)


@pytest.mark.parametrize("rows,cols,rnd", [(256, 256, 1), (640, 384, 4)])
@pytest.mark.parametrize("kind", [2, 3], ids=["tensor_core", "fp64"])
def test_rotation_kernels(cuda_device, rows, cols, rnd, kind):
    rng = np.random.default_rng(rows * cols + rnd)
    X = rng.standard_normal((rows, cols))
    nb = cols // 32
    Ws = np.stack([np.linalg.qr(rng.standard_normal((64, 64)))[0] for _ in range(nb // 2)])
    dX = _dev(X.T, cuda_device)
    dW = _dev(Ws.transpose(0, 2, 1), cuda_device)  # column-major W per pair
    jsvd.mixed_test_round(kind, dX.data_ptr(), rows, cols, rnd, dW.data_ptr())
    Y = dX.cpu().numpy().T
    for k in range(nb // 2):
        c = pair_cols(*block_pair(nb, rnd, k))
        ref = X[:, c] @ Ws[k]
        err = np.linalg.norm(Y[:, c] - ref) / np.linalg.norm(X[:, c])
        assert err <= (2e-6 if kind == 2 else 512 * U53), (k, err)


CASES = [
    ("tall_k1e6", lambda: W.spectrum_matrix(2048, 512, W.geometric_sigma(512, 1e-6), 41), 1e6),
    ("square_gauss", lambda: W.gaussian_splitmix(300, 300, 42), 1e4),
    ("tall_k1e8", lambda: W.spectrum_matrix(1000, 200, W.geometric_sigma(200, 1e-8), 43), 1e8),
    ("tall_k1e10_graded", lambda: W.spectrum_matrix(1200, 300, W.graded_clustered_sigma(300, 2, 16), 44), 1e10),
    ("odd_cols", lambda: W.gaussian_splitmix(257, 129, 45), 1e3),
    ("narrow_falls_back", lambda: W.gaussian_splitmix(200, 100, 46), 1e3),
]


def _check(a, res, kappa):
    u, s, v, sw = res
    n = a.shape[1]
    ref = np.linalg.svd(a, compute_uv=False)
    e = O.sigma_errors(s, ref)
    assert e["normwise"] <= 1e-15 * max(n, 100), e
    assert e["max_rel"] <= 1e-13 * n * max(1.0, kappa * 1e-6), e
    r = O.residuals(a, u, s, v)
    assert r["rho_A"] <= 1e-13 * n and r["rho_V"] <= 1e-12 * n and r["rho_U"] <= 1e-12 * n, r
    assert 1 <= sw < 128


@pytest.mark.parametrize("name,make,kappa", CASES, ids=[c[0] for c in CASES])
def test_mixed_accuracy(cuda_device, name, make, kappa):
    """Both phases (a tensor-core cap of 4 sweeps, whatever the width's
    automatic choice) on every case."""
    a = make()
    jsvd.mixed_set_options(tc_max_sweeps=4)
    jsvd.mixed_stats_reset()
    try:
        res = jsvd.mixed_svd(a, jsvd.default_config(epsilon=1e-14))
    finally:
        jsvd.mixed_set_options(None)
    _check(a, res, kappa)
    st = jsvd.mixed_stats()
    if a.shape[1] >= 128:
        assert st.solves == 1 and st.tc_sweeps >= 1 and st.f64_sweeps >= 1, (st.tc_sweeps, st.f64_sweeps)
        assert st.tc_discarded == 0


@pytest.mark.parametrize("m,n", [(600, 200), (1024, 384), (2048, 1024), (3000, 1500)])
def test_mixed_automatic_options(cuda_device, m, n):
    """The default (automatic) options, resolved from the built-in tuning
    table by width: accurate, and the tensor-core phase runs exactly when the
    width's entry gives it sweeps."""
    a = W.spectrum_matrix(m, n, W.geometric_sigma(n, 1e-6), 60 + n)
    jsvd.mixed_set_options(None)
    jsvd.mixed_stats_reset()
    res = jsvd.mixed_svd(a, jsvd.default_config(epsilon=1e-14))
    _check(a, res, 1e6)
    st = jsvd.mixed_stats()
    r = jsvd.mixed_resolved_options(n)
    assert st.solves == 1 and st.f64_sweeps >= 1
    assert (st.tc_sweeps >= 1) == (r.tc_max_sweeps > 0) and st.tc_sweeps <= r.tc_max_sweeps


@pytest.mark.parametrize("opts", [dict(tc_max_sweeps=0), dict(precondition=0), dict(inner_sweeps=1),
                                  dict(gram_splits=1), dict(tc_max_sweeps=2), dict(sort=0)],
                         ids=["fp64_only", "no_qr", "inner1", "splits1", "tc2", "unsorted"])
def test_mixed_options(cuda_device, opts):
    a = W.spectrum_matrix(1024, 384, W.geometric_sigma(384, 1e-6), 51)
    jsvd.mixed_set_options(**opts)
    try:
        res = jsvd.mixed_svd(a, jsvd.default_config(epsilon=1e-14))
    finally:
        jsvd.mixed_set_options(None)
    _check(a, res, 1e6)


def test_mixed_agrees_with_plain(cuda_device):
    a = W.spectrum_matrix(1024, 256, W.geometric_sigma(256, 1e-6), 48)
    cfg = jsvd.default_config(epsilon=1e-14)
    mu, ms, mv, msw = jsvd.mixed_svd(a, cfg)
    qu, qs, qv, qsw = jsvd.plain_svd(a, cfg)
    assert O.sigma_errors(ms, qs)["normwise"] <= 4e-15 * 256
    im, iq = np.argsort(-ms), np.argsort(-qs)
    big = ms[im] > 1e-3
    assert O.columns_match_up_to_sign(mv[:, im][:, big], qv[:, iq][:, big], 1e-8) <= 1e-8


def test_mixed_device_entry_deterministic(cuda_device):
    import torch

    a = W.spectrum_matrix(600, 300, W.geometric_sigma(300, 1e-4), 49)
    da = _dev(a, cuda_device)
    du = torch.empty((600, 300), dtype=torch.float64, device=cuda_device)
    ds = torch.empty(300, dtype=torch.float64, device=cuda_device)
    dv = torch.empty((300, 300), dtype=torch.float64, device=cuda_device)
    cfg = jsvd.default_config(epsilon=1e-14)
    sw = jsvd.mixed_svd_device(da.data_ptr(), 600, 300, du.data_ptr(), ds.data_ptr(), dv.data_ptr(), cfg)
    host = jsvd.mixed_svd(a, cfg)
    assert sw == host[3]
    assert np.array_equal(ds.cpu().numpy(), host[1])
    assert np.array_equal(dv.cpu().numpy(), host[2])


def test_mixed_cluster_subspaces_agree_with_lapack(cuda_device):
    """Graded spectrum 1 .. 1e-10 with runs of 8 values 1e-10 apart (the
    16384 x 8192 workload's spectrum shape at 600 x 320): cluster subspaces of
    V with sigma >= 1e-3 sigma_max agree with LAPACK's to sin(theta) <= 1e-10."""
    n, m = 320, 600
    s = W.graded_clustered_sigma(n, clusters=4, size=8, gap=1e-10)
    a = W.spectrum_matrix(m, n, s, 78)
    _, sp, vp, _ = jsvd.mixed_svd(a, jsvd.default_config(epsilon=1e-14))
    _, sl, vt = np.linalg.svd(a, full_matrices=False)
    r = O.cluster_subspace_sines(vp, sp, vt.T, sl, floor=1e-3)
    assert r["largest_cluster"] == 8 and r["max_sine"] <= 1e-10, r
