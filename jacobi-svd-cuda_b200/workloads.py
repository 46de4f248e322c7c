"""Seeded synthetic inputs for the five workloads of the one-sided Jacobi SVD.

No public dataset is involved; every matrix is generated from a seed:

* ``gaussian_splitmix(m, n, seed)``: i.i.d. N(0,1) entries from SplitMix64 +
  Box-Muller (reproducible in any language), e.g. the 512 x 512 plain case.
* ``spectrum_matrix(m, n, sigma, seed)``: A = U diag(sigma) V^T with Haar U
  (orthonormal columns) and Haar V, e.g. 4096 x 1024 with sigma geometric
  from 1 to 1e-6.
* ``batch_workload(count, seed)``: the mixed-size batch (m ~ U{16..256},
  n ~ U{8..m}, kappa log-uniform in [1e1, 1e6], sigma log-uniform in
  [1/kappa, 1]), stored as FP32.
* ``serving_requests(...)``: Poisson arrivals with m log-uniform in 32..2048,
  n = floor(m * U(0.25, 1)), kappa log-uniform in [1e2, 1e8].
* ``graded_clustered_sigma(n)``: sigma_i = 10^(-10 i / n) with 8 clusters of
  16 near-equal values (relative gaps 1e-10).
"""
from __future__ import annotations

import math

import numpy as np

_MASK = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed: int, count: int) -> np.ndarray:
    """`count` outputs of SplitMix64 (Steele, Lea, Flood 2014) from `seed`."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, count + 1, dtype=np.uint64)
        z = (np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)) & _MASK
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _MASK
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _MASK
        return z ^ (z >> np.uint64(31))


def gaussian_splitmix(m: int, n: int, seed: int = 1) -> np.ndarray:
    """Row-major m x n N(0,1) matrix: uniforms u = (x >> 11) * 2^-53 from SplitMix64,
    Box-Muller pairs (r cos t, r sin t) with r = sqrt(-2 ln(1 - u1)), t = 2 pi u2."""
    count = m * n
    pairs = (count + 1) // 2
    bits = splitmix64(seed, 2 * pairs)
    u = (bits >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    u1, u2 = u[0::2], u[1::2]
    r = np.sqrt(-2.0 * np.log1p(-u1))
    t = 2.0 * math.pi * u2
    z = np.empty(2 * pairs)
    z[0::2] = r * np.cos(t)
    z[1::2] = r * np.sin(t)
    return z[:count].reshape(m, n)


def haar(m: int, n: int, rng: np.random.Generator) -> np.ndarray:
    """m x n matrix with Haar-distributed orthonormal columns (QR of a Gaussian, diag(R) > 0)."""
    g = rng.standard_normal((m, n))
    q, r = np.linalg.qr(g)
    return q * np.sign(np.diag(r))[None, :]


def spectrum_matrix(m: int, n: int, sigma: np.ndarray, seed: int) -> np.ndarray:
    """A = U diag(sigma) V^T, U (m x n) and V (n x n) Haar, formed in FP64."""
    rng = np.random.default_rng(seed)
    u = haar(m, n, rng)
    v = haar(n, n, rng)
    return (u * np.asarray(sigma)[None, :]) @ v.T


def geometric_sigma(n: int, lo: float = 1e-6) -> np.ndarray:
    """sigma_i = lo^(i/(n-1)), i = 0..n-1 (1 down to lo)."""
    if n == 1:
        return np.ones(1)
    return lo ** (np.arange(n) / (n - 1))


def tall_case(seed: int = 2, m: int = 4096, n: int = 1024, kappa: float = 1e6) -> tuple[np.ndarray, np.ndarray]:
    """The tall blocked case: A (m x n) with sigma geometric from 1 to 1/kappa; returns (A, sigma)."""
    s = geometric_sigma(n, 1.0 / kappa)
    return spectrum_matrix(m, n, s, seed), s


def batch_shapes(count: int, seed: int = 3, m_lo: int = 16, m_hi: int = 256, n_lo: int = 8):
    rng = np.random.default_rng(seed)
    ms = rng.integers(m_lo, m_hi + 1, size=count)
    ns = np.array([rng.integers(n_lo, m + 1) for m in ms])
    kappas = 10.0 ** rng.uniform(1.0, 6.0, size=count)
    return ms, ns, kappas, rng


def batch_workload(count: int, seed: int = 3, m_lo: int = 16, m_hi: int = 256, n_lo: int = 8,
                   dtype=np.float32) -> list[np.ndarray]:
    """Mixed-size batch; each A = U diag(sigma) V^T with sigma log-uniform in [1/kappa, 1],
    stored as `dtype` (FP32 by default)."""
    ms, ns, kappas, rng = batch_shapes(count, seed, m_lo, m_hi, n_lo)
    out = []
    for m, n, kappa in zip(ms, ns, kappas):
        s = np.sort(10.0 ** rng.uniform(-math.log10(kappa), 0.0, size=n))[::-1]
        s[0] = 1.0
        u = haar(int(m), int(n), rng)
        v = haar(int(n), int(n), rng)
        out.append(((u * s[None, :]) @ v.T).astype(dtype))
    return out


def serving_requests(count: int, rate: float, seed: int = 4, m_lo: int = 32, m_hi: int = 2048):
    """Poisson arrival times (s) and shapes/kappas of `count` requests at `rate` req/s."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count)
    t = np.cumsum(gaps) - gaps[0]
    ms = np.floor(np.exp(rng.uniform(math.log(m_lo), math.log(m_hi), size=count))).astype(int)
    ns = np.maximum(1, np.floor(ms * rng.uniform(0.25, 1.0, size=count))).astype(int)
    kappas = 10.0 ** rng.uniform(2.0, 8.0, size=count)
    return t, ms, ns, kappas, rng


def request_matrix(m: int, n: int, kappa: float, rng: np.random.Generator) -> np.ndarray:
    s = np.sort(10.0 ** rng.uniform(-math.log10(kappa), 0.0, size=n))[::-1]
    s[0] = 1.0
    return (haar(m, n, rng) * s[None, :]) @ haar(n, n, rng).T


def graded_clustered_sigma(n: int, clusters: int = 8, size: int = 16, gap: float = 1e-10) -> np.ndarray:
    """sigma_i = 10^(-10 i / n), then `clusters` runs of `size` values set to c (1 + k gap)."""
    s = 10.0 ** (-10.0 * np.arange(n) / n)
    if n >= clusters * size * 2:
        centres = np.linspace(n // (clusters + 1), n - n // (clusters + 1) - size, clusters).astype(int)
        for c0 in centres:
            c = s[c0]
            s[c0: c0 + size] = c * (1.0 + gap * np.arange(size))
    return np.sort(s)[::-1]


def batch_workload_torch(count: int, seed: int = 3, device=None, m_lo: int = 16, m_hi: int = 256,
                         n_lo: int = 8) -> list[np.ndarray]:
    """Same distribution as batch_workload, generated with torch (FP64 QR on
    `device`, e.g. a GPU, for speed) and stored as FP32.  Shapes and kappas
    come from the numpy stream of `seed`; the Gaussian factors from a torch
    generator seeded with `seed`."""
    import torch

    ms, ns, kappas, rng = batch_shapes(count, seed, m_lo, m_hi, n_lo)
    dev = torch.device(device) if device is not None else torch.device("cpu")
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    out = []
    for m, n, kappa in zip(ms, ns, kappas):
        m, n = int(m), int(n)
        s = np.sort(10.0 ** rng.uniform(-math.log10(kappa), 0.0, size=n))[::-1].copy()
        s[0] = 1.0
        gu = torch.randn((m, n), generator=g, dtype=torch.float64, device=dev)
        gv = torch.randn((n, n), generator=g, dtype=torch.float64, device=dev)
        qu, ru = torch.linalg.qr(gu)
        qv, rv = torch.linalg.qr(gv)
        qu = qu * torch.sign(torch.diagonal(ru))[None, :]
        qv = qv * torch.sign(torch.diagonal(rv))[None, :]
        st = torch.from_numpy(s).to(dev)
        a = (qu * st[None, :]) @ qv.T
        out.append(a.to(torch.float32).cpu().numpy())
    return out
