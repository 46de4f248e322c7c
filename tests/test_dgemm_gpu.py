"""The library's FP64 GEMM (DMMA tensor cores, mma.sync m8n8k4 f64) on the GPU.

It replaces the cuBLAS DGEMM/DSYRK calls of the QR stage, the plain path's
Gram convergence test and the products that assemble U and V.  Checked
against numpy's FP64 product of the same operands: elementwise
|C - C_ref| <= 8 k u (|op(A)| |op(B)|)_ij (the classical bound for any
summation order), every op combination, ragged sizes, beta != 0 and the
lower-triangle (DSYRK) form, which must leave the upper triangle untouched.
"""
import numpy as np
import pytest

import jsvd

pytestmark = pytest.mark.gpu

U53 = 2.0 ** -53


def _run(dev, op_a, op_b, m, n, k, alpha, beta, lower, seed):
    import torch

    rng = np.random.default_rng(seed)
    a_shape = (k, m) if op_a == "T" else (m, k)  # op(A) is m x k
    b_shape = (n, k) if op_b == "T" else (k, n)
    A = rng.standard_normal(a_shape)
    B = rng.standard_normal(b_shape)
    C0 = rng.standard_normal((m, n))
    # column-major device buffers: a torch tensor of the transpose's shape
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).to(dev)
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).to(dev)
    dC = torch.from_numpy(np.ascontiguousarray(C0.T)).to(dev)
    jsvd.dgemm_device(op_a, op_b, m, n, k, alpha, dA.data_ptr(), a_shape[0], dB.data_ptr(), b_shape[0], beta,
                      dC.data_ptr(), m, lower)
    C = dC.cpu().numpy().T
    opA = A.T if op_a == "T" else A
    opB = B.T if op_b == "T" else B
    ref = alpha * (opA @ opB) + beta * C0
    bound = 8 * k * U53 * (abs(alpha) * (np.abs(opA) @ np.abs(opB)) + abs(beta) * np.abs(C0)) + 1e-300
    if lower:
        low = np.tril(np.ones((m, n), dtype=bool))
        assert np.all(np.abs(C - ref)[low] <= bound[low])
        assert np.array_equal(C[~low], C0[~low])  # upper triangle untouched
    else:
        assert np.all(np.abs(C - ref) <= bound), np.max(np.abs(C - ref) / bound)


@pytest.mark.parametrize("op_a,op_b", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
@pytest.mark.parametrize("m,n,k", [(64, 64, 16), (100, 37, 53), (257, 129, 1000), (640, 1280, 96)])
def test_dgemm_ops(cuda_device, op_a, op_b, m, n, k):
    _run(cuda_device, op_a, op_b, m, n, k, 1.0, 0.0, False, m * 7 + n + k)


def test_dgemm_alpha_beta(cuda_device):
    _run(cuda_device, "N", "T", 300, 200, 64, -1.0, 1.0, False, 5)
    _run(cuda_device, "T", "N", 96, 96, 4096, 0.5, -2.0, False, 6)


@pytest.mark.parametrize("n,k", [(200, 5000), (1100, 64)])
def test_dgemm_lower(cuda_device, n, k):
    _run(cuda_device, "T", "N", n, n, k, 1.0, 0.0, True, n + k)
    _run(cuda_device, "N", "T", n, n, k, -1.0, 1.0, True, n + k + 1)


def test_dgemm_large_tiles(cuda_device):
    """Big enough for the 128 x 128 tile kernel (>= 296 output tiles)."""
    _run(cuda_device, "N", "N", 2560, 2048, 256, 1.0, 0.0, False, 11)
    _run(cuda_device, "T", "N", 2048, 2560, 300, 1.0, 0.0, True, 12)
