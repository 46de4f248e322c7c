"""Why the tensor-core Gram products cannot replace the FP64 sweep (host,
numpy emulation, no GPU).

The rotation test of the reference (src/kernels.cu:503-505) asks whether
|g_pq| > eps * sqrt(g_pp g_qq) with eps = 1e-14 for the workloads measured
here.  A tcgen05 GEMM in split-BF16x3 or 3xTF32 form multiplies split terms
exactly but accumulates in FP32, so the Gram entry it returns carries an
error of order 2^-24 times its partial sums: for two unit columns of 4096
rows with cosine 1e-12 the emulation gives 1.5e-9 (split-BF16x3) and 2.5e-9
(3xTF32), five orders of magnitude above eps = 1e-14 and three above the
cosine being tested.  A tensor-core phase can drive the columns to about that
level of orthogonality and no further; FP64 sweeps still have to decide the
rotations below it.  The emulation below is bit-exact for the products
(8- or 11-bit significands multiply exactly into FP32's 24 bits) and
accumulates in FP32 in blocks of 16 products, as one MMA k-step does.
"""
import numpy as np


def _round_significand(x: np.ndarray, bits: int) -> np.ndarray:
    """Round float32 values to `bits` significand bits (sign and exponent kept),
    round-to-nearest-even: BF16 is 8 bits, TF32 is 11."""
    u = x.astype(np.float32).view(np.uint32).astype(np.uint64)
    drop = 24 - bits
    half = np.uint64(1) << np.uint64(drop - 1)
    lsb = (u >> np.uint64(drop)) & np.uint64(1)
    u = (u + half - np.uint64(1) + lsb) & ~((np.uint64(1) << np.uint64(drop)) - np.uint64(1))
    return u.astype(np.uint32).view(np.float32)


def _split3(x: np.ndarray, bits: int):
    """x ~ hi + mid + lo, each term with `bits` significand bits."""
    hi = _round_significand(x.astype(np.float32), bits)
    r1 = (x - hi.astype(np.float64)).astype(np.float32)
    mid = _round_significand(r1, bits)
    r2 = (x - hi.astype(np.float64) - mid.astype(np.float64)).astype(np.float32)
    lo = _round_significand(r2, bits)
    return hi, mid, lo


def _tensor_core_dot(x: np.ndarray, y: np.ndarray, bits: int) -> float:
    """Dot product as a split-by-3 tensor-core GEMM computes it: the six
    leading cross terms, each product exact in FP32, summed in FP32 in
    k-blocks of 16."""
    xs, ys = _split3(x, bits), _split3(y, bits)
    terms = [(0, 0), (0, 1), (1, 0), (1, 1), (0, 2), (2, 0)]
    acc = np.float32(0.0)
    for i, j in terms:
        prod = (xs[i] * ys[j]).astype(np.float32)  # exact: 2 * bits <= 24
        for k in range(0, prod.size, 16):
            acc = np.float32(acc + np.float32(np.sum(prod[k:k + 16], dtype=np.float32)))
    return float(acc)


def _near_orthogonal_pair(m: int, cos: float, seed: int):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((m, 2)))
    return q[:, 0], cos * q[:, 0] + np.sqrt(1.0 - cos * cos) * q[:, 1]


def test_fp32_accumulated_gram_cannot_resolve_the_rotation_test():
    # unit columns with cosine 1e-12: at eps = 1e-14 the pair rotates, and its
    # angle is computed from g_pq, so g_pq must be known well below 1e-12
    m, cos = 4096, 1e-12
    x, y = _near_orthogonal_pair(m, cos, 5)
    exact = float(np.dot(x, y))
    assert abs(exact - cos) < 1e-15  # FP64 resolves it
    for bits in (8, 11):  # split-BF16x3, 3xTF32
        got = _tensor_core_dot(x, y, bits)
        err = abs(got - exact)  # unit columns: err is relative to sqrt(g_pp g_qq)
        assert err > 1e-11, (bits, err)  # far above both eps and the cosine itself
        assert err < 1e-6, (bits, err)  # at the FP32-accumulation level


def test_split_products_are_exact_in_fp32():
    """The emulation's premise: a BF16 x BF16 or TF32 x TF32 product has at
    most 22 significand bits and is exact in FP32."""
    rng = np.random.default_rng(1)
    a = rng.standard_normal(1000)
    for bits in (8, 11):
        ha = _round_significand(a.astype(np.float32), bits)
        hb = _round_significand((a[::-1] * 3.7).astype(np.float32), bits)
        assert np.array_equal((ha * hb).astype(np.float64), ha.astype(np.float64) * hb.astype(np.float64))
