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


def _jacobi_in(x: np.ndarray, eps: float, dtype, max_sweeps: int = 60):
    """Cyclic one-sided Jacobi carried out in `dtype` (the reference's
    schedule, rotation test and Rutishauser angle, one round at a time);
    returns the rotated columns, V and the sweep count."""
    import oracle as O

    a = x.astype(dtype).copy()
    n = a.shape[1]
    v = np.eye(n, dtype=dtype)
    rounds = [(np.array([p for p, _ in r]), np.array([q for _, q in r])) for r in O.schedule(n)]
    for sweep in range(1, max_sweeps + 1):
        rotated = False
        for p, q in rounds:
            ap, aq = a[:, p], a[:, q]
            app, aqq = np.einsum("ij,ij->j", ap, ap), np.einsum("ij,ij->j", aq, aq)
            apq = np.einsum("ij,ij->j", ap, aq)
            rot = (np.abs(apq) > eps * np.sqrt(np.maximum(app, 0) * np.maximum(aqq, 0))) & (np.abs(apq) > 1e-300)
            if not rot.any():
                continue
            rotated = True
            zeta = (aqq - app) / (2 * np.where(rot, apq, 1))
            t = np.sign(zeta + (zeta == 0)) / (np.abs(zeta) + np.sqrt(1 + zeta * zeta))
            c = np.where(rot, 1 / np.sqrt(1 + t * t), 1).astype(dtype)
            s = np.where(rot, c * t, 0).astype(dtype)
            a[:, p], a[:, q] = c * ap - s * aq, s * ap + c * aq
            vp, vq = v[:, p], v[:, q]
            v[:, p], v[:, q] = c * vp - s * vq, s * vp + c * vq
        if not rotated:
            return a, v, sweep
    return a, v, max_sweeps


def test_fp32_phase_does_not_save_fp64_sweeps():
    """On the triangular factor of the tall case (1024 x 256 version, kappa
    1e6, after two QR factorisations): FP64 Jacobi alone takes 9 sweeps; an
    FP32 phase to eps = 1e-6 takes 8 (sigma to 1.4e-5) and FP64 refinement on
    X V32 (V32 re-orthogonalised in FP64) 3 more - 11 sequential sweeps, each
    as latency-bound as an FP64 one."""
    import os

    import oracle as O
    import workloads as W

    a, s_true = W.tall_case(seed=2, m=1024, n=256, kappa=1e6)
    _, r = np.linalg.qr(a)
    _, p = np.linalg.qr(r.T)
    x = p.T
    _, s64, _, sw64 = O.plain_svd(x, eps=1e-14, threads=os.cpu_count() or 1)
    a32, v32, sw32 = _jacobi_in(x, 1e-6, np.float32)
    s32 = np.linalg.norm(a32.astype(np.float64), axis=0)
    vq, _ = np.linalg.qr(v32.astype(np.float64))
    _, sref, _, swref = O.plain_svd(x @ vq, eps=1e-14, threads=os.cpu_count() or 1)
    assert 1e-6 < O.sigma_errors(s32, s_true)["max_rel"] < 1e-4  # the FP32 phase's level
    assert O.sigma_errors(sref, s_true)["max_rel"] < 1e-10 and O.sigma_errors(s64, s_true)["max_rel"] < 1e-10
    assert swref >= 2 and sw32 + swref > sw64, (sw64, sw32, swref)
