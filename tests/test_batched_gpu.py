"""Batched solver (one persistent launch per size class) against the oracle.

Every matrix of a batch uses the plain path's arithmetic, so each result must
be bit-identical to the oracle on the same FP64 (or FP32-promoted) input:
same sigma, U and V bytes and sweep count.  The batches span the five size
classes (A and V in <= 48 KiB, <= 100 KiB, <= ~226 KiB of shared memory; A
alone in shared memory; A and V in global memory) and odd/even n.
"""
import numpy as np
import pytest

import jsvd
import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu

SHAPES = [(16, 8), (17, 17), (40, 33), (60, 50), (31, 1), (2, 2), (100, 90), (120, 100), (129, 64),
          (256, 200), (256, 256), (250, 131), (8, 8), (64, 63), (200, 9), (160, 120), (161, 117)]


def _mats(seed, f32):
    rng = np.random.default_rng(seed)
    out = []
    for m, n in SHAPES:
        a = rng.standard_normal((m, n))
        out.append(a.astype(np.float32) if f32 else a)
    return out


@pytest.mark.parametrize("f32", [False, True])
def test_batch_bitwise_vs_oracle(cuda_device, f32):
    mats = _mats(11 + int(f32), f32)
    b = jsvd.DeviceBatch(mats, cuda_device, f32=f32, want_u=True)
    b.solve(jsvd.default_config(epsilon=1e-13))
    got = b.results()
    for a, (u, s, v, sw) in zip(mats, got):
        eu, es, ev, esw = O.plain_svd(a.astype(np.float64), eps=1e-13, variant=jsvd.arith_variant(), threads=4)
        assert sw == esw, a.shape
        assert np.array_equal(s, es), a.shape
        assert np.array_equal(v, ev), a.shape
        assert np.array_equal(u, eu), a.shape


# members of the three classes that clusters can take, odd and even n, and
# columns longer than the 256-row reduction chunk; each needs a different
# cluster size (2, 4 or 8 CTAs) or none
CLUSTER_SHAPES = [(100, 90), (120, 100), (129, 64), (160, 120), (161, 117), (170, 110), (200, 150), (250, 131),
                  (256, 200), (255, 255), (256, 256), (231, 229), (240, 15), (256, 9), (600, 120), (517, 131)]


def test_batch_cluster_classes_bitwise(cuda_device):
    """Members solved by thread-block clusters (classes 3 and 4 by default,
    class 2 as well, or none) give the same bytes and sweep counts, and they
    are the oracle's."""
    rng = np.random.default_rng(31)
    mats = [rng.standard_normal(s) for s in CLUSTER_SHAPES]
    cfg = jsvd.default_config(epsilon=1e-13)
    runs = []
    old = jsvd.batch_set_cluster_classes(0)
    try:
        for mask in (0, (1 << 3) | (1 << 4), (1 << 2) | (1 << 3) | (1 << 4)):
            jsvd.batch_set_cluster_classes(mask)
            b = jsvd.DeviceBatch(mats, cuda_device, want_u=True)
            b.solve(cfg)
            runs.append(b.results())
    finally:
        jsvd.batch_set_cluster_classes(old)
    for k, a in enumerate(mats):
        for other in runs[1:]:
            assert runs[0][k][3] == other[k][3], a.shape
            for x, y in zip(runs[0][k][:3], other[k][:3]):
                assert np.array_equal(x, y), a.shape
    for a, (u, s, v, sw) in list(zip(mats, runs[1]))[::3]:
        eu, es, ev, esw = O.plain_svd(a, eps=1e-13, variant=jsvd.arith_variant(), threads=4)
        assert sw == esw and np.array_equal(s, es) and np.array_equal(v, ev) and np.array_equal(u, eu), a.shape


def test_batch_workload_sample_accuracy(cuda_device):
    """A sample of the mixed-size FP32 batch workload: sigma against LAPACK on
    the FP32-promoted input and orthogonality of V."""
    mats = W.batch_workload(64, seed=3)
    b = jsvd.DeviceBatch(mats, cuda_device, f32=True)
    b.solve(jsvd.default_config(epsilon=1e-14))
    for a, (_, s, v, sw) in zip(mats, b.results()):
        ref = np.linalg.svd(a.astype(np.float64), compute_uv=False)
        e = O.sigma_errors(s, ref)
        assert e["normwise"] < 1e-13
        assert O.residuals(a.astype(np.float64), None, s, v)["rho_V"] < 1e-12
        assert 1 <= sw < 128


def test_batch_tuning_and_empty(cuda_device):
    mats = _mats(5, False)[:6]
    b = jsvd.DeviceBatch(mats, cuda_device)
    b.solve(jsvd.default_config(epsilon=1e-12), tuning=[(128, 2), (512, 1), (256, 1), (256, 1)])
    ref = jsvd.DeviceBatch(mats, cuda_device)
    ref.solve(jsvd.default_config(epsilon=1e-12))
    for x, y in zip(b.results(), ref.results()):
        assert np.array_equal(x[1], y[1]) and np.array_equal(x[2], y[2]) and x[3] == y[3]
    empty = jsvd.DeviceBatch([np.zeros((3, 2))], cuda_device)
    empty.count = 0
    empty.solve()


# two matrices per shape; the shapes fall in all five size classes
AUTOTUNE_SHAPES = [(16, 8), (40, 33), (31, 1), (64, 63), (60, 50), (100, 90), (120, 100), (160, 120),
                   (170, 110), (256, 200), (200, 150)]


def test_batch_autotune(cuda_device):
    """The autotuner times every class, leaves the batch statistics alone,
    and its chosen shapes give the same bytes as the built-in ones."""
    rng = np.random.default_rng(21)
    mats = [rng.standard_normal(s) for s in AUTOTUNE_SHAPES for _ in range(2)]
    b = jsvd.DeviceBatch(mats, cuda_device, want_u=True)
    cfg = jsvd.default_config(epsilon=1e-13)
    b.solve(cfg)
    ref = b.results()
    before = jsvd.batch_stats()
    rep = b.autotune(cfg, sample=0, reps=1)
    after = jsvd.batch_stats()
    assert after.calls == before.calls and after.kernel_ms == before.kernel_ms
    assert sum(rep.members) == len(mats) and all(x > 0 for x in rep.members)
    builtin = jsvd.batch_builtin_tuning()
    for c in range(5):
        assert rep.sampled[c] == rep.members[c]
        assert rep.candidates[c] >= 2
        assert (rep.builtin[c].threads, rep.builtin[c].ctas_per_sm, rep.builtin[c].max_ctas) == builtin[c]
        assert 0.0 < rep.best_ms[c] <= rep.builtin_ms[c]
        t = rep.best[c]
        assert t.threads in (128, 256, 512) and t.ctas_per_sm >= 1 and t.max_ctas >= 0
    best = [(t.threads, t.ctas_per_sm, t.max_ctas) for t in rep.best]
    b.solve(cfg, tuning=best)
    for x, y in zip(b.results(), ref):
        assert x[3] == y[3]
        for p, q in zip(x[:3], y[:3]):
            assert np.array_equal(p, q)
    one = b.autotune(cfg, sample=1, reps=1)
    assert list(one.sampled) == [1] * 5
