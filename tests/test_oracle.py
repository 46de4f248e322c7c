"""Oracle checks that need no GPU: schedule invariants, agreement with LAPACK,
thread invariance, and (when present) the reference's own golden outputs."""
import glob
import json
import os

import numpy as np
import pytest

import oracle as O
import workloads as W
from conftest import GOLDEN, golden_input


@pytest.mark.parametrize("n", list(range(1, 34)) + [64, 127, 128])
def test_schedule_covers_every_pair_once(n):
    rounds = O.schedule(n)
    if n < 2:
        assert rounds == []
        return
    ne = n + (n % 2)
    assert len(rounds) == ne - 1
    seen = set()
    for pairs in rounds:
        assert len(pairs) == n // 2
        cols = [c for pq in pairs for c in pq]
        assert len(cols) == len(set(cols)), "pairs of a round must be disjoint"
        for p, q in pairs:
            key = (min(p, q), max(p, q))
            assert key not in seen
            seen.add(key)
    assert len(seen) == n * (n - 1) // 2


def test_schedule_orientation_first_rounds():
    # Round 0 pairs (i, ne-1-i); round 1 after one rotation of circle[1:]
    # (kernels.cu:661-674): circle = [0, 5, 1, 2, 3, 4] for n = 6.
    r = O.schedule(6)
    assert r[0] == [(0, 5), (1, 4), (2, 3)]
    assert r[1] == [(0, 4), (5, 3), (1, 2)]
    # odd n: dummy column -1 occupies the last slot, its pair is dropped
    r5 = O.schedule(5)
    assert r5[0] == [(1, 4), (2, 3)]


@pytest.mark.parametrize("m,n", [(1, 1), (2, 2), (3, 2), (9, 9), (20, 7), (64, 33), (150, 150)])
def test_oracle_matches_lapack(m, n):
    a = W.gaussian_splitmix(m, n, seed=100 + m + n)
    u, s, v, sw = O.plain_svd(a, eps=1e-14, threads=2)
    ref = np.linalg.svd(a, compute_uv=False)
    err = O.sigma_errors(s, ref)
    assert err["max_rel"] <= 1e-13 * n
    r = O.residuals(a, u, s, v)
    assert r["rho_A"] < 1e-13 * max(1, n)
    assert r["rho_V"] < 1e-13 * max(1, n)
    assert 1 <= sw < 128


def test_oracle_thread_invariance():
    a = W.gaussian_splitmix(80, 40, seed=5)
    r1 = O.plain_svd(a, eps=1e-13, threads=1)
    r4 = O.plain_svd(a, eps=1e-13, threads=4)
    for x, y in zip(r1[:3], r4[:3]):
        assert np.array_equal(x, y)
    assert r1[3] == r4[3]


def test_oracle_unsorted_sigma_and_eps_cut():
    # U columns are zeroed when sigma <= eps (absolute cut, kernels.cu:622-627)
    a = W.gaussian_splitmix(30, 10, seed=9)
    a[:, 4] = 0.0
    u, s, v, _ = O.plain_svd(a, eps=1e-12)
    k = int(np.argmin(s))
    assert s[k] == 0.0
    assert np.all(u[:, k] == 0.0)


def test_identity_converges_in_one_sweep():
    u, s, v, sw = O.plain_svd(np.eye(12), eps=1e-9)
    assert sw == 1
    assert np.array_equal(s, np.ones(12))
    assert np.array_equal(v, np.eye(12))


def _golden_cases():
    """The fixtures recorded from the reference's own runs (summary.json);
    other .npz files in the folder (the oracle-made tall-case sigma) are not
    reference outputs."""
    summ = _summary() or {"cases": {}}
    return sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if os.path.basename(p)[:-4] in summ["cases"])


def _summary():
    p = os.path.join(GOLDEN, "summary.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


def test_golden_fixtures_present():
    assert _summary() is not None, "tests/golden/summary.json missing (run tests/golden/make_golden.py on a GPU)"
    assert len(_golden_cases()) >= 10


@pytest.mark.parametrize("path", _golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_reproduces_reference_outputs(path):
    """The oracle under the pinned FMA variant reproduces the reference's own
    outputs bit for bit (small cases keep full U/V; large ones SHA-256)."""
    summ = _summary()
    name = os.path.basename(path)[:-4]
    rec = summ["cases"][name]
    variant = summ["pinned_variant"]
    g = np.load(path)
    a = golden_input(name, g)
    u, s, v, sw = O.plain_svd(a, eps=float(g["eps"]), lanes=int(g["T"]), variant=O.VARIANTS[variant],
                              threads=os.cpu_count() or 1)
    assert sw == int(g["sweeps"])
    assert np.array_equal(s, g["sigma"])
    if "u" in g:
        assert np.array_equal(u, g["u"])
        assert np.array_equal(v, g["v"])
    else:
        import hashlib
        assert hashlib.sha256(u.tobytes()).hexdigest() == rec["u_sha256"]
        assert hashlib.sha256(v.tobytes()).hexdigest() == rec["v_sha256"]


def test_golden_comparison_rejects_planted_mistakes():
    """The bitwise golden comparison can fail: with any other FMA placement,
    or with a wrong reduction width, the oracle no longer reproduces some of
    the reference's outputs.  (Mistakes are planted in the oracle, on the CPU.)"""
    summ = _summary()
    small = [p for p in _golden_cases() if os.path.basename(p)[:-4] in ("g8x8", "g17x9", "g33x16", "g64x48")]
    assert small, "small golden cases missing"

    def reproduces(path, variant, lanes=None):
        g = np.load(path)
        name = os.path.basename(path)[:-4]
        a = golden_input(name, g)
        T = int(g["T"]) if lanes is None else lanes
        u, s, v, sw = O.plain_svd(a, eps=float(g["eps"]), lanes=T, variant=variant, threads=2)
        return sw == int(g["sweeps"]) and np.array_equal(s, g["sigma"]) and np.array_equal(u, g["u"])

    pinned = O.VARIANTS[summ["pinned_variant"]]
    assert all(reproduces(p, pinned) for p in small)
    for name, code in O.VARIANTS.items():
        if code != pinned:
            assert not all(reproduces(p, code) for p in small), name
    # T = 32 instead of 256 changes the summation order once a column has
    # more than 32 rows (up to 128 rows, T = 128 and T = 256 reduce alike:
    # the upper lanes hold zeros)
    assert not all(reproduces(p, pinned, lanes=32) for p in small), "reduction width"


def test_recorded_variant_votes_are_reproduced():
    """summary.json records, per golden case and FMA variant, whether that
    variant reproduces the reference bit for bit; the oracle reproduces each
    recorded vote (cases that store full U and V)."""
    summ = _summary()
    checked = 0
    for path in _golden_cases():
        name = os.path.basename(path)[:-4]
        g = np.load(path)
        if "u" not in g:
            continue
        a = golden_input(name, g)
        for vname, vote in summ["cases"][name]["match"].items():
            u, s, v, sw = O.plain_svd(a, eps=float(g["eps"]), lanes=int(g["T"]), variant=O.VARIANTS[vname],
                                      threads=2)
            bitwise = (sw == int(g["sweeps"]) and np.array_equal(s, g["sigma"]) and np.array_equal(u, g["u"])
                       and np.array_equal(v, g["v"]))
            assert bitwise == vote["bitwise"], (name, vname)
            checked += 1
    assert checked >= 5 * 10


def test_oracle_reproduces_reference_cli_output():
    """tests/golden/pipeline_ref_out.mat is the reference CLI's output for
    pipeline_in.mat at epsilon 1e-12: per testcase U, Sigma (1 x n) and V.
    The oracle under the pinned variant reproduces every record bit for bit."""
    import matfile

    summ = _summary()
    mats = matfile.read(os.path.join(GOLDEN, "pipeline_in.mat"))
    with open(os.path.join(GOLDEN, "pipeline_ref_out.mat"), "rb") as f:
        ref_bytes = f.read()
    out = matfile.decode(ref_bytes)
    assert len(out) == 3 * len(mats)
    records = []
    for k, a in enumerate(mats):
        u, s, v, _ = O.plain_svd(a, eps=1e-12, variant=O.VARIANTS[summ["pinned_variant"]], threads=2)
        ru, rs, rv = out[3 * k], out[3 * k + 1], out[3 * k + 2]
        assert rs.shape == (1, a.shape[1]) and np.array_equal(s, rs.ravel()), k
        assert np.array_equal(u, ru) and np.array_equal(v, rv), k
        records += [u, s.reshape(1, -1), v]
    # and the records, encoded as *.mat, are the reference CLI's file byte for byte
    assert matfile.encode(records) == ref_bytes


def test_cluster_subspaces_agree_with_lapack():
    """Clustered spectrum (graded 1 .. 1e-10 with runs of 8 values 1e-10
    apart, as in the 16384 x 8192 workload): single vectors are not defined
    inside a cluster, so the oracle's V is compared with LAPACK's cluster by
    cluster through principal angles.  Clusters with sigma >= 1e-3 sigma_max
    agree to sin(theta) <= 1e-10; below that the comparison is limited by
    LAPACK's own absolute-gap accuracy."""
    n, m = 160, 300
    s = W.graded_clustered_sigma(n, clusters=4, size=8, gap=1e-10)
    a = W.spectrum_matrix(m, n, s, 77)
    _, so, v, _ = O.plain_svd(a, eps=1e-14, threads=os.cpu_count() or 1)
    _, sl, vt = np.linalg.svd(a, full_matrices=False)
    r = O.cluster_subspace_sines(v, so, vt.T, sl, floor=1e-3)
    assert r["largest_cluster"] == 8 and r["clusters"] >= 30
    assert r["max_sine"] <= 1e-10, r
    # a planted mistake is seen: swapping two columns across a cluster boundary
    bad = v.copy()
    order = np.argsort(-so)
    bad[:, [order[0], order[1]]] = bad[:, [order[1], order[0]]]
    assert O.cluster_subspace_sines(bad, so, vt.T, sl, floor=1e-3)["max_sine"] > 0.5


@pytest.mark.parametrize("kind", ["tall", "clustered"])
def test_workload_generators_have_their_stated_spectrum(kind):
    """The bench's accuracy guard compares against the generators' own sigma
    (A = U diag(sigma) V^T with Haar factors, formed in FP64): LAPACK on the
    formed matrix agrees with it normwise to 1e-14 (smaller instances of the
    tall and the graded + clustered workloads)."""
    if kind == "tall":
        a, s = W.tall_case(seed=2, m=512, n=128, kappa=1e6)
    else:
        s = W.graded_clustered_sigma(128, clusters=2, size=16, gap=1e-10)
        a = W.spectrum_matrix(300, 128, s, 5)
    got = np.linalg.svd(a, compute_uv=False)
    assert O.sigma_errors(got, s)["normwise"] <= 1e-14


def test_batch_workload_matches_its_description():
    """m ~ U{16..256}, n ~ U{8..m}, kappa log-uniform in [1e1, 1e6], sigma in
    [1/kappa, 1], stored as FP32 - as the bench line describes it."""
    ms, ns, kappas, _ = W.batch_shapes(20000, seed=3)
    assert ms.min() == 16 and ms.max() == 256 and np.all(ns >= 8) and np.all(ns <= ms)
    assert kappas.min() >= 10.0 and kappas.max() <= 1e6
    lk = np.log10(kappas)
    assert abs(lk.mean() - 3.5) < 0.05  # log-uniform on [1, 6]
    mats = W.batch_workload(20, seed=3)
    ms20, ns20, _, _ = W.batch_shapes(20, seed=3)  # shapes depend on the count (all m drawn first)
    assert all(a.dtype == np.float32 and a.shape == (m, n) for a, m, n in zip(mats, ms20, ns20))
    for a in mats[:5]:
        s = np.linalg.svd(a.astype(np.float64), compute_uv=False)
        assert s[0] <= 1.0 + 1e-6 and s[-1] > 0.0


def test_tall_oracle_fixture_matches_its_input():
    """tests/golden/tall_4096x1024_oracle.npz (made by make_tall_sigma.py with
    the oracle, 30 sweeps on the seeded 4096 x 1024 input) belongs to the input
    that workloads.tall_case() generates here, and its sigma is the analytic one
    to the reference arithmetic's accuracy (normwise 2e-13, per value 1e-11)."""
    import hashlib

    d = np.load(os.path.join(GOLDEN, "tall_4096x1024_oracle.npz"))
    a, sig = W.tall_case()
    assert hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest() == str(d["a_sha256"])
    assert np.array_equal(d["sigma_analytic"], sig)
    assert int(d["sweeps"]) == 30
    s = np.sort(d["sigma"])[::-1]
    assert np.max(np.abs(s - sig)) / sig[0] <= 2e-13
    assert np.max(np.abs(s - sig) / sig) <= 1e-11
