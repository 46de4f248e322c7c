"""Serving core and pipeline on the GPU.

Every path of the serving core keeps the plain arithmetic, so each request's
result is bit-identical to jsvd_plain_svd on the same matrix and identical
whether it ran alone or in a mix of small (batched) and large (per-stream)
requests.  The CLI pipeline's *.mat output is compared byte for byte with the
reference CLI's output on the same input (tests/golden/pipeline_*).
"""
import json
import os
import subprocess

import numpy as np
import pytest

import jsvd
import matfile
import oracle as O
import workloads as W
from conftest import GOLDEN, PKG

pytestmark = pytest.mark.gpu

CLI = os.path.join(PKG, "jacobi-svd-b200")


def _mix(seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        m = int(np.exp(rng.uniform(np.log(8), np.log(700))))
        n = max(1, int(m * rng.uniform(0.25, 1.0)))
        out.append(rng.standard_normal((m, n)))
    return out


def _same(x, y):
    return all(np.array_equal(a, b) for a, b in zip(x, y) if a is not None)


def test_server_results_equal_alone_and_in_mix(cuda_device):
    cfg = jsvd.default_config(epsilon=1e-13)
    mats = _mix(1, 40)
    probe = [mats[3], mats[17], W.gaussian_splitmix(600, 500, 9)]
    alone = []
    with jsvd.Server(cfg) as s:
        for a in probe:
            alone.append(s.wait(s.submit(a, want_u=True)))
    with jsvd.Server(cfg, small_workers=2, large_workers=3, max_batch=8) as s:
        tickets = [s.submit(a, want_u=(i % 3 == 0)) for i, a in enumerate(mats[:20])]
        tp = [s.submit(a, want_u=True) for a in probe]
        tickets += [s.submit(a) for a in mats[20:]]
        mixed = [s.wait(t) for t in tp]
        rest = [s.wait(t) for t in tickets]
        st = s.stats()
    assert st.completed == len(mats) + len(probe) and st.failed == 0
    assert st.batches >= 1 and st.large_solves >= 1
    assert st.p99_ms >= st.p50_ms > 0
    for x, y in zip(alone, mixed):
        assert x[3] == y[3] and _same(x[:3], y[:3])
    # and bit-identical to the plain entry point
    for a, r in zip(probe, alone):
        ref = jsvd.plain_svd(a, cfg)
        assert r[3] == ref[3] and _same(r[:3], ref[:3])
    for (u, s_, v, sw, _), a in zip(rest[:5], mats[:5]):
        ref = jsvd.plain_svd(a, cfg)
        assert sw == ref[3] and np.array_equal(s_, ref[1]) and np.array_equal(v, ref[2])


def test_server_small_requests_step_by_sweep(cuda_device):
    """Sweep-granular batching: a request that converges in a few sweeps and
    arrives with (or after) one that needs many leaves the device after its
    own sweeps, not after the other's; both results equal the plain entry
    point's bit for bit, and the worker counts one step per sweep."""
    cfg = jsvd.default_config(epsilon=1e-14)
    big = W.gaussian_splitmix(200, 120, 21)  # small path (A fits shared memory), many sweeps
    tiny = [W.gaussian_splitmix(16, 4, 30 + i) for i in range(12)]
    with jsvd.Server(cfg, small_workers=1, large_workers=1) as s:
        tb = s.submit(big)
        tt = [s.submit(a) for a in tiny]
        got_t = [s.wait(t) for t in tt]
        got_b = s.wait(tb)
        st = s.stats()
    ref_b = jsvd.plain_svd(big, cfg)
    assert got_b[3] == ref_b[3] and np.array_equal(got_b[1], ref_b[1]) and np.array_equal(got_b[2], ref_b[2])
    for a, g in zip(tiny, got_t):
        ref = jsvd.plain_svd(a, cfg)
        assert g[3] == ref[3] and np.array_equal(g[1], ref[1]) and np.array_equal(g[2], ref[2])
        assert g[3] < got_b[3]
        assert g[4] < got_b[4]  # latency: retired before the long request
    assert st.batches >= got_b[3] and st.batched_requests == 13 and st.large_solves == 0


def test_server_budget_rejects_oversize(cuda_device):
    with jsvd.Server(budget_bytes=1 << 20) as s:
        with pytest.raises(jsvd.JsvdError) as e:
            s.submit(np.ones((512, 512)))
        assert e.value.code == jsvd.JSVD_ERR_BUDGET
        u, sg, v, sw, lat = s.wait(s.submit(np.eye(8)))
        assert np.array_equal(sg, np.ones(8))


def test_server_budget_admission_serialises(cuda_device):
    # budget fits one large request at a time: all still complete, in any order
    mats = [W.gaussian_splitmix(300, 280, k) for k in range(4)]
    with jsvd.Server(budget_bytes=12 << 20, large_workers=4) as s:
        ts = [s.submit(a) for a in mats]
        outs = [s.wait(t) for t in ts]
        assert s.stats().peak_device_bytes <= 12 << 20
    for a, o in zip(mats, outs):
        ref = jsvd.plain_svd(a, jsvd.default_config())
        assert np.array_equal(o[1], ref[1])


def _golden_pipeline():
    inp = os.path.join(GOLDEN, "pipeline_in.mat")
    out = os.path.join(GOLDEN, "pipeline_ref_out.mat")
    return (inp, out) if os.path.exists(inp) and os.path.exists(out) else (None, None)


def test_cli_pipeline_matches_reference_cli_bytes(cuda_device, tmp_path):
    inp, ref_out = _golden_pipeline()
    assert inp is not None, "pipeline golden fixture missing"
    out = tmp_path / "out.mat"
    r = subprocess.run([CLI, inp, str(out), "-e", "1e-12", "--json-report"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert out.read_bytes() == open(ref_out, "rb").read()
    js = json.loads(r.stdout[r.stdout.index("{"):])  # the text report comes first
    assert js["testcase_count"] == 12 and js["emitted_matrix_count"] == 36
    assert js["batched_testcases"] + js["large_solves"] == 12 and js["batches"] >= 1
    assert js["testcases_per_s"] > 0 and 0 <= js["latency_p50_ms"] <= js["latency_p99_ms"]


def test_cli_residual_report(cuda_device, tmp_path):
    """--residual-report leaves the output bytes unchanged and writes one
    record per testcase, in input order, whose sweeps match the oracle and whose
    rho_A, rho_U, rho_V match the oracle's metrics on the written factors."""
    inp, ref_out = _golden_pipeline()
    assert inp is not None, "pipeline golden fixture missing"
    out = tmp_path / "out.mat"
    rep = tmp_path / "res.jsonl"
    r = subprocess.run([CLI, inp, str(out), "-e", "1e-12", "-q", "--residual-report", str(rep)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert out.read_bytes() == open(ref_out, "rb").read()
    mats = matfile.read(inp)
    res = matfile.read(str(out))
    recs = [json.loads(line) for line in rep.read_text().splitlines()]
    assert len(recs) == len(mats)
    for k, (a, rec) in enumerate(zip(mats, recs)):
        u, s, v = res[3 * k], res[3 * k + 1].ravel(), res[3 * k + 2]
        assert rec["index"] == k and (rec["rows"], rec["columns"]) == a.shape
        assert rec["epsilon"] == 1e-12 and rec["max_sweeps"] == 128
        assert rec["sweeps"] == O.plain_svd(a, eps=1e-12, variant=jsvd.arith_variant())[3]
        ref = O.residuals(a, u, s, v)
        for key in ("rho_A", "rho_U", "rho_V"):
            assert abs(rec[key] - ref[key]) <= 1e-14 + 1e-10 * abs(ref[key]), (k, key, rec[key], ref[key])


def test_cli_pipeline_txt_roundtrip(cuda_device, tmp_path):
    mats = _mix(5, 6)
    src = tmp_path / "in.txt"
    with open(src, "w") as f:
        for k, a in enumerate(mats):
            if k:
                f.write("\n")
            for row in a:
                f.write(" ".join(repr(float(x)) for x in row) + "\n")
    out = tmp_path / "out.txt"
    r = subprocess.run([CLI, str(src), str(out), "-e", "1e-12", "-q"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    blocks = [b for b in out.read_text().split("\n\n") if b.strip()]
    assert len(blocks) == 3 * len(mats)
    cfg = jsvd.default_config(epsilon=1e-12)
    for k, a in enumerate(mats):
        sig = np.array([[float(x) for x in ln.split()] for ln in blocks[3 * k + 1].strip().splitlines()])
        ref = jsvd.plain_svd(a, cfg)
        assert np.array_equal(sig.ravel(), ref[1])
