"""Parity of the plain FP64 sweep (C-ABI, sm_100a) with the oracle and with
the reference's own outputs.

The plain path keeps the reference's arithmetic, so the expected result is
bit-for-bit equality with the oracle run under the library's FMA variant
(same sigma, U, V bytes and sweep count).  The reference's golden fixtures
are compared bit for bit when the pinned variant equals the library's, else
within the drop-in tolerance: sigma max relative error <= 1e-13 * n and U, V
columns equal up to sign within 1e-9.
"""
import glob
import json
import os

import numpy as np
import pytest

import jsvd
import oracle as O
import workloads as W
from conftest import GOLDEN, golden_input

pytestmark = pytest.mark.gpu

SHAPES = [
    (1, 1), (2, 1), (2, 2), (3, 2), (5, 5), (8, 3), (16, 16), (17, 9), (31, 30), (64, 48), (100, 100),
    (128, 127), (255, 17), (257, 64), (300, 1), (513, 40), (600, 257), (1100, 64), (2100, 24), (4500, 20),
]


def _oracle(a, eps, T=256):
    return O.plain_svd(a, eps=eps, lanes=T, variant=jsvd.arith_variant(), threads=os.cpu_count() or 1)


def _assert_bitwise(got, exp):
    gu, gs, gv, gsw = got
    eu, es, ev, esw = exp
    assert gsw == esw, f"sweeps {gsw} != {esw}"
    assert np.array_equal(gs, es), f"sigma differs: max {np.max(np.abs(gs - es))}"
    assert np.array_equal(gu, eu), f"U differs: max {np.max(np.abs(gu - eu))}"
    assert np.array_equal(gv, ev), f"V differs: max {np.max(np.abs(gv - ev))}"


@pytest.mark.parametrize("m,n", SHAPES)
def test_plain_bitwise_vs_oracle(cuda_device, m, n):
    a = W.gaussian_splitmix(m, n, seed=1000 + 7 * m + n)
    eps = 1e-13
    got = jsvd.plain_svd(a, jsvd.default_config(epsilon=eps))
    _assert_bitwise(got, _oracle(a, eps))


@pytest.mark.parametrize("T", [32, 64, 128, 512, 1024])
def test_plain_reduction_width(cuda_device, T):
    a = W.gaussian_splitmix(700, 37, seed=77)
    got = jsvd.plain_svd(a, jsvd.default_config(epsilon=1e-12, threads_per_block=T))
    _assert_bitwise(got, _oracle(a, 1e-12, T))


def test_plain_special_matrices(cuda_device):
    z = W.gaussian_splitmix(40, 12, 24)
    z[:, 3] = 0.0
    d = W.gaussian_splitmix(40, 12, 25)
    d[:, 7] = d[:, 2]
    for a in (np.eye(16), z, d, W.gaussian_splitmix(40, 12, 26) * 1e-160, np.ones((9, 4))):
        got = jsvd.plain_svd(a, jsvd.default_config(epsilon=1e-12))
        _assert_bitwise(got, _oracle(a, 1e-12))


def test_plain_max_sweeps_status(cuda_device):
    a = W.gaussian_splitmix(64, 64, 3)
    u, s, v, sw = jsvd.plain_svd(a, jsvd.default_config(epsilon=1e-15, max_sweeps=2))
    assert sw == 2  # non-convergence is reported through the sweep count, not an error
    _assert_bitwise((u, s, v, sw), O.plain_svd(a, eps=1e-15, max_sweeps=2, variant=jsvd.arith_variant(),
                                                threads=4))


def test_plain_device_entry_and_cache_reuse(cuda_device):
    import torch

    a = W.gaussian_splitmix(96, 80, 31)
    exp = _oracle(a, 1e-12)
    for _ in range(2):  # second call reuses the cached plan and graph
        da = torch.from_numpy(a).to(cuda_device)
        du = torch.empty((96, 80), dtype=torch.float64, device=cuda_device)
        ds = torch.empty(80, dtype=torch.float64, device=cuda_device)
        dv = torch.empty((80, 80), dtype=torch.float64, device=cuda_device)
        stream = torch.cuda.current_stream().cuda_stream
        sw = jsvd.plain_svd_device(da.data_ptr(), 96, 80, du.data_ptr(), ds.data_ptr(), dv.data_ptr(),
                                   jsvd.default_config(epsilon=1e-12), stream)
        _assert_bitwise((du.cpu().numpy(), ds.cpu().numpy(), dv.cpu().numpy(), sw), exp)


def test_plain_cfg1_512(cuda_device):
    """512 x 512 N(0,1) (SplitMix64 seed 1), eps 1e-14: bitwise vs oracle, plus
    the reference's validation metrics."""
    a = W.gaussian_splitmix(512, 512, 1)
    got = jsvd.plain_svd(a, jsvd.default_config(epsilon=1e-14))
    _assert_bitwise(got, _oracle(a, 1e-14))
    r = O.residuals(a, got[0], got[1], got[2])
    assert r["rho_A"] < 1e-12 and r["rho_U"] < 1e-11 and r["rho_V"] < 1e-11
    ref = np.linalg.svd(a, compute_uv=False)
    assert O.sigma_errors(got[1], ref)["max_rel"] <= 1e-13 * 512


def _golden():
    p = os.path.join(GOLDEN, "summary.json")
    if not os.path.exists(p):
        return None, []
    with open(p) as f:
        summ = json.load(f)
    # only the fixtures recorded from the reference's own runs; other .npz
    # files in the folder (the oracle-made tall-case sigma) are not
    return summ, sorted(q for q in glob.glob(os.path.join(GOLDEN, "*.npz")) if os.path.basename(q)[:-4] in summ["cases"])


_SUMMARY, _CASES = _golden()


@pytest.mark.parametrize("path", _CASES, ids=lambda p: os.path.basename(p)[:-4])
def test_plain_vs_reference_golden(cuda_device, path):
    name = os.path.basename(path)[:-4]
    g = np.load(path)
    rec = _SUMMARY["cases"][name]
    a = golden_input(name, g)
    cfg = jsvd.default_config(epsilon=float(g["eps"]), threads_per_block=int(g["T"]),
                              layout_transpose_mode=int(g["layout"]))
    u, s, v, sw = jsvd.plain_svd(a, cfg)
    n = a.shape[1]
    bitwise = O.VARIANTS[_SUMMARY["pinned_variant"]] == jsvd.arith_variant()
    if bitwise:
        assert sw == int(g["sweeps"])
        assert np.array_equal(s, g["sigma"])
        if "u" in g:
            assert np.array_equal(u, g["u"]) and np.array_equal(v, g["v"])
        else:
            import hashlib
            assert hashlib.sha256(u.tobytes()).hexdigest() == rec["u_sha256"]
            assert hashlib.sha256(v.tobytes()).hexdigest() == rec["v_sha256"]
    else:
        assert O.sigma_errors(s, g["sigma"])["max_rel"] <= 1e-13 * n
        if "u" in g:
            assert O.columns_match_up_to_sign(v, g["v"], 1e-9) <= 1e-9


@pytest.mark.parametrize("m,n", [(2, 2), (17, 9), (257, 64), (600, 257), (2100, 24)])
def test_plain_persistent_sweep_bitwise(cuda_device, m, n):
    """The persistent cooperative sweep (one launch per sweep, neighbour
    round counters) gives the same bytes as the per-round graph path."""
    a = W.gaussian_splitmix(m, n, seed=4242 + m + 3 * n)
    eps = 1e-13
    jsvd.set_sweep_mode(1)
    try:
        got = jsvd.plain_svd(a, jsvd.default_config(epsilon=eps))
    finally:
        jsvd.set_sweep_mode(0)
    _assert_bitwise(got, _oracle(a, eps))


@pytest.mark.parametrize("m,n", [(17, 9), (300, 257), (600, 600), (1100, 64)])
def test_plain_vpass_in_global_memory_bitwise(cuda_device, m, n):
    """The V pass that rotates V in place in global memory (used by itself
    above 25600 columns, where a row of V does not fit shared memory; forced
    here) gives the same bytes, on the first call (direct launches) and the
    second (captured sweep graph)."""
    a = W.gaussian_splitmix(m, n, seed=5151 + m + 7 * n)
    cfg = jsvd.default_config(epsilon=1e-13)
    jsvd.set_vpass_in_global(True)
    try:
        first = jsvd.plain_svd(a, cfg)
        second = jsvd.plain_svd(a, cfg)
    finally:
        jsvd.set_vpass_in_global(False)
    exp = _oracle(a, 1e-13)
    _assert_bitwise(first, exp)
    _assert_bitwise(second, exp)


def test_plain_rows_beyond_one_transpose_grid(cuda_device):
    """More than 65535 * 32 = 2,097,120 rows: the input transpose takes one
    launch per 2,097,120-row chunk (the grid's y limit); bit-identical to the
    oracle, and the QR-preconditioned path agrees with LAPACK."""
    a = W.gaussian_splitmix(2_100_000, 3, seed=818)
    cfg = jsvd.default_config(epsilon=1e-13)
    got = jsvd.plain_svd(a, cfg)
    _assert_bitwise(got, _oracle(a, 1e-13))
    ref = np.linalg.svd(a, compute_uv=False)
    pc = jsvd.precond_svd(a, cfg)
    assert O.sigma_errors(pc[1], ref)["normwise"] <= 1e-13
    assert O.residuals(a, pc[0], pc[1], pc[2])["rho_A"] <= 1e-12


def test_precond_with_vpass_in_global_memory_identical(cuda_device):
    """The preconditioned path's Jacobi stage through the global-memory V pass
    gives the same bytes as through the staged one."""
    a = W.gaussian_splitmix(700, 300, seed=6262)
    cfg = jsvd.default_config(epsilon=1e-13)
    ref = jsvd.precond_svd(a, cfg)
    jsvd.set_vpass_in_global(True)
    try:
        got = jsvd.precond_svd(a, cfg)
    finally:
        jsvd.set_vpass_in_global(False)
    assert got[3] == ref[3]
    for x, y in zip(got[:3], ref[:3]):
        assert np.array_equal(x, y)


def test_plain_rounds_with_pdl_bitwise(cuda_device):
    """Sweep mode 2 (programmatic dependent launch between rounds) gives the
    same bytes."""
    a = W.gaussian_splitmix(300, 120, seed=99)
    jsvd.set_sweep_mode(2)
    try:
        got = jsvd.plain_svd(a, jsvd.default_config(epsilon=1e-13))
    finally:
        jsvd.set_sweep_mode(0)
    _assert_bitwise(got, _oracle(a, 1e-13))


@pytest.mark.parametrize("T", [32, 256, 1024])
def test_plain_angle_every_warp_bitwise(cuda_device, T):
    """Sweep mode 3 (every warp reduces and derives the angle itself, the
    single-barrier form) gives the same bytes as the oracle."""
    a = W.gaussian_splitmix(700, 90, seed=123)
    jsvd.set_sweep_mode(3)
    try:
        got = jsvd.plain_svd(a, jsvd.default_config(epsilon=1e-13, threads_per_block=T))
    finally:
        jsvd.set_sweep_mode(0)
    _assert_bitwise(got, _oracle(a, 1e-13, T))


def test_svd_entry_matches_the_solver_entries(cuda_device):
    """jsvd.svd(a, solver) through each host entry: plain is the oracle bit
    for bit; every solver returns its device entry's bytes and is accurate to
    working precision."""
    import torch

    a = W.gaussian_splitmix(200, 96, seed=31)  # 96 columns: three blocks for the blocked engine
    m, n = a.shape
    cfg = jsvd.default_config(epsilon=1e-13)
    r = jsvd.svd(a, "plain", cfg)
    _assert_bitwise(r, _oracle(a, 1e-13))
    ref = np.linalg.svd(a, compute_uv=False)
    device_entries = {"plain": jsvd.plain_svd_device, "precond": jsvd.precond_svd_device,
                      "blockpair": jsvd.blockpair_svd_device, "blocked": jsvd.blocked_svd_device}
    for solver, entry in device_entries.items():
        r = jsvd.svd(a, solver, cfg)
        assert O.sigma_errors(r.sigma, ref)["normwise"] <= 1e-13, solver
        da = torch.from_numpy(a).to(cuda_device)
        du = torch.empty((m, n), dtype=torch.float64, device=cuda_device)
        ds = torch.empty(n, dtype=torch.float64, device=cuda_device)
        dv = torch.empty((n, n), dtype=torch.float64, device=cuda_device)
        torch.cuda.synchronize(cuda_device)
        sw = entry(da.data_ptr(), m, n, du.data_ptr(), ds.data_ptr(), dv.data_ptr(), cfg)
        _assert_bitwise(r, (du.cpu().numpy(), ds.cpu().numpy(), dv.cpu().numpy(), sw))
