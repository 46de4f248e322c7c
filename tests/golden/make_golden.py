"""Generates the golden fixtures of the plain path from the reference itself.

Runs the UNMODIFIED kleedaisuki/jacobi-svd-cuda solver
(jacobi::svd::one_sided_jacobi_svd, built from its own sources into
oracle/_ref/libjsvd_ref.so by oracle/Makefile) on seeded inputs on a GPU, and
records its outputs.  It also runs the oracle under every FMA-placement variant
and records which variant reproduces the reference bit for bit.

Usage (needs a GPU and a built oracle/_ref):
    python tests/golden/make_golden.py OUTDIR [--pipeline-only]
Writes OUTDIR/<case>.npz and OUTDIR/summary.json.  Small cases keep the full
U, Sigma, V; large cases keep Sigma, the sweep count and SHA-256 digests of
the U and V bytes.  It also writes OUTDIR/pipeline_in.mat (a seeded stream of
testcases) and OUTDIR/pipeline_ref_out.mat, the output of the reference's own
CLI (oracle/_ref/jacobi-svd-cuda -e 1e-12) on it.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "jacobi-svd-cuda_b200"))

import matfile  # noqa: E402
import oracle as O  # noqa: E402
import workloads as W  # noqa: E402

FULL_LIMIT = 40_000  # store full U/V below this many elements


def cases():
    """(name, matrix, eps, threads_per_block, layout_mode)."""
    g = W.gaussian_splitmix
    out = [
        ("g3x2", g(3, 2, 11), 1e-9, 256, 0),
        ("g2x2", g(2, 2, 12), 1e-12, 256, 0),
        ("g8x8", g(8, 8, 13), 1e-12, 256, 0),
        ("g17x9", g(17, 9, 14), 1e-12, 256, 0),
        ("g33x16", g(33, 16, 15), 1e-12, 256, 0),
        ("g64x48", g(64, 48, 16), 1e-12, 256, 0),
        ("g64x48_on", g(64, 48, 16), 1e-12, 256, 1),
        ("g64x48_off", g(64, 48, 16), 1e-12, 256, 2),
        ("g100x100", g(100, 100, 17), 1e-13, 256, 0),
        ("g128x127", g(128, 127, 18), 1e-12, 256, 0),
        ("g257x64", g(257, 64, 19), 1e-12, 256, 0),
        ("g300x1", g(300, 1, 20), 1e-9, 256, 0),
        ("g600x40", g(600, 40, 21), 1e-12, 256, 0),
        ("g96x40_t32", g(96, 40, 22), 1e-12, 32, 0),
        ("g96x40_t64", g(96, 40, 22), 1e-12, 64, 0),
        ("g96x40_t128", g(96, 40, 22), 1e-12, 128, 0),
        ("g96x40_t512", g(96, 40, 22), 1e-12, 512, 0),
        ("g96x40_t1024", g(96, 40, 22), 1e-12, 1024, 0),
        ("g2100x24_t256", g(2100, 24, 23), 1e-12, 256, 0),
        ("eye16", np.eye(16), 1e-9, 256, 0),
    ]
    z = g(40, 12, 24)
    z[:, 3] = 0.0
    out.append(("zero_col40x12", z, 1e-12, 256, 0))
    d = g(40, 12, 25)
    d[:, 7] = d[:, 2]
    out.append(("dup_col40x12", d, 1e-12, 256, 0))
    out.append(("tiny40x12", g(40, 12, 26) * 1e-160, 1e-12, 256, 0))
    s = W.geometric_sigma(48, 1e-8)
    out.append(("kappa1e8_96x48", W.spectrum_matrix(96, 48, s, 27), 1e-14, 256, 0))
    out.append(("cfg1_512x512", g(512, 512, 1), 1e-14, 256, 0))
    out.append(("g1024x256", g(1024, 256, 28), 1e-12, 256, 0))
    return out


def ref_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libjsvd_ref.so")
    L = ctypes.CDLL(path)
    P, S, I, D = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_double
    L.ref_plain_svd.argtypes = [P, S, S, D, I, I, I, P, P, P, P]
    L.ref_plain_svd.restype = I
    L.ref_last_error.restype = ctypes.c_char_p
    return L


def run_ref(L, a, eps, T, layout):
    m, n = a.shape
    a = np.ascontiguousarray(a)
    u, s, v = np.empty((m, n)), np.empty(n), np.empty((n, n))
    sw = ctypes.c_int(0)
    rc = L.ref_plain_svd(a.ctypes.data, m, n, eps, 128, T, layout, u.ctypes.data, s.ctypes.data, v.ctypes.data,
                         ctypes.byref(sw))
    if rc != 0:
        raise RuntimeError(L.ref_last_error().decode())
    return u, s, v, sw.value


def digest(x: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(x, dtype=np.float64).tobytes()).hexdigest()


def pipeline_golden(outdir: str) -> None:
    """Seeded testcase stream through the reference CLI."""
    rng = np.random.default_rng(2024)
    mats = [W.gaussian_splitmix(5, 3, 31), np.eye(4), W.gaussian_splitmix(7, 1, 32)]
    for k in range(9):
        m = int(rng.integers(2, 90))
        n = int(rng.integers(1, m + 1))
        mats.append(rng.standard_normal((m, n)))
    inp = os.path.join(outdir, "pipeline_in.mat")
    out = os.path.join(outdir, "pipeline_ref_out.mat")
    matfile.write(inp, mats)
    cli = os.path.join(ROOT, "oracle", "_ref", "jacobi-svd-cuda")
    subprocess.check_call([cli, "-i", inp, "-o", out, "-e", "1e-12", "--force", "-q"])
    print("pipeline golden:", len(mats), "testcases,", os.path.getsize(out), "bytes")


def main(outdir: str) -> int:
    os.makedirs(outdir, exist_ok=True)
    pipeline_golden(outdir)
    if "--pipeline-only" in sys.argv:
        return 0
    L = ref_lib()
    threads = os.cpu_count() or 1
    summary = {"variants": {}, "cases": {}}
    votes = {k: 0 for k in O.VARIANTS}
    for name, a, eps, T, layout in cases():
        u, s, v, sw = run_ref(L, a, eps, T, layout)
        rec = {"m": a.shape[0], "n": a.shape[1], "eps": eps, "threads_per_block": T, "layout": layout,
               "sweeps": sw, "u_sha256": digest(u), "v_sha256": digest(v), "sigma_sha256": digest(s),
               "match": {}}
        for vname, code in O.VARIANTS.items():
            ou, os_, ov, osw = O.plain_svd(a, eps=eps, lanes=T, variant=code, threads=threads)
            exact = bool(osw == sw and np.array_equal(ou, u) and np.array_equal(os_, s) and np.array_equal(ov, v))
            rec["match"][vname] = {
                "bitwise": exact,
                "sweeps": osw,
                "max_abs_u": float(np.max(np.abs(ou - u))),
                "max_abs_v": float(np.max(np.abs(ov - v))),
                "sigma": O.sigma_errors(os_, s),
            }
            votes[vname] += int(exact)
        payload = {"sigma": s, "sweeps": np.array(sw), "eps": np.array(eps), "T": np.array(T),
                   "layout": np.array(layout)}
        if a.size <= FULL_LIMIT:
            payload.update({"a": a, "u": u, "v": v})
        else:
            payload.update({"u_head": u[:4].copy(), "v_head": v[:4].copy()})
        np.savez_compressed(os.path.join(outdir, f"{name}.npz"), **payload)
        summary["cases"][name] = rec
        print(name, "sweeps", sw, {k: r["bitwise"] for k, r in rec["match"].items()}, flush=True)
    summary["variants"] = votes
    summary["variant_codes"] = O.VARIANTS
    with open(os.path.join(outdir, "summary.json"), "w") as f:
        json.dump(summary, f, indent=1)
    print("votes", votes)
    return 0


if __name__ == "__main__":
    if len(sys.argv) < 2 or sys.argv[1].startswith("-"):
        sys.exit("usage: python tests/golden/make_golden.py OUTDIR [--pipeline-only]")
    sys.exit(main(sys.argv[1]))
