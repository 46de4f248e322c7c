"""Generates tests/golden/tall_4096x1024_oracle.npz: the FP64 oracle's solve
of the seeded 4096 x 1024 input (A = U diag(sigma) V^T, Haar U and V from
seed 2, sigma geometric from 1 to 1e-6), epsilon 1e-14.

The oracle restates the reference's arithmetic (src/kernels.cu) and is pinned
bit for bit against the reference's own outputs (tests/golden/summary.json),
so this is the reference's result on this input.  Stored: sigma in the
oracle's column order, the sweep count, the residuals rho_A, rho_U, rho_V,
SHA-256 digests of the input and of the oracle's V, and the analytic sigma.
bench.py reports the error of every path's sigma against it (max relative and
normwise), beside the error against the analytic sigma; it uses the fixture
only when the SHA-256 of the input it generated matches.

Usage: python tests/golden/make_tall_sigma.py [THREADS]
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "jacobi-svd-cuda_b200"))

import oracle as O  # noqa: E402
import workloads as W  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "tall_4096x1024_oracle.npz")


def main() -> None:
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else os.cpu_count() or 1
    a, sig = W.tall_case()
    a = np.ascontiguousarray(a)
    t0 = time.time()
    u, s, v, sweeps = O.plain_svd(a, eps=1e-14, threads=threads)
    elapsed = time.time() - t0
    r = O.residuals(a, u, s, v)
    np.savez_compressed(
        OUT,
        sigma=s,
        sweeps=np.int64(sweeps),
        rho=np.array([r["rho_A"], r["rho_U"], r["rho_V"]]),
        a_sha256=np.array(hashlib.sha256(a.tobytes()).hexdigest()),
        v_sha256=np.array(hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()),
        sigma_analytic=sig,
        epsilon=np.float64(1e-14),
    )
    print(f"wrote {OUT}: {sweeps} sweeps in {elapsed:.0f} s on {threads} threads; residuals {r}")


if __name__ == "__main__":
    main()
