"""FP64 host oracle (ctypes front end of jacobi_oracle.c) and result metrics.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by the CPU-baseline leg of ``bench.py`` - as the checker, never as the
thing measured or shipped.  The product path does not import this module.

The C file restates kleedaisuki/jacobi-svd-cuda src/kernels.cu (schedule
:637-678, pair statistics :412-472, rotation :485-575, convergence :889-981,
U/Sigma :586-629).  The metrics follow the validation contract of the
reference's report (tex/sections/03-gpu-parallel-reduction.tex:28-58):
rho_A = ||A - U S V^T||_F / max(1, ||A||_F), rho_U = ||U^T U - I||_F,
rho_V = ||V^T V - I||_F, vectors compared up to sign.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

# FMA placement variant codes (see jacobi_oracle.c): p form | q form << 2.
VARIANTS = {
    "p_cx_q_sx": 1 | (1 << 2),
    "p_cx_q_cy": 1 | (2 << 2),
    "p_sy_q_sx": 2 | (1 << 2),
    "p_sy_q_cy": 2 | (2 << 2),
    "p_plain_q_plain": 0,
}


def build() -> str:
    """Compile libjsvd_oracle.so in place (gcc) and return its path."""
    path = os.path.join(_HERE, "libjsvd_oracle.so")
    src = os.path.join(_HERE, "jacobi_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-C", _HERE, "oracle"], stdout=subprocess.DEVNULL)
    return path


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(build())
        L = ctypes.c_long
        P = ctypes.c_void_p
        _LIB.jo_plain_svd.argtypes = [P, L, L, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, P, P, P, P]
        _LIB.jo_plain_svd.restype = ctypes.c_int
        _LIB.jo_schedule.argtypes = [ctypes.c_int, P, P]
        _LIB.jo_schedule_rounds.argtypes = [ctypes.c_int]
        _LIB.jo_batch_svd.argtypes = [ctypes.c_int, P, P, P, P, P, P, P, P, P, P, P, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _LIB.jo_plain_partial_sweep.argtypes = [P, P, L, L, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_int]
    return _LIB


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def schedule(n: int) -> list[list[tuple[int, int]]]:
    """Round-robin rounds of pairs, src/kernels.cu:637-678."""
    rounds = lib().jo_schedule_rounds(n)
    if rounds == 0:
        return []
    ne = n + (n % 2)
    pairs = np.zeros((rounds, ne // 2, 2), dtype=np.int32)
    counts = np.zeros(rounds, dtype=np.int32)
    lib().jo_schedule(n, _ptr(pairs), _ptr(counts))
    return [[(int(p), int(q)) for p, q in pairs[r, : counts[r]]] for r in range(rounds)]


def plain_svd(a: np.ndarray, eps: float = 1e-9, max_sweeps: int = 128, lanes: int = 256,
              variant: int = VARIANTS["p_cx_q_sx"], threads: int = 1):
    """Oracle solve of one row-major FP64 matrix -> (U, sigma, V, sweeps)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    m, n = a.shape
    u = np.empty((m, n))
    s = np.empty(n)
    v = np.empty((n, n))
    sw = np.zeros(1, dtype=np.int32)
    rc = lib().jo_plain_svd(_ptr(a), m, n, eps, max_sweeps, lanes, variant, threads, _ptr(u), _ptr(s), _ptr(v),
                            _ptr(sw))
    if rc != 0:
        raise ValueError(f"oracle rejected the request (code {rc})")
    return u, s, v, int(sw[0])


def batch_svd(mats: list[np.ndarray], eps: float = 1e-9, max_sweeps: int = 128, lanes: int = 256,
              variant: int = VARIANTS["p_cx_q_sx"], threads: int = 1, want_u: bool = False):
    """Oracle solve of many matrices, threads across matrices -> (sigmas, Vs, sweeps[, Us])."""
    count = len(mats)
    ms = np.array([a.shape[0] for a in mats], dtype=np.int64)
    ns = np.array([a.shape[1] for a in mats], dtype=np.int64)
    a_off = np.concatenate([[0], np.cumsum(ms * ns)[:-1]]).astype(np.int64)
    s_off = np.concatenate([[0], np.cumsum(ns)[:-1]]).astype(np.int64)
    v_off = np.concatenate([[0], np.cumsum(ns * ns)[:-1]]).astype(np.int64)
    packed = np.concatenate([np.ascontiguousarray(a, dtype=np.float64).ravel() for a in mats])
    sig = np.empty(int(ns.sum()))
    vv = np.empty(int((ns * ns).sum()))
    uu = np.empty(int((ms * ns).sum())) if want_u else None
    sweeps = np.zeros(count, dtype=np.int32)
    lib().jo_batch_svd(count, _ptr(ms), _ptr(ns), _ptr(a_off), _ptr(packed),
                       _ptr(a_off) if want_u else None, _ptr(uu) if want_u else None,
                       _ptr(s_off), _ptr(sig), _ptr(v_off), _ptr(vv), _ptr(sweeps),
                       eps, max_sweeps, lanes, variant, threads)
    sigmas = [sig[s_off[k]: s_off[k] + ns[k]] for k in range(count)]
    vs = [vv[v_off[k]: v_off[k] + ns[k] * ns[k]].reshape(ns[k], ns[k]) for k in range(count)]
    if want_u:
        us = [uu[a_off[k]: a_off[k] + ms[k] * ns[k]].reshape(ms[k], ns[k]) for k in range(count)]
        return sigmas, vs, sweeps, us
    return sigmas, vs, sweeps


def partial_sweep(a: np.ndarray, eps: float, lanes: int = 256, variant: int = VARIANTS["p_cx_q_sx"],
                  rounds: int | None = None, threads: int = 1) -> int:
    """Runs the first `rounds` rounds of one sweep in place on a copy (timing helper)."""
    m, n = a.shape
    aw = np.asfortranarray(a, dtype=np.float64).copy(order="F")
    vw = np.eye(n, order="F")
    r = lib().jo_schedule_rounds(n) if rounds is None else rounds
    return lib().jo_plain_partial_sweep(_ptr(aw), _ptr(vw), m, n, eps, lanes, variant, r, threads)


# ---- metrics -----------------------------------------------------------------

def residuals(a: np.ndarray, u: np.ndarray | None, s: np.ndarray, v: np.ndarray) -> dict:
    """rho_A = ||A - U S V^T||_F / max(1, ||A||_F), rho_U = ||U^T U - I||_F,
    rho_V = ||V^T V - I||_F, the reference's validation metrics
    (tex/sections/03-gpu-parallel-reduction.tex:30-40).  rho_U runs over the
    columns with sigma > 0: the reference writes zero U columns where
    sigma <= eps (src/kernels.cu:599-627), which carry no orthogonality."""
    out = {}
    n = s.shape[0]
    if u is not None:
        rec = (u * s[None, :]) @ v.T
        out["rho_A"] = float(np.linalg.norm(a - rec) / max(1.0, np.linalg.norm(a)))
        nz = s > 0
        uu = u[:, nz]
        out["rho_U"] = float(np.linalg.norm(uu.T @ uu - np.eye(uu.shape[1])))
    out["rho_V"] = float(np.linalg.norm(v.T @ v - np.eye(n)))
    return out


def sigma_errors(s_test: np.ndarray, s_ref: np.ndarray) -> dict:
    """Max per-value relative error and normwise (|d sigma_i| / sigma_max) error after sorting."""
    a = np.sort(np.asarray(s_test))[::-1]
    b = np.sort(np.asarray(s_ref))[::-1]
    d = np.abs(a - b)
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.where(b > 0, d / b, np.where(d == 0, 0.0, np.inf))
    smax = float(b[0]) if b.size and b[0] > 0 else 1.0
    return {"max_rel": float(rel.max()) if rel.size else 0.0, "normwise": float(d.max() / smax) if d.size else 0.0}


def cluster_subspace_sines(v_test, s_test, v_ref, s_ref, rel_gap: float = 1e-6, floor: float = 0.0) -> dict:
    """Singular-subspace agreement where singular values cluster (single
    vectors are not defined inside a cluster): both results are sorted by
    sigma, consecutive reference values closer than rel_gap (relative) form
    one cluster, and for every cluster with sigma >= floor * sigma_max the
    largest principal-angle sine between span(V_test[:, cluster]) and
    span(V_ref[:, cluster]) is ||T - R (R^T T)||_2 (accurate for tiny angles,
    R orthonormal).  Returns the largest sine, the clusters compared and the
    largest cluster size."""
    it = np.argsort(-np.asarray(s_test), kind="stable")
    ir = np.argsort(-np.asarray(s_ref), kind="stable")
    sr = np.asarray(s_ref)[ir]
    vt, vr = np.asarray(v_test)[:, it], np.asarray(v_ref)[:, ir]
    n = sr.shape[0]
    worst, used, largest, start = 0.0, 0, 0, 0
    for i in range(1, n + 1):
        if i < n and abs(sr[i - 1] - sr[i]) <= rel_gap * abs(sr[i - 1]):
            continue
        if sr[start] >= floor * sr[0]:
            t, r = vt[:, start:i], vr[:, start:i]
            worst = max(worst, float(np.linalg.norm(t - r @ (r.T @ t), 2)))
            used += 1
            largest = max(largest, i - start)
        start = i
    return {"max_sine": worst, "clusters": used, "largest_cluster": largest}


def columns_match_up_to_sign(x: np.ndarray, y: np.ndarray, tol: float) -> float:
    """Max over columns of min(||x_j - y_j||, ||x_j + y_j||); returns that maximum."""
    dp = np.linalg.norm(x - y, axis=0)
    dm = np.linalg.norm(x + y, axis=0)
    return float(np.minimum(dp, dm).max()) if x.size else 0.0
