"""Times the reference's own GPU solver (jacobi::svd::one_sided_jacobi_svd,
built unmodified from its sources into oracle/_ref/libjsvd_ref.so) on the
seeded single-matrix workloads, through its full host path (its own
cudaMalloc, host<->device copies and per-round synchronisations).  Not a
test; run on a GPU box:  python tests/reference_gpu_timing.py OUT.json
"""
import ctypes
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "jacobi-svd-cuda_b200"))
import workloads as W  # noqa: E402


def main(out):
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libjsvd_ref.so"))
    P, S, I, D = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_double
    L.ref_plain_svd.argtypes = [P, S, S, D, I, I, I, P, P, P, P]
    cases = {"square512": (W.gaussian_splitmix(512, 512, 1), 1e-14, 2),
             "tall": (W.tall_case(seed=2)[0], 1e-14, 1)}
    res = {}
    for name, (a, eps, reps) in cases.items():
        m, n = a.shape
        u, s, v = np.empty((m, n)), np.empty(n), np.empty((n, n))
        sw = ctypes.c_int(0)
        times = []
        for _ in range(reps):
            t0 = time.perf_counter()
            rc = L.ref_plain_svd(a.ctypes.data, m, n, eps, 128, 256, 0, u.ctypes.data, s.ctypes.data, v.ctypes.data,
                                 ctypes.byref(sw))
            times.append(time.perf_counter() - t0)
            assert rc == 0
        res[name] = {"svd_per_s": 1.0 / min(times), "seconds": min(times), "sweeps": sw.value}
        print(name, res[name], flush=True)
    with open(out, "w") as f:
        json.dump(res, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/reference_gpu_timing.py OUT.json")
    main(sys.argv[1])
