"""The reference-compatible C++ API on the GPU: code written against the
reference's include/kernels.hpp (one_sided_jacobi_svd, DeviceMatrix,
auto_tune_layout_transpose_threshold) and the jacobi_svd solver extension of
include/kernels_ext.hpp, compiled with g++ and linked against libjsvd.so,
run through tests/cpp/api_gpu_driver.cpp.  one_sided_jacobi_svd on the
reference's own 512 x 512 golden case gives the reference's bytes (sigma, U,
V) and sweep count; the C++ result equals the C ABI's; the other solvers are
accurate to working precision."""
import os
import subprocess

import numpy as np
import pytest

import jsvd
import oracle as O
from conftest import GOLDEN, PKG, ROOT, golden_input

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "tests", "cpp", "api_gpu_driver.cpp")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = tmp_path_factory.mktemp("api_gpu") / "api_gpu_driver"
    subprocess.check_call(["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"),
                           "-I/usr/local/cuda/include", DRIVER, "-o", str(out), "-L", PKG, "-ljsvd",
                           f"-Wl,-rpath,{PKG}"])
    return str(out)


def _solve(driver, tmp_path, a, eps, threads, solver):
    m, n = a.shape
    fin, fout = tmp_path / "a.bin", tmp_path / "r.bin"
    with open(fin, "wb") as f:
        np.array([m, n], dtype=np.int64).tofile(f)
        np.ascontiguousarray(a, dtype=np.float64).tofile(f)
    subprocess.run([driver, "solve", str(fin), str(fout), repr(eps), str(threads), solver], check=True)
    raw = np.fromfile(fout, dtype=np.uint8)
    sweeps = int(np.frombuffer(raw[:4].tobytes(), dtype=np.int32)[0])
    d = np.frombuffer(raw[4:].tobytes(), dtype=np.float64)
    return d[n:n + m * n].reshape(m, n), d[:n].copy(), d[n + m * n:].reshape(n, n), sweeps


def test_one_sided_jacobi_svd_reproduces_reference_golden(cuda_device, driver, tmp_path):
    g = np.load(os.path.join(GOLDEN, "cfg1_512x512.npz"))
    a = golden_input("cfg1_512x512", g)
    u, s, v, sw = _solve(driver, tmp_path, a, float(g["eps"]), int(g["T"]), "reference")
    assert sw == int(g["sweeps"])
    assert np.array_equal(s, g["sigma"])
    if "u" in g:
        assert np.array_equal(u, g["u"]) and np.array_equal(v, g["v"])
    r = O.residuals(a, u, s, v)
    assert r["rho_A"] < 1e-12 and r["rho_U"] < 1e-11 and r["rho_V"] < 1e-11


@pytest.mark.parametrize("m,n", [(1, 1), (7, 3), (300, 257), (1100, 64)])
def test_cxx_result_equals_c_abi(cuda_device, driver, tmp_path, m, n):
    a = np.random.default_rng(m * 7 + n).standard_normal((m, n))
    u, s, v, sw = _solve(driver, tmp_path, a, 1e-13, 256, "reference")
    u2, s2, v2, sw2 = jsvd.plain_svd(a, jsvd.default_config(epsilon=1e-13))
    assert sw == sw2 and np.array_equal(s, s2) and np.array_equal(u, u2) and np.array_equal(v, v2)


@pytest.mark.parametrize("solver", ["plain", "precond", "blockpair", "blocked", "mixed"])
def test_jacobi_svd_solvers(cuda_device, driver, tmp_path, solver):
    a = np.random.default_rng(11).standard_normal((400, 300))
    u, s, v, sw = _solve(driver, tmp_path, a, 1e-14, 256, solver)
    ref = np.linalg.svd(a, compute_uv=False)
    assert O.sigma_errors(s, ref)["max_rel"] <= 1e-12
    r = O.residuals(a, u, s, v)
    assert r["rho_A"] < 1e-12 and r["rho_U"] < 1e-11 and r["rho_V"] < 1e-11


def test_device_matrix_round_trips(cuda_device, driver):
    out = subprocess.run([driver, "device-matrix"], capture_output=True, text=True, check=True).stdout.splitlines()
    assert out == ["shape 3x4 12 96", "round_trip 1", "move_construct 1 1", "move_assign 1 1", "reset 5x2 10",
                   "reset_round_trip 1", "size_check Host data size does not match device matrix shape."]


def test_auto_tune_report(cuda_device, driver):
    out = dict(line.split(" ", 1) for line in
               subprocess.run([driver, "auto-tune"], capture_output=True, text=True, check=True).stdout.splitlines())
    assert out["executed"] == "1"
    assert int(out["sample_count"]) > 0
    assert int(out["recommended_min_columns"]) >= 1 and int(out["recommended_min_elements"]) >= 1
    assert float(out["estimated_best_speedup"]) > 0.0
