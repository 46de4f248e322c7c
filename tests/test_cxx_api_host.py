"""The jacobi::svd C++ extensions (include/kernels_ext.hpp) on the host (no
GPU): every solver validates like one_sided_jacobi_svd and throws the
reference's exception types before any CUDA call, and residuals() agrees with
the oracle's restatement of the reference's validation metrics."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import PKG, ROOT

DRIVER = os.path.join(ROOT, "tests", "cpp", "api_driver.cpp")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = tmp_path_factory.mktemp("api") / "api_driver"
    subprocess.check_call(["g++", "-std=c++20", "-O1", "-I", os.path.join(ROOT, "include"),
                           "-I/usr/local/cuda/include", DRIVER, "-o", str(out), "-L", PKG, "-ljsvd",
                           f"-Wl,-rpath,{PKG}"])
    return str(out)


def test_every_solver_validates_like_the_reference(driver):
    out = subprocess.run([driver, "validate"], capture_output=True, text=True, check=True).stdout.splitlines()
    assert len(out) == 12
    for k, solver in enumerate(["plain", "precond", "blockpair", "blocked"]):
        assert out[3 * k] == f"{solver} invalid_argument " \
                             "One-sided Jacobi SVD requires rows >= columns in this implementation."
        assert out[3 * k + 1] == f"{solver} invalid_argument Input buffer size mismatch."
        assert out[3 * k + 2] == f"{solver} invalid_argument epsilon must be positive."


@pytest.mark.parametrize("m,n", [(3, 2), (30, 17), (64, 64)])
def test_residuals_match_oracle(driver, tmp_path, m, n):
    rng = np.random.default_rng(m * 100 + n)
    a = rng.standard_normal((m, n))
    uu, s, vt = np.linalg.svd(a, full_matrices=False)
    u = uu + 1e-9 * rng.standard_normal(uu.shape)
    v = vt.T + 1e-8 * rng.standard_normal((n, n))
    f = tmp_path / "case.txt"
    with open(f, "w") as fh:
        fh.write(f"{m} {n}\n")
        for arr in (a, u, s, v):
            fh.write(" ".join(repr(float(x)) for x in np.ravel(arr)) + "\n")
    got = [float(x) for x in subprocess.run([driver, "residuals", str(f)], capture_output=True, text=True,
                                            check=True).stdout.split()]
    ref = O.residuals(a, u, s, v)
    for g, key in zip(got, ("rho_A", "rho_U", "rho_V")):
        assert abs(g - ref[key]) <= 1e-14 + 1e-10 * ref[key], (key, g, ref[key])


def test_residuals_reject_mismatched_result(driver):
    out = subprocess.run([driver, "bad-result"], capture_output=True, text=True, check=True).stdout.strip()
    assert out == "Result buffers do not match rows and columns."


def test_cuda_failures_surface_as_cuda_error(driver):
    """Without a GPU the first CUDA call of every solver fails: the C++ API
    throws jacobi::svd::CudaError with the reference's message format
    ("CUDA call failed: <expr> @ <file>:<line>, code=<n>, message=<text>")."""
    import re

    import torch

    if torch.cuda.is_available():
        pytest.skip("checks the failure path of a machine without a GPU")
    out = subprocess.run([driver, "cuda-error"], capture_output=True, text=True, check=True).stdout.splitlines()
    assert len(out) == 4
    for line, solver in zip(out, ["plain", "precond", "blockpair", "blocked"]):
        assert re.match(rf"{solver} CudaError CUDA call failed: .+ @ .+:\d+, code=\d+, message=.+", line), line


def test_device_matrix_argument_checks(driver):
    """DeviceMatrix (reference include/kernels.hpp:130-244) rejects zero
    dimensions and mismatched host data with the reference's messages,
    before any device allocation or copy."""
    out = subprocess.run([driver, "device-matrix"], capture_output=True, text=True, check=True).stdout.splitlines()
    assert out == ["DeviceMatrix dimensions must be positive."] * 2 + \
        ["Host data size does not match device matrix shape."]


def test_documented_build_line_builds_a_caller(tmp_path):
    """The integration guide's build line (g++ -std=c++20 -I include ...
    -ljsvd) compiles and links a caller of the drop-in headers without the
    CUDA headers on the include path."""
    src = tmp_path / "app.cpp"
    src.write_text(
        "#include <vector>\n#include \"kernels.hpp\"\n#include \"kernels_ext.hpp\"\n"
        "#include \"pipeline.hpp\"\n#include \"pipeline_ext.hpp\"\n#include \"io.hpp\"\n"
        "int main() {\n  std::vector<double> a(12, 1.0);\n  jacobi::svd::JacobiSvdConfig cfg;\n"
        "  try { (void)jacobi::svd::one_sided_jacobi_svd(a, 4, 3, cfg); } catch (const std::exception &) {}\n"
        "  jacobi::svd::pipeline::PipelineConfig p;\n  (void)p;\n  return 0;\n}\n")
    subprocess.check_call(["g++", "-std=c++20", "-I", os.path.join(ROOT, "include"), str(src), "-L", PKG,
                           "-ljsvd", f"-Wl,-rpath,{PKG}", "-o", str(tmp_path / "app")])
