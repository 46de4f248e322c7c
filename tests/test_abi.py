"""C-ABI checks that need no GPU: the library loads, exports every symbol
declared in include/jsvd.h, and rejects invalid requests with the reference's
messages (validation runs before any CUDA call)."""
import ctypes
import os
import re

import numpy as np
import pytest

import jsvd
from conftest import ROOT


def _declared_functions():
    names = []
    for hdr in ("jsvd.h",):
        text = open(os.path.join(ROOT, "include", hdr)).read()
        names += re.findall(r"^\s*(?:const\s+)?\w[\w\s\*]*?\b(jsvd_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_loads_and_exports_declared_symbols():
    lib = jsvd.lib()
    declared = _declared_functions()
    assert len(declared) >= 8
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/jsvd.h but not exported"
    assert set(jsvd.exported_symbols()) <= set(declared)


def test_version_and_variant():
    assert b"sm_100a" in jsvd.lib().jsvd_version()
    assert jsvd.arith_variant() in (5, 9, 6, 10, 0, 1, 2, 4, 8)


def test_default_config_matches_reference():
    c = jsvd.default_config()
    assert c.epsilon == 1e-9 and c.max_sweeps == 128 and c.threads_per_block == 256
    assert c.layout_transpose_mode == jsvd.LAYOUT_AUTO
    assert c.layout_transpose_min_columns == 16 and c.layout_transpose_min_elements == 4096
    assert c.layout_transpose_auto_tune == 0
    assert c.layout_transpose_benchmark_repetitions == 2 and c.layout_transpose_benchmark_sweeps == 8


@pytest.mark.parametrize(
    "shape,overrides,message",
    [
        ((0, 3), {}, "Input matrix shape must be non-zero."),
        ((3, 0), {}, "Input matrix shape must be non-zero."),
        ((2, 3), {}, "One-sided Jacobi SVD requires rows >= columns in this implementation."),
        ((4, 3), {"epsilon": 0.0}, "epsilon must be positive."),
        ((4, 3), {"epsilon": -1.0}, "epsilon must be positive."),
        ((4, 3), {"max_sweeps": 0}, "max_sweeps must be positive."),
        ((4, 3), {"layout_transpose_min_columns": 0}, "layout_transpose_min_columns must be positive."),
        ((4, 3), {"layout_transpose_min_elements": 0}, "layout_transpose_min_elements must be positive."),
        ((4, 3), {"layout_transpose_benchmark_repetitions": 0},
         "layout_transpose_benchmark_repetitions must be positive."),
        ((4, 3), {"layout_transpose_benchmark_sweeps": 0}, "layout_transpose_benchmark_sweeps must be positive."),
    ],
)
def test_invalid_arguments(shape, overrides, message):
    cfg = jsvd.default_config(**overrides)
    m, n = shape
    buf = np.zeros(max(1, m * n))
    rc = jsvd.lib().jsvd_plain_svd(buf.ctypes.data, m, n, ctypes.byref(cfg), None, None, None, None)
    assert rc == jsvd.JSVD_ERR_INVALID_ARGUMENT
    code, msg = jsvd.last_error()
    assert code == jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert msg == message


def test_null_input_is_rejected():
    cfg = jsvd.default_config()
    rc = jsvd.lib().jsvd_plain_svd(None, 4, 3, ctypes.byref(cfg), None, None, None, None)
    assert rc == jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert jsvd.last_error()[1] == "Input buffer size mismatch."


def test_python_wrapper_raises_invalid_argument():
    with pytest.raises(jsvd.InvalidArgument, match="rows >= columns"):
        jsvd.plain_svd(np.zeros((2, 5)))


@pytest.mark.parametrize("rows,cols", [(1 << 31, 1), (2147481601, 1), (1 << 30, 1 << 30), (1 << 31, 1 << 31)])
def test_oversized_dimensions_are_rejected_before_any_access(rows, cols):
    """Shapes whose byte counts would overflow are refused with
    JSVD_ERR_OVERFLOW before the (dummy) buffer is touched."""
    cfg = jsvd.default_config()
    dummy = ctypes.c_void_p(16)
    rc = jsvd.lib().jsvd_plain_svd(dummy, rows, cols, ctypes.byref(cfg), None, None, None, None)
    assert rc == jsvd.JSVD_ERR_OVERFLOW
    assert jsvd.last_error() == (jsvd.JSVD_ERR_OVERFLOW, "Matrix dimensions exceed the supported range.")


def test_noalloc_refuses_rows_beyond_its_transpose_grid_before_cuda():
    """jsvd_plain_svd_noalloc transposes in one launch (row tiles of 32 along
    grid.y): a 2097130 x 1 request fits its scratch but not that grid, and is
    refused before any CUDA call (the dummy buffer is never touched)."""
    fn = jsvd.lib().jsvd_plain_svd_noalloc
    P, S = ctypes.c_void_p, ctypes.c_size_t
    fn.argtypes = [P, S, S, ctypes.POINTER(jsvd.Config), P, P, P, P, P]
    fn.restype = ctypes.c_int
    rc = fn(ctypes.c_void_p(16), 2097130, 1, ctypes.byref(jsvd.default_config()), None, None, None, None, None)
    assert rc == jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert jsvd.last_error()[1] == "jsvd_plain_svd_noalloc: at most 2097120 rows."


def test_integration_guide_names_every_entry_point():
    """Every C entry point declared in include/jsvd.h is described in the
    integration guide a reference-side caller reads."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    missing = [n for n in _declared_functions() if f"`{n}`" not in text]
    assert not missing, missing


@pytest.mark.parametrize(
    "overrides,message",
    [
        ({"layout_transpose_min_columns": 0}, "layout_transpose_min_columns must be positive."),
        ({"layout_transpose_min_elements": 0}, "layout_transpose_min_elements must be positive."),
        ({"layout_transpose_benchmark_repetitions": 0}, "layout_transpose_benchmark_repetitions must be positive."),
        ({"layout_transpose_benchmark_sweeps": 0}, "layout_transpose_benchmark_sweeps must be positive."),
        ({"max_sweeps": 0}, "max_sweeps must be positive."),
        # the layout settings are checked first, as in the reference
        ({"max_sweeps": 0, "layout_transpose_min_columns": 0}, "layout_transpose_min_columns must be positive."),
    ],
)
def test_auto_tune_layout_validates_before_any_solve(overrides, message):
    """jsvd_auto_tune_layout checks its settings in the reference's order
    (src/kernels.cu:1078-1086) before running any benchmark solve."""
    cfg = jsvd.default_config(**overrides)
    rep = jsvd.AutoTuneReport()
    assert jsvd.lib().jsvd_auto_tune_layout(ctypes.byref(cfg), ctypes.byref(rep)) == jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert jsvd.last_error()[1] == message


def test_auto_tune_layout_needs_a_report():
    cfg = jsvd.default_config()
    assert jsvd.lib().jsvd_auto_tune_layout(ctypes.byref(cfg), None) == jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert jsvd.last_error()[1] == "report must not be null."


def test_integration_guide_ctypes_snippet_runs():
    """The ctypes binding shown in the integration guide runs as written
    (library path adjusted to this checkout): it loads the library, builds the
    config and makes the call; without a GPU the call returns the CUDA status,
    with one it solves."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    start = text.index("```python\n", text.index("A ctypes binding")) + len("```python\n")
    code = text[start:text.index("```", start)]
    code = code.replace('"jacobi-svd-cuda_b200/libjsvd.so"', repr(os.path.join(ROOT, "jacobi-svd-cuda_b200",
                                                                                "libjsvd.so")))
    scope = {"A": np.arange(12.0).reshape(4, 3) + np.eye(4, 3)}
    exec(compile(code, "INTEGRATION.md", "exec"), scope)
    assert scope["rc"] in (jsvd.JSVD_OK, jsvd.JSVD_ERR_CUDA)
    assert scope["cfg"].epsilon == 1e-9 and scope["cfg"].max_sweeps == 128


def test_svd_entry_validates_before_cuda():
    with pytest.raises(ValueError):
        jsvd.svd(np.ones((4, 3)), solver="lapack")
    for solver in ("plain", "precond", "blockpair", "blocked"):
        with pytest.raises(jsvd.InvalidArgument) as e:
            jsvd.svd(np.ones((3, 4)), solver=solver)
        assert "rows >= columns" in str(e.value)


def test_host_wrappers_reach_the_library_call():
    """plain_svd / precond_svd / svd marshal their arguments down to the C
    call; without a GPU that call fails with the CUDA status, not earlier."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("checks the no-GPU failure")
    a = np.ones((5, 3))
    for call in (lambda: jsvd.plain_svd(a), lambda: jsvd.precond_svd(a, want_u=False),
                 lambda: jsvd.svd(a, "blocked", want_v=False), lambda: jsvd.svd(a, "blockpair")):
        with pytest.raises(jsvd.JsvdError) as e:
            call()
        assert e.value.code == jsvd.JSVD_ERR_CUDA


def test_integration_guide_covers_every_declared_function():
    """Every entry point of include/jsvd.h has its line in the integration
    guide (the reference interface it replaces, or why it has none)."""
    guide = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    missing = [name for name in _declared_functions() if name not in guide]
    assert missing == [], missing


def test_batch_cluster_classes_setter():
    """Only classes 2-4 may go to clusters; the setter reports the previous
    mask and needs no GPU."""
    old = jsvd.batch_set_cluster_classes((1 << 3) | (1 << 4))
    try:
        assert jsvd.batch_set_cluster_classes(1 << 2) == (1 << 3) | (1 << 4)
        for bad in (1, 1 << 1, 1 << 5, -1):
            with pytest.raises(jsvd.JsvdError) as e:
                jsvd.batch_set_cluster_classes(bad)
            assert e.value.code == jsvd.JSVD_ERR_INVALID_ARGUMENT
        assert jsvd.batch_set_cluster_classes(0) == 1 << 2
    finally:
        jsvd.batch_set_cluster_classes(old)
