"""ctypes binding of libjsvd.so (include/jsvd.h) for tests, benchmarks and tooling.

The library is the product; this module only marshals arguments.  Loading
fails loudly when libjsvd.so has not been built - there is no fallback.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libjsvd.so")

JSVD_OK = 0
JSVD_ERR_INVALID_ARGUMENT = 1
JSVD_ERR_CUDA = 2
JSVD_ERR_OVERFLOW = 3
JSVD_ERR_RUNTIME = 4
JSVD_ERR_BUDGET = 5

LAYOUT_AUTO, LAYOUT_FORCE_ENABLE, LAYOUT_FORCE_DISABLE = 0, 1, 2


class Config(ctypes.Structure):
    """jsvd_config (mirrors JacobiSvdConfig, reference include/kernels.hpp:78-124)."""

    _fields_ = [
        ("epsilon", ctypes.c_double),
        ("max_sweeps", ctypes.c_int),
        ("threads_per_block", ctypes.c_int),
        ("layout_transpose_mode", ctypes.c_int),
        ("layout_transpose_min_columns", ctypes.c_int),
        ("layout_transpose_min_elements", ctypes.c_size_t),
        ("layout_transpose_auto_tune", ctypes.c_int),
        ("layout_transpose_benchmark_repetitions", ctypes.c_int),
        ("layout_transpose_benchmark_sweeps", ctypes.c_int),
    ]


class AutoTuneReport(ctypes.Structure):
    _fields_ = [
        ("executed", ctypes.c_int),
        ("recommended_min_columns", ctypes.c_int),
        ("recommended_min_elements", ctypes.c_size_t),
        ("estimated_best_speedup", ctypes.c_double),
        ("sample_count", ctypes.c_size_t),
    ]


class PlainStats(ctypes.Structure):
    _fields_ = [
        ("solves", ctypes.c_ulonglong),
        ("sweeps", ctypes.c_ulonglong),
        ("round_launches", ctypes.c_ulonglong),
        ("vpass_launches", ctypes.c_ulonglong),
        ("other_launches", ctypes.c_ulonglong),
        ("round_ms", ctypes.c_double),
        ("vpass_ms", ctypes.c_double),
    ]


class JsvdError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


class InvalidArgument(JsvdError, ValueError):
    pass


_LIB = None


def build(quiet: bool = True) -> str:
    """Runs `make` in the package directory (nvcc, sm_100a)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.check_call(["make", "-C", HERE, "-j8"], stdout=out)
    return LIB_PATH


def exported_symbols() -> list[str]:
    """Names declared in include/jsvd.h (checked against the built library by tests)."""
    return [
        "jsvd_config_default", "jsvd_last_error", "jsvd_version", "jsvd_plain_arith_variant",
        "jsvd_plain_svd", "jsvd_plain_svd_device", "jsvd_auto_tune_layout", "jsvd_release_thread_cache",
        "jsvd_plain_stats_get", "jsvd_plain_stats_reset",
    ]


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with `make -C {HERE}` (no fallback exists)")
        L = ctypes.CDLL(LIB_PATH)
        P, S, I = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
        L.jsvd_config_default.argtypes = [ctypes.POINTER(Config)]
        L.jsvd_config_default.restype = None
        L.jsvd_last_error.argtypes = [ctypes.c_char_p, S]
        L.jsvd_last_error.restype = I
        L.jsvd_version.restype = ctypes.c_char_p
        L.jsvd_plain_arith_variant.restype = I
        L.jsvd_plain_svd.argtypes = [P, S, S, ctypes.POINTER(Config), P, P, P, P]
        L.jsvd_plain_svd.restype = I
        L.jsvd_plain_svd_device.argtypes = [P, S, S, ctypes.POINTER(Config), P, P, P, P, P]
        L.jsvd_plain_svd_device.restype = I
        L.jsvd_auto_tune_layout.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(AutoTuneReport)]
        L.jsvd_auto_tune_layout.restype = I
        L.jsvd_release_thread_cache.restype = None
        L.jsvd_plain_stats_get.argtypes = [ctypes.POINTER(PlainStats)]
        L.jsvd_plain_stats_get.restype = None
        L.jsvd_plain_stats_reset.restype = None
        _LIB = L
    return _LIB


def default_config(**overrides) -> Config:
    cfg = Config()
    lib().jsvd_config_default(ctypes.byref(cfg))
    for k, v in overrides.items():
        setattr(cfg, k, v)
    return cfg


def last_error() -> tuple[int, str]:
    buf = ctypes.create_string_buffer(4096)
    code = lib().jsvd_last_error(buf, len(buf))
    return code, buf.value.decode()


def check(rc: int) -> None:
    if rc != JSVD_OK:
        code, msg = last_error()
        if rc == JSVD_ERR_INVALID_ARGUMENT:
            raise InvalidArgument(rc, msg)
        raise JsvdError(rc, msg)


def arith_variant() -> int:
    return int(lib().jsvd_plain_arith_variant())


def plain_svd(a: np.ndarray, cfg: Config | None = None, want_u: bool = True, want_v: bool = True):
    """Host-buffer plain solve -> (U or None, sigma, V or None, sweeps)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError("expected a 2-D matrix")
    m, n = a.shape
    cfg = cfg or default_config()
    u = np.empty((m, n)) if want_u else None
    s = np.empty(n)
    v = np.empty((n, n)) if want_v else None
    sw = ctypes.c_int(0)
    rc = lib().jsvd_plain_svd(a.ctypes.data if a.size else None, m, n, ctypes.byref(cfg),
                              u.ctypes.data if u is not None else None, s.ctypes.data,
                              v.ctypes.data if v is not None else None, ctypes.byref(sw))
    check(rc)
    return u, s, v, sw.value


def plain_svd_device(d_a, m: int, n: int, d_u, d_sigma, d_v, cfg: Config | None = None, stream: int = 0) -> int:
    """Device-buffer plain solve on raw pointers (ints); returns sweeps."""
    cfg = cfg or default_config()
    sw = ctypes.c_int(0)
    rc = lib().jsvd_plain_svd_device(d_a, m, n, ctypes.byref(cfg), d_u, d_sigma, d_v, ctypes.byref(sw),
                                     stream or None)
    check(rc)
    return sw.value


def plain_stats() -> PlainStats:
    st = PlainStats()
    lib().jsvd_plain_stats_get(ctypes.byref(st))
    return st


def plain_stats_reset() -> None:
    lib().jsvd_plain_stats_reset()


def auto_tune_layout(cfg: Config | None = None) -> AutoTuneReport:
    cfg = cfg or default_config()
    rep = AutoTuneReport()
    check(lib().jsvd_auto_tune_layout(ctypes.byref(cfg), ctypes.byref(rep)))
    return rep
