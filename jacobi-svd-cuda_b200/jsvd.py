"""ctypes binding of libjsvd.so (include/jsvd.h) for tests, benchmarks and tooling.

The library is the product; this module only marshals arguments.  Loading
fails loudly when libjsvd.so has not been built - there is no fallback.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import NamedTuple

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
        ("gram_checks", ctypes.c_ulonglong),
    ]


class BlockPairStats(ctypes.Structure):
    _fields_ = [
        ("solves", ctypes.c_ulonglong),
        ("sweeps", ctypes.c_ulonglong),
        ("round_launches", ctypes.c_ulonglong),
        ("round_ms", ctypes.c_double),
    ]


class BatchTuning(ctypes.Structure):
    _fields_ = [("threads", ctypes.c_int), ("ctas_per_sm", ctypes.c_int), ("max_ctas", ctypes.c_int)]


class ResidualReport(ctypes.Structure):
    _fields_ = [("rho_a", ctypes.c_double), ("rho_u", ctypes.c_double), ("rho_v", ctypes.c_double),
                ("sigma_max", ctypes.c_double)]


class BatchAutotuneReport(ctypes.Structure):
    _fields_ = [
        ("best", BatchTuning * 5),
        ("builtin", BatchTuning * 5),
        ("best_ms", ctypes.c_double * 5),
        ("builtin_ms", ctypes.c_double * 5),
        ("members", ctypes.c_int * 5),
        ("sampled", ctypes.c_int * 5),
        ("candidates", ctypes.c_int * 5),
    ]


class BatchStats(ctypes.Structure):
    _fields_ = [
        ("calls", ctypes.c_ulonglong),
        ("launches", ctypes.c_ulonglong),
        ("matrices", ctypes.c_ulonglong),
        ("sweeps", ctypes.c_ulonglong),
        ("kernel_ms", ctypes.c_double),
        ("class_count", ctypes.c_ulonglong * 5),
        ("class_ms", ctypes.c_double * 5),
    ]


class ServerOptions(ctypes.Structure):
    _fields_ = [
        ("device_budget_bytes", ctypes.c_size_t),
        ("small_workers", ctypes.c_int),
        ("large_workers", ctypes.c_int),
        ("max_batch", ctypes.c_int),
        ("cfg", Config),
        ("large_path", ctypes.c_int),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_ulonglong), ("completed", ctypes.c_ulonglong), ("failed", ctypes.c_ulonglong),
        ("batches", ctypes.c_ulonglong), ("batched_requests", ctypes.c_ulonglong),
        ("large_solves", ctypes.c_ulonglong),
        ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
        ("peak_device_bytes", ctypes.c_size_t), ("device_bytes_in_use", ctypes.c_size_t),
    ]


class PrecondStats(ctypes.Structure):
    _fields_ = [("solves", ctypes.c_ulonglong), ("fallbacks", ctypes.c_ulonglong), ("qr_ms", ctypes.c_double),
                ("jacobi_ms", ctypes.c_double), ("u_ms", ctypes.c_double)]


class BlockedStats(ctypes.Structure):
    _fields_ = [("solves", ctypes.c_ulonglong), ("sweeps", ctypes.c_ulonglong),
                ("block_rounds", ctypes.c_ulonglong), ("sweep_ms", ctypes.c_double)]


class MixedOptions(ctypes.Structure):
    _fields_ = [("precondition", ctypes.c_int), ("tc_max_sweeps", ctypes.c_int), ("tc_tol", ctypes.c_double),
                ("inner_sweeps", ctypes.c_int), ("refine", ctypes.c_int), ("f64_max_sweeps", ctypes.c_int),
                ("gram_splits", ctypes.c_int), ("sort", ctypes.c_int)]


class MixedStats(ctypes.Structure):
    _fields_ = [("solves", ctypes.c_ulonglong), ("tc_sweeps", ctypes.c_ulonglong), ("f64_sweeps", ctypes.c_ulonglong),
                ("block_rounds", ctypes.c_ulonglong), ("fallbacks", ctypes.c_ulonglong),
                ("qr_ms", ctypes.c_double), ("tc_ms", ctypes.c_double), ("orth_ms", ctypes.c_double),
                ("refine_ms", ctypes.c_double), ("out_ms", ctypes.c_double),
                ("last_tc_offdiag", ctypes.c_double), ("last_f64_offdiag", ctypes.c_double),
                ("last_tc_sweeps", ctypes.c_int), ("last_f64_sweeps", ctypes.c_int),
                ("tc_gram_launches", ctypes.c_ulonglong), ("tc_rot_launches", ctypes.c_ulonglong),
                ("f64_gram_launches", ctypes.c_ulonglong), ("f64_rot_launches", ctypes.c_ulonglong),
                ("evd_launches", ctypes.c_ulonglong), ("tc_discarded", ctypes.c_ulonglong),
                ("tc_gram_ms", ctypes.c_double), ("tc_evd_ms", ctypes.c_double), ("tc_rot_ms", ctypes.c_double),
                ("f64_gram_ms", ctypes.c_double), ("f64_evd_ms", ctypes.c_double), ("f64_rot_ms", ctypes.c_double),
                ("tc_sampled_rounds", ctypes.c_ulonglong), ("f64_sampled_rounds", ctypes.c_ulonglong),
                ("tc_sampled_pairs", ctypes.c_ulonglong), ("f64_sampled_pairs", ctypes.c_ulonglong),
                ("rows_pad", ctypes.c_int), ("cols_pad", ctypes.c_int), ("block_pairs", ctypes.c_int)]


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
        "jsvd_plain_stats_get", "jsvd_plain_stats_reset", "jsvd_plain_svd_noalloc",
        "jsvd_batch_svd_device", "jsvd_batch_stats_get", "jsvd_batch_stats_reset", "jsvd_probe_fp64_tflops",
        "jsvd_server_options_default", "jsvd_server_create", "jsvd_server_submit", "jsvd_server_wait",
        "jsvd_server_get_stats", "jsvd_server_destroy", "jsvd_precond_svd", "jsvd_precond_svd_device",
        "jsvd_precond_stats_get", "jsvd_precond_stats_reset", "jsvd_blocked_svd_device",
        "jsvd_blocked_svd", "jsvd_blocked_stats_get", "jsvd_blocked_stats_reset", "jsvd_plain_set_sweep_mode",
        "jsvd_plain_get_sweep_mode", "jsvd_blockpair_svd_device", "jsvd_blockpair_svd", "jsvd_blockpair_set_variant",
        "jsvd_blockpair_stats_get", "jsvd_blockpair_stats_reset", "jsvd_precond_set_inner",
        "jsvd_precond_set_gram_stop", "jsvd_batch_builtin_tuning", "jsvd_batch_autotune", "jsvd_residuals",
        "jsvd_round_robin_schedule", "jsvd_plain_set_vpass_in_global", "jsvd_server_poll",
        "jsvd_mixed_options_default", "jsvd_mixed_set_options", "jsvd_mixed_svd", "jsvd_mixed_svd_device",
        "jsvd_mixed_stats_get", "jsvd_mixed_stats_reset", "jsvd_dgemm_device", "jsvd_mixed_test_round",
        "jsvd_test_wait_limit", "jsvd_mixed_builtin_tuning",
        "jsvd_mixed_sweep_history", "jsvd_batch_set_cluster_classes",
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
        L.jsvd_batch_svd_device.argtypes = [I, P, P, P, P, I, ctypes.POINTER(Config), P, P, P, P,
                                            ctypes.POINTER(BatchTuning), P]
        L.jsvd_batch_svd_device.restype = I
        L.jsvd_plain_set_vpass_in_global.argtypes = [I]
        L.jsvd_plain_set_vpass_in_global.restype = None
        L.jsvd_round_robin_schedule.argtypes = [I, I, P, S, ctypes.POINTER(S)]
        L.jsvd_round_robin_schedule.restype = I
        L.jsvd_residuals.argtypes = [P, P, P, P, S, S, ctypes.POINTER(ResidualReport)]
        L.jsvd_residuals.restype = I
        L.jsvd_batch_builtin_tuning.argtypes = [ctypes.POINTER(BatchTuning)]
        L.jsvd_batch_builtin_tuning.restype = None
        L.jsvd_batch_set_cluster_classes.argtypes = [I, ctypes.POINTER(I)]
        L.jsvd_batch_set_cluster_classes.restype = I
        L.jsvd_batch_autotune.argtypes = [I, P, P, P, P, I, ctypes.POINTER(Config), I, I, I, I,
                                          ctypes.POINTER(BatchAutotuneReport), P]
        L.jsvd_batch_autotune.restype = I
        L.jsvd_batch_stats_get.argtypes = [ctypes.POINTER(BatchStats)]
        L.jsvd_batch_stats_get.restype = None
        L.jsvd_batch_stats_reset.restype = None
        L.jsvd_probe_fp64_tflops.argtypes = [ctypes.POINTER(ctypes.c_double)]
        L.jsvd_probe_fp64_tflops.restype = I
        L.jsvd_server_options_default.argtypes = [ctypes.POINTER(ServerOptions)]
        L.jsvd_server_options_default.restype = None
        L.jsvd_server_create.argtypes = [ctypes.POINTER(ServerOptions), ctypes.POINTER(P)]
        L.jsvd_server_create.restype = I
        L.jsvd_server_submit.argtypes = [P, P, S, S, I, ctypes.POINTER(ctypes.c_uint64)]
        L.jsvd_server_submit.restype = I
        L.jsvd_server_wait.argtypes = [P, ctypes.c_uint64, P, P, P, ctypes.POINTER(I), ctypes.POINTER(ctypes.c_double)]
        L.jsvd_server_wait.restype = I
        L.jsvd_server_poll.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(I)]
        L.jsvd_server_poll.restype = I
        L.jsvd_server_get_stats.argtypes = [P, ctypes.POINTER(ServerStats)]
        L.jsvd_server_get_stats.restype = I
        L.jsvd_server_destroy.argtypes = [P]
        L.jsvd_server_destroy.restype = None
        L.jsvd_precond_svd.argtypes = [P, S, S, ctypes.POINTER(Config), P, P, P, P]
        L.jsvd_precond_svd.restype = I
        L.jsvd_precond_svd_device.argtypes = [P, S, S, ctypes.POINTER(Config), P, P, P, P, P]
        L.jsvd_precond_svd_device.restype = I
        L.jsvd_precond_stats_get.argtypes = [ctypes.POINTER(PrecondStats)]
        L.jsvd_precond_stats_get.restype = None
        L.jsvd_precond_stats_reset.restype = None
        L.jsvd_blocked_svd_device.argtypes = [P, S, S, ctypes.POINTER(Config), P, P, P, P, P]
        L.jsvd_blocked_svd_device.restype = I
        L.jsvd_blocked_svd.argtypes = [P, S, S, ctypes.POINTER(Config), P, P, P, P]
        L.jsvd_blocked_svd.restype = I
        L.jsvd_blocked_stats_get.argtypes = [ctypes.POINTER(BlockedStats)]
        L.jsvd_blocked_stats_get.restype = None
        L.jsvd_blocked_stats_reset.restype = None
        L.jsvd_plain_set_sweep_mode.argtypes = [I]
        L.jsvd_plain_set_sweep_mode.restype = None
        L.jsvd_plain_get_sweep_mode.restype = I
        L.jsvd_blockpair_svd_device.argtypes = [P, S, S, ctypes.POINTER(Config), P, P, P, P, P]
        L.jsvd_blockpair_svd_device.restype = I
        L.jsvd_blockpair_svd.argtypes = [P, S, S, ctypes.POINTER(Config), P, P, P, P]
        L.jsvd_blockpair_svd.restype = I
        L.jsvd_blockpair_set_variant.argtypes = [I, I]
        L.jsvd_blockpair_set_variant.restype = None
        L.jsvd_blockpair_stats_get.argtypes = [ctypes.POINTER(BlockPairStats)]
        L.jsvd_blockpair_stats_get.restype = None
        L.jsvd_blockpair_stats_reset.restype = None
        L.jsvd_precond_set_inner.argtypes = [I]
        L.jsvd_precond_set_inner.restype = None
        L.jsvd_precond_set_gram_stop.argtypes = [I]
        L.jsvd_precond_set_gram_stop.restype = None
        L.jsvd_mixed_options_default.argtypes = [ctypes.POINTER(MixedOptions)]
        L.jsvd_mixed_options_default.restype = None
        L.jsvd_mixed_set_options.argtypes = [ctypes.POINTER(MixedOptions)]
        L.jsvd_mixed_set_options.restype = None
        L.jsvd_mixed_svd.argtypes = [P, S, S, ctypes.POINTER(Config), P, P, P, P]
        L.jsvd_mixed_svd.restype = I
        L.jsvd_mixed_svd_device.argtypes = [P, S, S, ctypes.POINTER(Config), P, P, P, P, P]
        L.jsvd_mixed_svd_device.restype = I
        L.jsvd_mixed_stats_get.argtypes = [ctypes.POINTER(MixedStats)]
        L.jsvd_mixed_stats_get.restype = None
        L.jsvd_mixed_stats_reset.restype = None
        D, LG = ctypes.c_double, ctypes.c_long
        L.jsvd_dgemm_device.argtypes = [ctypes.c_char, ctypes.c_char, I, I, I, D, P, LG, P, LG, D, P, LG, I]
        L.jsvd_dgemm_device.restype = I
        L.jsvd_mixed_test_round.argtypes = [I, P, I, I, I, P]
        L.jsvd_mixed_test_round.restype = I
        L.jsvd_test_wait_limit.argtypes = [I, I, I, ctypes.POINTER(I), ctypes.POINTER(D)]
        L.jsvd_test_wait_limit.restype = I
        L.jsvd_mixed_builtin_tuning.argtypes = [ctypes.POINTER(I), I]
        L.jsvd_mixed_builtin_tuning.restype = I
        L.jsvd_mixed_sweep_history.argtypes = [ctypes.POINTER(I), ctypes.POINTER(ctypes.c_double),
                                               ctypes.POINTER(ctypes.c_ulonglong), I]
        L.jsvd_mixed_sweep_history.restype = I
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


class SvdResult(NamedTuple):
    u: np.ndarray | None
    sigma: np.ndarray
    v: np.ndarray | None
    sweeps: int


_HOST_ENTRIES = {"plain": "jsvd_plain_svd", "precond": "jsvd_precond_svd", "blockpair": "jsvd_blockpair_svd",
                 "blocked": "jsvd_blocked_svd", "mixed": "jsvd_mixed_svd"}


def svd(a: np.ndarray, solver: str = "plain", cfg: Config | None = None, want_u: bool = True,
        want_v: bool = True) -> SvdResult:
    """One-sided Jacobi SVD of a row-major host matrix (rows >= columns)
    through the chosen solver's host-buffer entry point.  "plain" is the
    reference's arithmetic bit for bit; "precond", "blockpair", "blocked" and
    "mixed" are accurate to working precision.  sigma is unsorted, as the reference
    returns it; U and V are row-major."""
    if solver not in _HOST_ENTRIES:
        raise ValueError(f"solver must be one of {sorted(_HOST_ENTRIES)}")
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError("expected a 2-D matrix")
    m, n = a.shape
    cfg = cfg or default_config()
    u = np.empty((m, n)) if want_u else None
    s = np.empty(n)
    v = np.empty((n, n)) if want_v else None
    sw = ctypes.c_int(0)
    fn = getattr(lib(), _HOST_ENTRIES[solver])
    check(fn(a.ctypes.data if a.size else None, m, n, ctypes.byref(cfg), u.ctypes.data if u is not None else None,
             s.ctypes.data, v.ctypes.data if v is not None else None, ctypes.byref(sw)))
    return SvdResult(u, s, v, sw.value)


def plain_svd(a: np.ndarray, cfg: Config | None = None, want_u: bool = True, want_v: bool = True) -> SvdResult:
    """Host-buffer plain solve -> (U or None, sigma, V or None, sweeps)."""
    return svd(a, "plain", cfg, want_u, want_v)


def precond_svd(a: np.ndarray, cfg: Config | None = None, want_u: bool = True, want_v: bool = True) -> SvdResult:
    """Host-buffer QR-preconditioned solve -> (U or None, sigma, V or None, sweeps on R^T)."""
    return svd(a, "precond", cfg, want_u, want_v)


def precond_svd_device(d_a, m: int, n: int, d_u, d_sigma, d_v, cfg: Config | None = None, stream: int = 0) -> int:
    cfg = cfg or default_config()
    sw = ctypes.c_int(0)
    check(lib().jsvd_precond_svd_device(d_a, m, n, ctypes.byref(cfg), d_u, d_sigma, d_v, ctypes.byref(sw),
                                        stream or None))
    return sw.value


def blocked_svd_device(d_a, m: int, n: int, d_u, d_sigma, d_v, cfg: Config | None = None, stream: int = 0) -> int:
    cfg = cfg or default_config()
    sw = ctypes.c_int(0)
    check(lib().jsvd_blocked_svd_device(d_a, m, n, ctypes.byref(cfg), d_u, d_sigma, d_v, ctypes.byref(sw),
                                        stream or None))
    return sw.value


def blocked_stats() -> BlockedStats:
    st = BlockedStats()
    lib().jsvd_blocked_stats_get(ctypes.byref(st))
    return st


def blocked_stats_reset() -> None:
    lib().jsvd_blocked_stats_reset()


def blockpair_svd_device(d_a, m: int, n: int, d_u, d_sigma, d_v, cfg: Config | None = None, stream: int = 0) -> int:
    """Device-buffer block-pair Jacobi solve on raw pointers; returns outer sweeps."""
    cfg = cfg or default_config()
    sw = ctypes.c_int(0)
    check(lib().jsvd_blockpair_svd_device(d_a, m, n, ctypes.byref(cfg), d_u, d_sigma, d_v, ctypes.byref(sw),
                                          stream or None))
    return sw.value


def blockpair_svd(a: np.ndarray, cfg: Config | None = None, device=None):
    """Block-pair solve of a host matrix through the device entry point
    (torch buffers) -> (U, sigma, V, outer sweeps)."""
    import torch

    dev = device or torch.device("cuda", torch.cuda.current_device())
    a = np.ascontiguousarray(a, dtype=np.float64)
    m, n = a.shape
    da = torch.from_numpy(a).to(dev)
    du = torch.empty((m, n), dtype=torch.float64, device=dev)
    ds = torch.empty(n, dtype=torch.float64, device=dev)
    dv = torch.empty((n, n), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    sw = blockpair_svd_device(da.data_ptr(), m, n, du.data_ptr(), ds.data_ptr(), dv.data_ptr(), cfg)
    return du.cpu().numpy(), ds.cpu().numpy(), dv.cpu().numpy(), sw


def blockpair_set_variant(block_columns: int = 0, threads: int = 0) -> None:
    lib().jsvd_blockpair_set_variant(block_columns, threads)


def blockpair_stats() -> BlockPairStats:
    st = BlockPairStats()
    lib().jsvd_blockpair_stats_get(ctypes.byref(st))
    return st


def blockpair_stats_reset() -> None:
    lib().jsvd_blockpair_stats_reset()


def precond_set_inner(engine: int) -> None:
    """0 = block-pair Jacobi stage where it applies, 1 = plain sweep (default)."""
    lib().jsvd_precond_set_inner(engine)


def precond_set_gram_stop(enable: bool) -> None:
    """True (default): the precond path's final, rotation-free sweep is
    replaced by a test of every pair on the Gram matrix."""
    lib().jsvd_precond_set_gram_stop(1 if enable else 0)


def precond_stats() -> PrecondStats:
    st = PrecondStats()
    lib().jsvd_precond_stats_get(ctypes.byref(st))
    return st


def precond_stats_reset() -> None:
    lib().jsvd_precond_stats_reset()


def mixed_options(**overrides) -> MixedOptions:
    """The library's default mixed-path options with `overrides` applied."""
    o = MixedOptions()
    lib().jsvd_mixed_options_default(ctypes.byref(o))
    for k, v in overrides.items():
        setattr(o, k, v)
    return o


def mixed_set_options(opts: MixedOptions | None = None, **overrides) -> None:
    """Sets the calling thread's mixed-path options (defaults when None)."""
    if opts is None and not overrides:
        lib().jsvd_mixed_set_options(None)
        return
    o = opts if opts is not None else mixed_options()
    for k, v in overrides.items():
        setattr(o, k, v)
    lib().jsvd_mixed_set_options(ctypes.byref(o))


def mixed_svd(a: np.ndarray, cfg: Config | None = None, want_u: bool = True, want_v: bool = True) -> SvdResult:
    """Host-buffer blocked mixed-precision solve (tcgen05 3xTF32 phase + FP64 refinement)."""
    return svd(a, "mixed", cfg, want_u, want_v)


def mixed_svd_device(d_a, m: int, n: int, d_u, d_sigma, d_v, cfg: Config | None = None, stream: int = 0) -> int:
    cfg = cfg or default_config()
    sw = ctypes.c_int(0)
    check(lib().jsvd_mixed_svd_device(d_a, m, n, ctypes.byref(cfg), d_u, d_sigma, d_v, ctypes.byref(sw),
                                      stream or None))
    return sw.value


def mixed_stats() -> MixedStats:
    st = MixedStats()
    lib().jsvd_mixed_stats_get(ctypes.byref(st))
    return st


def mixed_stats_reset() -> None:
    lib().jsvd_mixed_stats_reset()


def mixed_sweep_history() -> list[tuple[int, float, int]]:
    """(phase, largest scaled off-diagonal, rotated block pairs) per sweep of the last mixed solve."""
    cap = 64
    ph = (ctypes.c_int * cap)()
    off = (ctypes.c_double * cap)()
    rot = (ctypes.c_ulonglong * cap)()
    n = lib().jsvd_mixed_sweep_history(ph, off, rot, cap)
    return [(int(ph[i]), float(off[i]), int(rot[i])) for i in range(min(n, cap))]


def mixed_test_round(kind: int, d_x, rows: int, cols: int, rnd: int, d_gw) -> None:
    """One block round of the mixed engine's kernels (0 TC Gram, 1 FP64 Gram, 2 TC rotation, 3 FP64 rotation)."""
    check(lib().jsvd_mixed_test_round(kind, d_x, rows, cols, rnd, d_gw))


def mixed_builtin_tuning() -> list[tuple[int, int, int, int]]:
    """The mixed path's built-in tuning table: (max_cols (0 = any),
    tc_max_sweeps, inner_sweeps, gram_splits) per entry, in lookup order."""
    n = lib().jsvd_mixed_builtin_tuning(None, 0)
    buf = (ctypes.c_int * (4 * n))()
    lib().jsvd_mixed_builtin_tuning(buf, n)
    return [tuple(buf[4 * i:4 * i + 4]) for i in range(n)]


def mixed_resolved_options(cols: int, opts: MixedOptions | None = None) -> MixedOptions:
    """The options a mixed solve of `cols` columns runs with: the automatic
    fields of `opts` (defaults when None) filled from the built-in table, as
    the library does."""
    o = opts if opts is not None else mixed_options()
    table = mixed_builtin_tuning()
    t = next((e for e in table if e[0] == 0 or cols <= e[0]), table[-1])
    r = MixedOptions()
    ctypes.memmove(ctypes.byref(r), ctypes.byref(o), ctypes.sizeof(MixedOptions))
    if r.tc_max_sweeps < 0:
        r.tc_max_sweeps = t[1]
    if r.inner_sweeps <= 0:
        r.inner_sweeps = t[2]
    if r.gram_splits <= 0:
        r.gram_splits = t[3]
    return r


def test_wait_limit(which: int, limit_ms: int, preset: bool = False) -> tuple[int, int, float]:
    """Runs one bounded device wait with a short limit: which 0 = the
    persistent sweep's wait on another CTA's round flag, 1 = the tensor-core
    kernels' mbarrier wait.  With preset the awaited flag is set (the barrier
    arrived on) beforehand.  Returns (return code, device status word,
    elapsed ms); a wait that ran out gives JSVD_ERR_RUNTIME and status 2."""
    st = ctypes.c_int(-1)
    ms = ctypes.c_double(0.0)
    rc = lib().jsvd_test_wait_limit(which, limit_ms, 1 if preset else 0, ctypes.byref(st), ctypes.byref(ms))
    return int(rc), int(st.value), float(ms.value)


def dgemm_device(op_a: str, op_b: str, m: int, n: int, k: int, alpha: float, d_a, lda: int, d_b, ldb: int,
                 beta: float, d_c, ldc: int, lower: bool = False) -> None:
    """C = alpha op(A) op(B) + beta C on column-major device buffers (the library's DMMA GEMM)."""
    check(lib().jsvd_dgemm_device(op_a.encode(), op_b.encode(), m, n, k, alpha, d_a, lda, d_b, ldb, beta, d_c, ldc,
                                  1 if lower else 0))


def plain_svd_device(d_a, m: int, n: int, d_u, d_sigma, d_v, cfg: Config | None = None, stream: int = 0) -> int:
    """Device-buffer plain solve on raw pointers (ints); returns sweeps."""
    cfg = cfg or default_config()
    sw = ctypes.c_int(0)
    rc = lib().jsvd_plain_svd_device(d_a, m, n, ctypes.byref(cfg), d_u, d_sigma, d_v, ctypes.byref(sw),
                                     stream or None)
    check(rc)
    return sw.value


def set_vpass_in_global(enable: bool) -> None:
    """Forces the plain path's deferred V pass to rotate V in place in global
    memory (the form used by itself above 25600 columns) for plans created
    afterwards; same bytes either way."""
    lib().jsvd_plain_set_vpass_in_global(1 if enable else 0)


def set_sweep_mode(mode: int) -> None:
    """0 = per-round kernels in a replayed graph, angle derived once per CTA
    (default), 1 = persistent sweep, 2 = as 0 with programmatic dependent
    launch, 3 = as 0 with every warp deriving the angle."""
    lib().jsvd_plain_set_sweep_mode(mode)


def plain_stats() -> PlainStats:
    st = PlainStats()
    lib().jsvd_plain_stats_get(ctypes.byref(st))
    return st


def plain_stats_reset() -> None:
    lib().jsvd_plain_stats_reset()


class DeviceBatch:
    """A batch of matrices packed on the device (torch tensors), ready for
    jsvd_batch_svd_device.  Outputs are packed in input order."""

    def __init__(self, mats, device, f32: bool = False, want_u: bool = False, want_v: bool = True):
        import torch

        self.count = len(mats)
        self.rows = np.array([a.shape[0] for a in mats], dtype=np.int32)
        self.cols = np.array([a.shape[1] for a in mats], dtype=np.int32)
        sizes = self.rows.astype(np.int64) * self.cols
        self.a_off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        self.s_off = np.concatenate([[0], np.cumsum(self.cols)[:-1]]).astype(np.int64)
        self.v_off = np.concatenate([[0], np.cumsum(self.cols.astype(np.int64) ** 2)[:-1]]).astype(np.int64)
        dt = np.float32 if f32 else np.float64
        packed = np.concatenate([np.ascontiguousarray(a, dtype=dt).ravel() for a in mats])
        self.f32 = f32
        self.h2d_bytes = packed.nbytes
        self.host_a = torch.from_numpy(packed)
        self.a = self.host_a.to(device)
        self.sigma = torch.empty(int(self.cols.sum()), dtype=torch.float64, device=device)
        self.v = torch.empty(int((self.cols.astype(np.int64) ** 2).sum()), dtype=torch.float64,
                             device=device) if want_v else None
        self.u = torch.empty(int(sizes.sum()), dtype=torch.float64, device=device) if want_u else None
        self.sweeps = np.zeros(self.count, dtype=np.int32)

    def solve(self, cfg: Config | None = None, tuning=None, stream: int = 0) -> None:
        cfg = cfg or default_config()
        tun = None
        if tuning is not None:
            # one (threads, ctas_per_sm[, max_ctas]) tuple per size class; missing classes keep defaults
            ents = [BatchTuning(*t) for t in tuning] + [BatchTuning(0, 0, 0)] * (5 - len(tuning))
            tun = (BatchTuning * 5)(*ents[:5])
        rc = lib().jsvd_batch_svd_device(
            self.count, self.rows.ctypes.data, self.cols.ctypes.data, self.a_off.ctypes.data, self.a.data_ptr(),
            1 if self.f32 else 0, ctypes.byref(cfg), self.sigma.data_ptr(),
            self.v.data_ptr() if self.v is not None else None,
            self.u.data_ptr() if self.u is not None else None, self.sweeps.ctypes.data, tun, stream or None)
        check(rc)

    def autotune(self, cfg: Config | None = None, sample: int = 0, reps: int = 2,
                 stream: int = 0) -> BatchAutotuneReport:
        """jsvd_batch_autotune on this batch (computing U and V as this batch
        was set up to)."""
        cfg = cfg or default_config()
        rep = BatchAutotuneReport()
        rc = lib().jsvd_batch_autotune(
            self.count, self.rows.ctypes.data, self.cols.ctypes.data, self.a_off.ctypes.data, self.a.data_ptr(),
            1 if self.f32 else 0, ctypes.byref(cfg), sample, reps, 1 if self.u is not None else 0,
            1 if self.v is not None else 0, ctypes.byref(rep), stream or None)
        check(rc)
        return rep

    def results(self):
        s = self.sigma.cpu().numpy()
        v = self.v.cpu().numpy() if self.v is not None else None
        u = self.u.cpu().numpy() if self.u is not None else None
        out = []
        for k in range(self.count):
            m, n = int(self.rows[k]), int(self.cols[k])
            sk = s[self.s_off[k]: self.s_off[k] + n]
            vk = v[self.v_off[k]: self.v_off[k] + n * n].reshape(n, n) if v is not None else None
            uk = u[self.a_off[k]: self.a_off[k] + m * n].reshape(m, n) if u is not None else None
            out.append((uk, sk, vk, int(self.sweeps[k])))
        return out


def residuals(a, u, s, v) -> dict:
    """rho_A, rho_U, rho_V and sigma_max of one result (jsvd_residuals, host
    threads); a and u may be None (their metrics are then -1)."""
    s = np.ascontiguousarray(s, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    n = s.shape[0]
    m = u.shape[0] if u is not None else (a.shape[0] if a is not None else n)
    a = np.ascontiguousarray(a, dtype=np.float64) if a is not None else None
    u = np.ascontiguousarray(u, dtype=np.float64) if u is not None else None
    rep = ResidualReport()
    check(lib().jsvd_residuals(a.ctypes.data if a is not None else None, u.ctypes.data if u is not None else None,
                               s.ctypes.data, v.ctypes.data, m, n, ctypes.byref(rep)))
    return {"rho_A": rep.rho_a, "rho_U": rep.rho_u, "rho_V": rep.rho_v, "sigma_max": rep.sigma_max}


def round_robin_schedule(n: int, form: int = 1) -> np.ndarray:
    """The library's pair schedule for n columns as an array (rounds, n/2, 2):
    form 0 = the plain path's uploaded table, 1 = the kernels' closed form."""
    need = ctypes.c_size_t(0)
    check(lib().jsvd_round_robin_schedule(n, form, None, 0, ctypes.byref(need)))
    out = np.empty(need.value, dtype=np.int32)
    check(lib().jsvd_round_robin_schedule(n, form, out.ctypes.data if out.size else None, out.size,
                                          ctypes.byref(need)))
    half = n // 2
    rounds = need.value // (2 * half) if half else 0
    return out.reshape(rounds, half, 2)


def batch_builtin_tuning() -> list[tuple[int, int, int]]:
    """The batched solver's compiled-in launch shapes, (threads, ctas_per_sm,
    max_ctas) per size class."""
    out = (BatchTuning * 5)()
    lib().jsvd_batch_builtin_tuning(out)
    return [(t.threads, t.ctas_per_sm, t.max_ctas) for t in out]


def batch_set_cluster_classes(mask: int) -> int:
    """Size classes (bit c = class c; 2, 3, 4 only) whose members the batched
    solver runs on thread-block clusters; returns the previous mask."""
    old = ctypes.c_int(0)
    check(lib().jsvd_batch_set_cluster_classes(int(mask), ctypes.byref(old)))
    return old.value


def probe_fp64_tflops() -> float:
    x = ctypes.c_double(0.0)
    check(lib().jsvd_probe_fp64_tflops(ctypes.byref(x)))
    return x.value


class Server:
    """Serving core (jsvd_server_*): submit host matrices, wait for results."""

    def __init__(self, cfg: Config | None = None, budget_bytes: int = 0, small_workers: int = 0,
                 large_workers: int = 0, max_batch: int = 0, large_path: int = 0):
        opt = ServerOptions()
        lib().jsvd_server_options_default(ctypes.byref(opt))
        if cfg is not None:
            opt.cfg = cfg
        if budget_bytes:
            opt.device_budget_bytes = budget_bytes
        if small_workers:
            opt.small_workers = small_workers
        if large_workers:
            opt.large_workers = large_workers
        if max_batch:
            opt.max_batch = max_batch
        opt.large_path = large_path
        h = ctypes.c_void_p()
        check(lib().jsvd_server_create(ctypes.byref(opt), ctypes.byref(h)))
        self.h = h
        self.shapes = {}

    def submit(self, a: np.ndarray, want_u: bool = False) -> int:
        a = np.ascontiguousarray(a, dtype=np.float64)
        t = ctypes.c_uint64(0)
        check(lib().jsvd_server_submit(self.h, a.ctypes.data, a.shape[0], a.shape[1], int(want_u), ctypes.byref(t)))
        self.shapes[t.value] = (a.shape[0], a.shape[1], want_u)
        return t.value

    def wait(self, ticket: int):
        m, n, want_u = self.shapes.pop(ticket)
        u = np.empty((m, n)) if want_u else None
        s = np.empty(n)
        v = np.empty((n, n))
        sw = ctypes.c_int(0)
        lat = ctypes.c_double(0.0)
        check(lib().jsvd_server_wait(self.h, ticket, u.ctypes.data if u is not None else None, s.ctypes.data,
                                     v.ctypes.data, ctypes.byref(sw), ctypes.byref(lat)))
        return u, s, v, sw.value, lat.value

    def poll(self, ticket: int) -> bool:
        """True when the request has finished (wait() will not block)."""
        done = ctypes.c_int(0)
        check(lib().jsvd_server_poll(self.h, ticket, ctypes.byref(done)))
        return bool(done.value)

    def stats(self) -> ServerStats:
        st = ServerStats()
        check(lib().jsvd_server_get_stats(self.h, ctypes.byref(st)))
        return st

    def close(self) -> None:
        if self.h:
            lib().jsvd_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def batch_stats() -> BatchStats:
    st = BatchStats()
    lib().jsvd_batch_stats_get(ctypes.byref(st))
    return st


def batch_stats_reset() -> None:
    lib().jsvd_batch_stats_reset()


def auto_tune_layout(cfg: Config | None = None) -> AutoTuneReport:
    cfg = cfg or default_config()
    rep = AutoTuneReport()
    check(lib().jsvd_auto_tune_layout(ctypes.byref(cfg), ctypes.byref(rep)))
    return rep
