"""The batched solver's launch-shape table and autotuner, host side (no GPU).

The built-in shapes are compiled from csrc/batch_tuning_table.h, which
batch_autotune.py writes from jsvd_batch_autotune; the library must carry the
committed table, and the generator's text must parse back to its report.
"""
import ctypes
import os

import numpy as np
import pytest

import batch_autotune as BA
import jsvd
from conftest import PKG

TABLE = os.path.join(PKG, "csrc", "batch_tuning_table.h")


def _parse_committed():
    with open(TABLE) as f:
        return BA.parse_table(f.read())


def test_library_carries_committed_table():
    assert jsvd.batch_builtin_tuning() == _parse_committed()


def test_committed_table_shapes_are_launchable():
    for c, (threads, ctas, cap) in enumerate(_parse_committed()):
        assert threads % 32 == 0 and 32 <= threads <= 512, c
        assert ctas >= 1 and threads * ctas <= 2048, c
        assert cap >= 0, c
        if c >= 3:
            assert ctas == 1, "classes 3-4 take a whole SM's shared memory per CTA"


def _fake_report():
    return {
        "best": [(128, 8, 0), (256, 2, 0), (512, 1, 0), (256, 1, 111), (512, 1, 74)],
        "builtin": [(256, 4, 0), (256, 2, 0), (512, 1, 0), (512, 1, 0), (512, 1, 0)],
        "best_ms": [1.5, 2.0, 3.0, 4.0, 5.0],
        "builtin_ms": [2.0, 2.0, 3.0, 4.5, 6.0],
        "members": [10, 3, 4, 0, 7],
        "sampled": [10, 3, 4, 0, 5],
        "candidates": [10, 7, 3, 0, 9],
    }


_FAKE_CLUSTER = {"mask": 0x14, "single_ms": [1.0, 2.0, 30.0, 40.0, 100.0], "cluster_ms": [0, 0, 20.0, 41.0, 60.0],
                 "note": "Timed on the same batch."}


def test_render_parse_round_trip():
    rep = _fake_report()
    text = BA.render_table(rep, {"device": "NVIDIA B200", "sms": 148, "date": "2026-01-01", "reps": 2,
                                 "workload": "test batch"}, _FAKE_CLUSTER)
    got = BA.parse_table(text)
    # a class without members keeps its built-in shape
    assert got == [rep["best"][0], rep["best"][1], rep["best"][2], rep["builtin"][3], rep["best"][4]]
    assert "#pragma once" in text and "NVIDIA B200" in text and "2.00 -> 1.50" in text
    assert BA.parse_cluster_mask(text) == 0x14
    assert " *   2: 30.0, 20.0 -> clusters" in text and " *   3: 40.0, 41.0 -> one CTA" in text


def test_library_default_cluster_classes_are_the_committed_table():
    with open(TABLE) as f:
        mask = BA.parse_cluster_mask(f.read())
    assert mask & ~BA.CLUSTER_CAPABLE == 0
    old = jsvd.batch_set_cluster_classes(mask)
    jsvd.batch_set_cluster_classes(old)
    # nothing else in this process has changed it, or the change was undone
    assert old == mask


def test_cluster_choice_needs_a_two_percent_gain():
    members = [5, 5, 5, 5, 5]
    single = [1.0, 1.0, 100.0, 100.0, 100.0]
    # clusters 1% faster for class 2, 10% faster for 3, 5% slower for 4
    clus = [1.0, 1.0, 99.0, 90.0, 105.0]
    assert BA.choose_cluster_mask(single, clus, members, previous=0) == 1 << 3
    # from all on: class 2 stays (single not > 2% faster), class 4 goes back to one CTA
    assert BA.choose_cluster_mask(single, clus, members, previous=0x1C) == (1 << 2) | (1 << 3)
    # a class without members keeps its previous choice
    assert BA.choose_cluster_mask(single, clus, [5, 5, 5, 0, 5], previous=0) == 0
    # bits outside the cluster-capable classes are dropped
    assert BA.choose_cluster_mask(single, single, members, previous=0x3) == 0


def test_parse_rejects_wrong_entry_count():
    with pytest.raises(ValueError):
        BA.parse_table("#define JSVD_BATCH_TUNING_TABLE { {256, 4, 0}, {256, 2, 0} }")


def test_autotune_rejects_bad_arguments_before_cuda():
    cfg = jsvd.default_config()
    rows = np.array([4], dtype=np.int32)
    cols = np.array([3], dtype=np.int32)
    off = np.array([0], dtype=np.int64)
    rep = jsvd.BatchAutotuneReport()
    L = jsvd.lib()
    rc = L.jsvd_batch_autotune(1, rows.ctypes.data, cols.ctypes.data, off.ctypes.data, 8, 0, ctypes.byref(cfg),
                               0, 2, 0, 1, None, None)
    assert rc == jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert jsvd.last_error()[1] == "Autotune report must not be null."
    rc = L.jsvd_batch_autotune(-1, rows.ctypes.data, cols.ctypes.data, off.ctypes.data, 8, 0, ctypes.byref(cfg),
                               0, 2, 0, 1, ctypes.byref(rep), None)
    assert rc == jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert jsvd.last_error()[1] == "count must be non-negative."
    rc = L.jsvd_batch_autotune(1, None, cols.ctypes.data, off.ctypes.data, 8, 0, ctypes.byref(cfg),
                               0, 2, 0, 1, ctypes.byref(rep), None)
    assert rc == jsvd.JSVD_ERR_INVALID_ARGUMENT
    bad = jsvd.default_config(threads_per_block=128)
    rc = L.jsvd_batch_autotune(1, rows.ctypes.data, cols.ctypes.data, off.ctypes.data, 8, 0, ctypes.byref(bad),
                               0, 2, 0, 1, ctypes.byref(rep), None)
    assert rc == jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert jsvd.last_error()[1] == "The batched solver reduces with threads_per_block = 256."


def test_batch_solver_rejects_bad_arguments_before_cuda():
    cfg = jsvd.default_config()
    rows = np.array([4], dtype=np.int32)
    cols = np.array([3], dtype=np.int32)
    off = np.array([0], dtype=np.int64)
    L = jsvd.lib()
    P = ctypes.c_void_p

    def call(count, r, c, o, a, sigma, c_cfg):
        return L.jsvd_batch_svd_device(count, r, c, o, a, 0, ctypes.byref(c_cfg), sigma, None, None, None, None,
                                       None)

    assert call(-1, rows.ctypes.data, cols.ctypes.data, off.ctypes.data, P(8), P(8), cfg) == \
        jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert jsvd.last_error()[1] == "count must be non-negative."
    assert call(1, rows.ctypes.data, cols.ctypes.data, off.ctypes.data, P(8), None, cfg) == \
        jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert jsvd.last_error()[1] == "Batch buffers must not be null."
    bad = jsvd.default_config(epsilon=0.0)
    assert call(1, rows.ctypes.data, cols.ctypes.data, off.ctypes.data, P(8), P(8), bad) == \
        jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert jsvd.last_error()[1] == "epsilon must be positive."
    bad = jsvd.default_config(threads_per_block=512)
    assert call(1, rows.ctypes.data, cols.ctypes.data, off.ctypes.data, P(8), P(8), bad) == \
        jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert jsvd.last_error()[1] == "The batched solver reduces with threads_per_block = 256."
    # an empty batch is a no-op
    assert call(0, None, None, None, None, None, cfg) == jsvd.JSVD_OK
