"""The mixed path's built-in tuning table (csrc/mixed_tuning_table.h) and its
generator (jacobi-svd-cuda_b200/mixed_autotune.py): the library carries the
committed table, the automatic options resolve from it by width, the
generator's text round-trips, and (on a GPU) one shape is tuned end to end."""
import os

import numpy as np
import pytest

import jsvd
import mixed_autotune as MA
from conftest import PKG

TABLE = os.path.join(PKG, "csrc", "mixed_tuning_table.h")


def test_library_carries_committed_table():
    assert jsvd.mixed_builtin_tuning() == MA.parse_table(open(TABLE).read())


def test_table_entries_are_usable():
    ents = jsvd.mixed_builtin_tuning()
    assert ents[-1][0] == 0
    bounds = [e[0] for e in ents[:-1]]
    assert bounds == sorted(bounds) and all(b >= 128 for b in bounds)
    for _, cap, inner, splits in ents:
        assert 0 <= cap <= 64 and 1 <= inner <= 8 and 0 <= splits <= 256


def test_automatic_options_resolve_by_width():
    ents = jsvd.mixed_builtin_tuning()
    for cols in (128, 1024, 2048, 2049, 4096, 30000):
        e = next(x for x in ents if x[0] == 0 or cols <= x[0])
        r = jsvd.mixed_resolved_options(cols)
        assert (r.tc_max_sweeps, r.inner_sweeps, r.gram_splits) == e[1:]
    # explicit values are kept
    r = jsvd.mixed_resolved_options(1024, jsvd.mixed_options(tc_max_sweeps=7, inner_sweeps=2, gram_splits=5))
    assert (r.tc_max_sweeps, r.inner_sweeps, r.gram_splits) == (7, 2, 5)


def test_render_parse_round_trip():
    ents = [(512, 3, 1, 0), (2048, 4, 2, 8), (0, 10, 1, 16)]
    text = MA.render_table(ents, ["note"], {"device": "dev", "date": "d", "workload": "w", "reps": 2})
    assert MA.parse_table(text) == ents


def test_parse_rejects_bad_tables():
    with pytest.raises(ValueError):
        MA.parse_table("#define JSVD_MIXED_TUNING_TABLE \\\n    { {512, 3, 1} }")
    with pytest.raises(ValueError):
        MA.parse_table("#define JSVD_MIXED_TUNING_TABLE \\\n    { {512, 3, 1, 0} }")


@pytest.mark.gpu
def test_tune_one_shape(cuda_device):
    r = MA.tune_shape(512, 256, reps=1, tc_caps=(0, 4), inner=(1,), splits=(0, 4))
    cap, inner, splits = r["best"]
    assert cap in (0, 4) and inner == 1 and splits in (0, 4)
    assert r["tried"] == 3 and r["rejected"] == 0
    assert np.isfinite(r["best_ms"]) and r["best_ms"] <= r["default_ms"] * 1.5
