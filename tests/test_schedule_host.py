"""The library's round-robin schedule, checked on the host (no GPU).

The plain path uploads a table built on the host; the batched, allocation-free
and V-pass kernels evaluate a closed form (round_robin_pair, compiled for host
and device from one definition).  Both must equal the oracle's restatement of
src/kernels.cu:637-678 pair for pair, orientation included, and every round
must hold disjoint pairs, so that the pairs of a round can run concurrently
without touching the same column: the race-freedom argument of the
one-sided sweep.
"""
import numpy as np
import pytest

import jsvd
import oracle as O

NS = list(range(1, 66)) + [127, 128, 129, 255, 256, 257, 511, 1000, 1023, 1024]


@pytest.mark.parametrize("n", NS)
def test_both_forms_equal_oracle_schedule(n):
    ref = O.schedule(n)
    for form in (0, 1):
        got = jsvd.round_robin_schedule(n, form)
        if n < 2:
            assert got.size == 0
            continue
        assert got.shape == (len(ref), n // 2, 2)
        assert [[tuple(map(int, pq)) for pq in rnd] for rnd in got] == ref, form


@pytest.mark.parametrize("n", NS)
def test_rounds_disjoint_and_every_pair_once(n):
    sched = jsvd.round_robin_schedule(n, 1)
    if n < 2:
        return
    seen = np.zeros((n, n), dtype=np.int32)
    for rnd in sched:
        cols = rnd.ravel()
        assert cols.min() >= 0 and cols.max() < n
        assert len(np.unique(cols)) == cols.size, "pairs of a round must be disjoint"
        lo = np.minimum(rnd[:, 0], rnd[:, 1])
        hi = np.maximum(rnd[:, 0], rnd[:, 1])
        assert np.all(lo < hi)
        np.add.at(seen, (lo, hi), 1)
    iu = np.triu_indices(n, 1)
    assert np.all(seen[iu] == 1) and seen.sum() == n * (n - 1) // 2


def test_large_n_closed_form_matches_table():
    for n in (4095, 4096, 8191, 8192):
        assert np.array_equal(jsvd.round_robin_schedule(n, 0), jsvd.round_robin_schedule(n, 1))


def test_schedule_argument_errors():
    import ctypes

    need = ctypes.c_size_t(0)
    L = jsvd.lib()
    assert L.jsvd_round_robin_schedule(0, 1, None, 0, ctypes.byref(need)) == jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert L.jsvd_round_robin_schedule(8, 2, None, 0, ctypes.byref(need)) == jsvd.JSVD_ERR_INVALID_ARGUMENT
    buf = (ctypes.c_int * 4)()
    assert L.jsvd_round_robin_schedule(8, 0, buf, 4, ctypes.byref(need)) == jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert need.value == 2 * 7 * 4
    assert jsvd.last_error()[1] == "Schedule buffer too small."
