"""Serving-core bookkeeping on the host: tickets, waits, budget admission and
counters (jsvd_server_*).

These run with or without a GPU.  Without one every request ends with a CUDA
error status; with one they succeed.  Either way each ticket is collected
exactly once, a second wait on it is rejected, and submitted = completed +
failed.  Submitters and waiters run in separate threads (ctypes releases the
GIL for the call), so waits overlap submits that grow the ticket table.
"""
import ctypes
import threading

import numpy as np
import pytest

import jsvd


def _server(**kw):
    opt = jsvd.ServerOptions()
    jsvd.lib().jsvd_server_options_default(ctypes.byref(opt))
    for k, v in kw.items():
        setattr(opt, k, v)
    h = ctypes.c_void_p()
    jsvd.check(jsvd.lib().jsvd_server_create(ctypes.byref(opt), ctypes.byref(h)))
    return h


def _submit(h, a):
    t = ctypes.c_uint64(0)
    rc = jsvd.lib().jsvd_server_submit(h, a.ctypes.data, a.shape[0], a.shape[1], 0, ctypes.byref(t))
    return rc, t.value


def _wait(h, ticket, n):
    s = np.empty(n)
    v = np.empty((n, n))
    sw = ctypes.c_int(0)
    lat = ctypes.c_double(0.0)
    return jsvd.lib().jsvd_server_wait(h, ticket, None, s.ctypes.data, v.ctypes.data, ctypes.byref(sw),
                                       ctypes.byref(lat))


def _stats(h):
    st = jsvd.ServerStats()
    jsvd.check(jsvd.lib().jsvd_server_get_stats(h, ctypes.byref(st)))
    return st


def test_request_over_budget_is_rejected_at_submit():
    h = _server(device_budget_bytes=64 * 1024)
    try:
        rc, _ = _submit(h, np.ones((80, 64)))  # needs 107,008 bytes
        assert rc == jsvd.JSVD_ERR_BUDGET
        assert "more than the serving budget of 65536" in jsvd.last_error()[1]
        rc, _ = _submit(h, np.ones((3, 4)))
        assert rc == jsvd.JSVD_ERR_INVALID_ARGUMENT
        assert _stats(h).submitted == 0
    finally:
        jsvd.lib().jsvd_server_destroy(h)


@pytest.mark.timeout(300)
def test_tickets_collected_once_under_concurrent_submit_and_wait():
    h = _server(small_workers=2, large_workers=2, max_batch=16)
    shapes = [(8, 4), (300, 260), (33, 17), (2, 2), (70, 64), (257, 200)] * 40
    rng = np.random.default_rng(5)
    mats = [rng.standard_normal(s) for s in shapes]
    tickets = [None] * len(mats)
    ready = [threading.Event() for _ in mats]
    results = [None] * len(mats)

    def submitter(lo, step):
        for i in range(lo, len(mats), step):
            rc, t = _submit(h, mats[i])
            assert rc == jsvd.JSVD_OK
            tickets[i] = t
            ready[i].set()

    def waiter(lo, step):
        for i in range(lo, len(mats), step):
            ready[i].wait()
            results[i] = _wait(h, tickets[i], mats[i].shape[1])

    try:
        ths = [threading.Thread(target=submitter, args=(k, 2)) for k in range(2)]
        ths += [threading.Thread(target=waiter, args=(k, 4)) for k in range(4)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        assert all(rc in (jsvd.JSVD_OK, jsvd.JSVD_ERR_CUDA) for rc in results), set(results)
        assert len(set(tickets)) == len(mats)
        st = _stats(h)
        assert st.submitted == len(mats)
        assert st.completed + st.failed == len(mats)
        assert st.completed == sum(rc == jsvd.JSVD_OK for rc in results)
        assert st.device_bytes_in_use == 0
        # a collected ticket cannot be waited on again; an unknown one neither
        for t in (tickets[0], max(tickets) + 1):
            assert _wait(h, t, 4) == jsvd.JSVD_ERR_INVALID_ARGUMENT
            assert jsvd.last_error()[1] == "Unknown or already collected ticket."
    finally:
        jsvd.lib().jsvd_server_destroy(h)


@pytest.mark.timeout(120)
def test_two_concurrent_waits_on_one_ticket():
    """Whatever the timing, exactly one of two threads waiting on the same
    ticket collects it; the other is rejected (ticket claimed or collected)."""
    h = _server(small_workers=1, large_workers=1)
    try:
        rng = np.random.default_rng(1)
        for shape in [(40, 30), (300, 260)] * 10:
            a = rng.standard_normal(shape)
            rc, t = _submit(h, a)
            assert rc == jsvd.JSVD_OK
            out = [None, None]
            ths = [threading.Thread(target=lambda k=k: out.__setitem__(k, _wait(h, t, shape[1]))) for k in range(2)]
            for th in ths:
                th.start()
            for th in ths:
                th.join()
            assert sorted(out) in ([jsvd.JSVD_OK, jsvd.JSVD_ERR_INVALID_ARGUMENT],
                                   [jsvd.JSVD_ERR_INVALID_ARGUMENT, jsvd.JSVD_ERR_CUDA]), out
    finally:
        jsvd.lib().jsvd_server_destroy(h)


def test_oversized_request_is_rejected_before_copy():
    h = _server()
    try:
        t = ctypes.c_uint64(0)
        rc = jsvd.lib().jsvd_server_submit(h, ctypes.c_void_p(16), 1 << 31, 1, 0, ctypes.byref(t))
        assert rc == jsvd.JSVD_ERR_OVERFLOW
        assert jsvd.last_error()[1] == "Matrix dimensions exceed the supported range."
        assert _stats(h).submitted == 0
    finally:
        jsvd.lib().jsvd_server_destroy(h)


@pytest.mark.timeout(120)
def test_poll_reports_completion_without_blocking():
    import time

    h = _server(small_workers=1, large_workers=1)
    try:
        a = np.random.default_rng(4).standard_normal((30, 20))
        rc, t = _submit(h, a)
        assert rc == jsvd.JSVD_OK
        done = ctypes.c_int(-1)
        deadline = time.monotonic() + 60.0
        while True:
            assert jsvd.lib().jsvd_server_poll(h, t, ctypes.byref(done)) == jsvd.JSVD_OK
            if done.value == 1 or time.monotonic() > deadline:
                break
            time.sleep(0.01)
        assert done.value == 1
        assert _wait(h, t, 20) in (jsvd.JSVD_OK, jsvd.JSVD_ERR_CUDA)
        for ticket in (t, t + 1000):
            assert jsvd.lib().jsvd_server_poll(h, ticket, ctypes.byref(done)) == jsvd.JSVD_ERR_INVALID_ARGUMENT
            assert jsvd.last_error()[1] == "Unknown or already collected ticket."
        rc, t2 = _submit(h, a)
        assert jsvd.lib().jsvd_server_poll(h, t2, None) == jsvd.JSVD_ERR_INVALID_ARGUMENT
        _wait(h, t2, 20)
    finally:
        jsvd.lib().jsvd_server_destroy(h)


@pytest.mark.timeout(120)
def test_destroy_fails_queued_requests_and_releases_their_waiter():
    """Destroying the server with requests still queued fails them and wakes
    a thread waiting on one; destroy returns once that thread has left the
    wait.  The waiter is known to be inside the wait (or past it) before
    destroy starts: a claimed ticket polls as invalid."""
    import time

    h = _server(small_workers=1, large_workers=1)
    a = np.random.default_rng(3).standard_normal((40, 30))
    tickets = [_submit(h, a)[1] for _ in range(300)]
    out = {}
    th = threading.Thread(target=lambda: out.__setitem__("rc", _wait(h, tickets[-1], 30)))
    th.start()
    done = ctypes.c_int(0)
    deadline = time.monotonic() + 60.0
    while jsvd.lib().jsvd_server_poll(h, tickets[-1], ctypes.byref(done)) == jsvd.JSVD_OK:
        assert time.monotonic() < deadline
        time.sleep(0.001)
    jsvd.lib().jsvd_server_destroy(h)
    th.join(timeout=60)
    assert not th.is_alive()
    assert out["rc"] in (jsvd.JSVD_OK, jsvd.JSVD_ERR_CUDA, jsvd.JSVD_ERR_RUNTIME)


@pytest.mark.parametrize("field,value,message", [
    ("epsilon", 0.0, "epsilon must be positive."),
    ("epsilon", -1.0, "epsilon must be positive."),
    ("max_sweeps", 0, "max_sweeps must be positive."),
])
def test_create_rejects_bad_settings(field, value, message):
    opt = jsvd.ServerOptions()
    jsvd.lib().jsvd_server_options_default(ctypes.byref(opt))
    setattr(opt.cfg, field, value)
    h = ctypes.c_void_p()
    assert jsvd.lib().jsvd_server_create(ctypes.byref(opt), ctypes.byref(h)) == jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert jsvd.last_error()[1] == message and not h.value


def test_options_defaults_and_null_handles():
    opt = jsvd.ServerOptions()
    jsvd.lib().jsvd_server_options_default(ctypes.byref(opt))
    assert opt.device_budget_bytes == 40 << 30 and opt.small_workers == 2 and opt.large_workers == 4
    assert opt.max_batch == 4096 and opt.large_path == 0 and opt.cfg.epsilon == 1e-9
    L = jsvd.lib()
    assert L.jsvd_server_create(ctypes.byref(opt), None) == jsvd.JSVD_ERR_INVALID_ARGUMENT
    t = ctypes.c_uint64(0)
    a = np.ones((2, 2))
    assert L.jsvd_server_submit(None, a.ctypes.data, 2, 2, 0, ctypes.byref(t)) == jsvd.JSVD_ERR_INVALID_ARGUMENT
    assert L.jsvd_server_wait(None, 1, None, None, None, None, None) == jsvd.JSVD_ERR_INVALID_ARGUMENT
    done = ctypes.c_int(0)
    assert L.jsvd_server_poll(None, 1, ctypes.byref(done)) == jsvd.JSVD_ERR_INVALID_ARGUMENT
    st = jsvd.ServerStats()
    assert L.jsvd_server_get_stats(None, ctypes.byref(st)) == jsvd.JSVD_ERR_INVALID_ARGUMENT
    L.jsvd_server_destroy(None)  # no-op


@pytest.fixture(scope="module")
def tsan_stress(tmp_path_factory):
    """tests/cpp/server_stress.cpp linked with the library's host code built
    under ThreadSanitizer (device code compiled as usual)."""
    import concurrent.futures
    import os
    import subprocess

    from conftest import PKG, ROOT

    d = tmp_path_factory.mktemp("tsan")
    src = os.path.join(PKG, "csrc")
    flags = ["-std=c++20", "-O1", "-g", "-gencode", "arch=compute_100a,code=sm_100a", "--fmad=false",
             "-Xcompiler", "-fsanitize=thread,-fPIC", "-I", os.path.join(ROOT, "include"), "-I", src]
    units = [os.path.join(src, f) for f in sorted(os.listdir(src)) if f.endswith(".cu")]
    units += [os.path.join(src, f + ".cpp") for f in ("server", "pipeline", "io", "kernels", "residuals")]
    units.append(os.path.join(ROOT, "tests", "cpp", "server_stress.cpp"))

    def build(path):
        obj = str(d / (os.path.basename(path) + ".o"))
        extra = ["-x", "cu"] if path.endswith(".cpp") else []
        subprocess.check_call(["nvcc", *flags, *extra, "-c", path, "-o", obj])
        return obj

    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(build, units))
    exe = str(d / "server_stress")
    subprocess.check_call(["g++", "-fsanitize=thread", *objs, "-o", exe, "-L/usr/local/cuda/lib64", "-lcublas",
                           "-lcudart", "-lpthread"])
    for obj in objs:
        os.remove(obj)
    yield exe
    os.remove(exe)  # the build is tens of MB


@pytest.mark.timeout(900)
def test_serving_core_has_no_data_races(tsan_stress, tmp_path):
    """Many submit / poll / wait / stats threads, destroy with a waiter, and
    the pipeline's reader and writer threads on its failure path, under
    ThreadSanitizer: no race reported, every request accounted for.
    (Without a GPU each request fails fast; the locking is exercised all the
    same.)"""
    import os
    import subprocess

    import torch

    if torch.cuda.is_available():
        pytest.skip("the stress relies on requests failing fast without a GPU")
    env = dict(os.environ, TSAN_OPTIONS="halt_on_error=1 exitcode=66")
    r = subprocess.run([tsan_stress, str(tmp_path)], capture_output=True, text=True, timeout=600, env=env)
    assert "ThreadSanitizer" not in r.stderr, r.stderr[-3000:]
    assert r.returncode == 0, (r.returncode, r.stderr[-2000:])
    assert r.stdout.split("\n")[0] == "mixed 800 800 800" and "destroy 10" in r.stdout
    assert "pipeline 20" in r.stdout  # every run failed cleanly (no device)
