"""Failure detection of the bounded device waits, without a GPU fault.

Every spin-wait in the library's kernels (the persistent sweep's acquire-load
wait on another CTA's round flag, the tensor-core kernels' mbarrier waits)
gives up after a wall-clock limit read from %globaltimer, writes a status word
and returns.  Here each wait is given a short limit on something that nothing
completes during the launch; the test checks the status word (2 = wait
timeout), the C error code (JSVD_ERR_RUNTIME) and message, that the launch
ended near the limit, and that the context still runs a solve afterwards.
The preset arm is the control: the flag is set beforehand and the wait ends
at once with status 0."""
import numpy as np
import pytest

import jsvd

pytestmark = pytest.mark.gpu

LIMIT_MS = 100


@pytest.mark.parametrize("which", [0, 1], ids=["round_flag", "mbarrier"])
def test_wait_runs_out_and_reports(cuda_device, which):
    rc, status, ms = jsvd.test_wait_limit(which, LIMIT_MS)
    assert rc == jsvd.JSVD_ERR_RUNTIME
    assert status == 2
    assert LIMIT_MS * 0.9 <= ms <= LIMIT_MS + 1000.0
    code, msg = jsvd.last_error()
    assert code == jsvd.JSVD_ERR_RUNTIME and "stopped at its limit" in msg
    # the context is still usable: a small solve runs and is correct
    a = np.random.default_rng(3).standard_normal((64, 48))
    u, s, v, sw = jsvd.plain_svd(a)
    assert np.max(np.abs(np.sort(s)[::-1] - np.linalg.svd(a, compute_uv=False))) < 1e-12


@pytest.mark.parametrize("which", [0, 1], ids=["round_flag", "mbarrier"])
def test_wait_completes_when_released(cuda_device, which):
    rc, status, ms = jsvd.test_wait_limit(which, LIMIT_MS, preset=True)
    assert rc == jsvd.JSVD_OK and status == 0
    assert ms < LIMIT_MS


def test_wait_limit_arguments(cuda_device):
    with pytest.raises(jsvd.InvalidArgument):
        jsvd.check(jsvd.test_wait_limit(2, LIMIT_MS)[0])
    with pytest.raises(jsvd.InvalidArgument):
        jsvd.check(jsvd.test_wait_limit(0, 0)[0])
