"""jsvd_residuals (host, no GPU) against the oracle's numpy restatement of the
reference's validation metrics (tex/sections/03-gpu-parallel-reduction.tex:30-40):
rho_A = ||A - U S V^T||_F / max(1, ||A||_F), rho_U, rho_V = ||X^T X - I||_F.

The factors come from the FP64 host oracle (plain cyclic Jacobi) or from
LAPACK with planted perturbations, so both tiny and large residuals are
checked.  Agreement: within 1e-14 absolute plus 1e-10 relative (the two
implementations sum in different orders).
"""
import numpy as np
import pytest

import jsvd
import oracle as O


def _close(x, y):
    assert abs(x - y) <= 1e-14 + 1e-10 * abs(y), (x, y)


@pytest.mark.parametrize("m,n", [(1, 1), (2, 2), (7, 3), (40, 33), (130, 64), (257, 256)])
def test_residuals_match_oracle_on_oracle_factors(m, n):
    rng = np.random.default_rng(100 + m + n)
    a = rng.standard_normal((m, n))
    u, s, v, _ = O.plain_svd(a, eps=1e-13, threads=4)
    got = jsvd.residuals(a, u, s, v)
    ref = O.residuals(a, u, s, v)
    for k in ("rho_A", "rho_U", "rho_V"):
        _close(got[k], ref[k])
    assert got["sigma_max"] == s.max()
    assert got["rho_A"] < 1e-13 * max(n, 10) and got["rho_V"] < 1e-12 * max(n, 10)


def test_residuals_see_planted_errors():
    rng = np.random.default_rng(9)
    a = rng.standard_normal((60, 20))
    uu, s, vt = np.linalg.svd(a, full_matrices=False)
    v = vt.T.copy()
    u = uu.copy()
    u[3, 4] += 1e-6
    v[7, 2] -= 3e-5
    s2 = s.copy()
    s2[0] *= 1 + 1e-7
    got = jsvd.residuals(a, u, s2, v)
    ref = O.residuals(a, u, s2, v)
    for k in ("rho_A", "rho_U", "rho_V"):
        _close(got[k], ref[k])
        assert got[k] > 1e-9


def test_small_norm_uses_absolute_residual():
    """||A||_F < 1: rho_A divides by 1, not by the norm."""
    a = np.diag([1e-3, 5e-4, 0.0])
    u = np.eye(3)
    s = np.array([1e-3, 5e-4, 0.0])
    got = jsvd.residuals(a, u, s, np.eye(3))
    assert got["rho_A"] == 0.0
    # the zero-sigma column of U is left out of rho_U (the solver zeroes it)
    u0 = u.copy()
    u0[:, 2] = 0.0
    assert jsvd.residuals(a, u0, s, np.eye(3))["rho_U"] == 0.0
    a2 = a.copy()
    a2[0, 0] += 1e-6
    _close(jsvd.residuals(a2, u, s, np.eye(3))["rho_A"], 1e-6)


def test_optional_operands_and_errors():
    v = np.eye(4)
    s = np.ones(4)
    got = jsvd.residuals(None, None, s, v)
    assert got["rho_A"] == -1.0 and got["rho_U"] == -1.0 and got["rho_V"] == 0.0
    u = np.eye(6)[:, :4]
    got = jsvd.residuals(None, u, s, v)
    assert got["rho_A"] == -1.0 and got["rho_U"] == 0.0
    with pytest.raises(jsvd.JsvdError):
        jsvd.residuals(None, np.eye(3)[:, :2].T.copy(), np.ones(3), np.eye(3))  # rows < columns
