"""The simulations' dependency-level pass (k_sgs_levels) through hpgl_b200_sim_levels.

Bars: levels identical to a sequential CPU computation on random dependency
lists and on one long chain (every rank waiting on the one before, inside and
across warps); a rank that waits on itself (a level nothing publishes) makes
the bounded wait run out: the call returns ECUDA with "timed out" and the
next call on the same device succeeds.
"""
import ctypes as C

import numpy as np
import pytest

from geo_bsd import hpgl_wrap as W

pytestmark = pytest.mark.gpu


def _levels(nb):
    n, k = nb.shape
    out = np.zeros(n, np.int32)
    rc = W._hpgl_so.hpgl_b200_sim_levels(n, k, np.ascontiguousarray(nb, np.int32).ctypes.data, out.ctypes.data)
    return rc, out


def _cpu_levels(nb):
    lv = np.zeros(len(nb), np.int64)
    for r in range(len(nb)):
        deps = nb[r][nb[r] >= 0]
        lv[r] = 1 + lv[deps].max() if len(deps) else 0
    return lv


@pytest.mark.parametrize("n,k,frac_recent", [(50000, 12, 0.3), (120000, 32, 0.05)])
def test_levels_match_a_sequential_pass(n, k, frac_recent):
    rng = np.random.default_rng(n + k)
    r = np.arange(n)[:, None]
    far = (rng.random((n, k)) * r).astype(np.int64)                         # any lower rank
    near = r - 1 - (rng.random((n, k)) * np.minimum(r, 64)).astype(np.int64)  # a recent one
    nb = np.where(rng.random((n, k)) < frac_recent, near, far)
    nb[(rng.random((n, k)) < 0.2) | (nb < 0) | (r == 0)] = -1
    rc, got = _levels(nb.astype(np.int32))
    W.check(rc, "sim_levels")
    np.testing.assert_array_equal(got, _cpu_levels(nb))
    assert W.last_stats()["sgs_levels"] == got.max() + 1


def test_a_long_chain():
    n = 20000
    nb = np.full((n, 2), -1, np.int32)
    nb[1:, 0] = np.arange(n - 1)
    rc, got = _levels(nb)
    W.check(rc, "sim_levels")
    np.testing.assert_array_equal(got, np.arange(n))


def test_a_wait_that_nothing_ends_times_out_and_the_device_stays_usable():
    nb = np.full((64, 2), -1, np.int32)
    nb[1:, 0] = np.arange(63)
    nb[10, 1] = 10  # rank 10 waits for its own level
    rc, _ = _levels(nb)
    assert rc == W.ECUDA
    assert "timed out" in W.last_error()
    nb[10, 1] = -1
    rc, got = _levels(nb)
    W.check(rc, "sim_levels")
    np.testing.assert_array_equal(got, np.arange(64))
