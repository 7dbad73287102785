"""The allocation-free SK-weights entry point (hpgl_b200_sk_weights_noalloc).

It exists for callers that cannot allocate device memory while they run (their
GPU memory is owned by another allocator, or they work within a budget fixed
up front): it solves in a fixed device array instead of allocated buffers.
Checked through the C ABI against the regular entry point,
hpgl_simple_kriging_weights, on two calls in a row, against the oracle's FP64
weights, with the device's free memory unchanged over calls after the first,
plus its size limit. This file is collected last so that a run stopping at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import oracle as O
import pytest
import torch

from geo_bsd import hpgl_wrap as W
from geo_bsd import workloads as WL

pytestmark = pytest.mark.gpu

TOL = 1e-6  # relative, as the other FP32-output parity checks


def _covp(cov):
    return W._HPGL_COV_PARAMS(covariance_type=cov.cov_type, ranges=cov.ranges, angles=cov.angles, sill=cov.sill,
                              nugget=cov.nugget)


def _system(rng, n):
    xs, ys, zs = (rng.uniform(0, 30, n).astype(np.float32) for _ in range(3))
    centre = rng.uniform(5, 25, 3).astype(np.float32)
    return centre, xs, ys, zs


def _regular(centre, xs, ys, zs, cov):
    w = np.zeros(len(xs), np.float32)
    rc = W._hpgl_so.hpgl_simple_kriging_weights((C.c_float * 3)(*centre), xs, ys, zs, len(xs), C.byref(_covp(cov)), w)
    assert rc == 0, W.last_error()
    return w


def _noalloc(centre, xs, ys, zs, cov):
    w = np.zeros(len(xs), np.float32)
    rc = W._hpgl_so.hpgl_b200_sk_weights_noalloc((C.c_float * 3)(*centre), xs, ys, zs, len(xs),
                                                 C.byref(_covp(cov)), w, None)
    assert rc == 0, W.last_error()
    return w


@pytest.mark.parametrize("cov", [WL.CovSpec(WL.EXPONENTIAL, (20.0, 12.0, 8.0), (30.0, 0.0, 0.0), 1.0, 0.05),
                                 WL.CovSpec(WL.SPHERICAL, (25.0, 25.0, 10.0), (0.0, 0.0, 0.0), 2.0, 0.2),
                                 WL.CovSpec(WL.GAUSSIAN, (15.0, 15.0, 6.0), (10.0, 5.0, 0.0), 1.0, 0.1)])
def test_noalloc_matches_regular_entry_point_twice(cov):
    rng = np.random.default_rng(21)
    for n in (1, 12, 40, 128):
        sys_ = _system(rng, n)
        ref = _regular(*sys_, cov)
        first = _noalloc(*sys_, cov)
        second = _noalloc(*sys_, cov)  # the shared array keeps the previous call's contents
        scale = max(1.0, float(np.abs(ref).max()))
        assert np.abs(first - ref).max() <= TOL * scale
        assert np.abs(second - ref).max() <= TOL * scale
    # a smaller system right after a larger one in the same array
    small = _system(rng, 5)
    assert np.abs(_noalloc(*small, cov) - _regular(*small, cov)).max() <= TOL * 10


@pytest.mark.parametrize("cov", [WL.CovSpec(WL.EXPONENTIAL, (20.0, 12.0, 8.0), (30.0, 0.0, 0.0), 1.0, 0.05),
                                 WL.CovSpec(WL.SPHERICAL, (25.0, 25.0, 10.0), (0.0, 0.0, 0.0), 2.0, 0.2),
                                 WL.CovSpec(WL.GAUSSIAN, (15.0, 15.0, 6.0), (10.0, 5.0, 0.0), 1.0, 0.1)])
def test_noalloc_matches_oracle(cov):
    """Independent of the regular entry point: the CPU oracle's FP64 weights."""
    rng = np.random.default_rng(22)
    for n in (12, 40, 128):
        centre, xs, ys, zs = _system(rng, n)
        ref, _ = O.sk_weights("port", centre, xs, ys, zs, cov)
        assert ref is not None
        got = _noalloc(centre, xs, ys, zs, cov)
        scale = max(1.0, float(np.abs(ref).max()))
        assert np.abs(got.astype(np.float64) - ref).max() <= TOL * scale


def test_noalloc_allocates_nothing_after_the_first_call():
    """After a first call (which may load the kernel and its array onto the
    device), further calls leave the device's free memory unchanged."""
    rng = np.random.default_rng(23)
    cov = WL.CovSpec(WL.EXPONENTIAL, (20.0, 12.0, 8.0), (30.0, 0.0, 0.0), 1.0, 0.05)
    _noalloc(*_system(rng, 64), cov)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for n in (1, 64, 128, 7):
        _noalloc(*_system(rng, n), cov)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_sizes_beyond_its_array():
    rng = np.random.default_rng(3)
    centre, xs, ys, zs = _system(rng, 129)
    cov = WL.CovSpec(WL.EXPONENTIAL, (20.0, 20.0, 20.0), (0.0, 0.0, 0.0), 1.0, 0.0)
    w = np.zeros(129, np.float32)
    rc = W._hpgl_so.hpgl_b200_sk_weights_noalloc((C.c_float * 3)(*centre), xs, ys, zs, 129, C.byref(_covp(cov)), w,
                                                 None)
    assert rc == -4
    assert "128" in W.last_error()
    assert not w.any()
