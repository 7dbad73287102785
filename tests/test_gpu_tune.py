"""The solve-kernel tuner on the GPU.

* Tuning mode: a call whose bucket of an untuned key holds at least 20000
  systems runs every variant the key can run, keeps the fastest as the key's
  setting, and its outputs are the chosen variant's (checked against the FP64
  oracle's statuses and within the precision's error bound).
* Every variant the table can pick gives the same statuses and meets the
  error bound (FP32-refined 1e-6, FP64 plain 1e-10 against the FP64 plain
  built-in pick), for the buckets up to 32 on the benchmark's model and for
  the 33-64 bucket on the clustered grid.
* The picks of the committed cache are not slower than the built-in picks
  on the benchmark's model (the bucket's kernel time, median of five calls,
  within 5 % for timing noise).
"""
import os

import numpy as np
import pytest

import helpers as H
from geo_bsd import hpgl_wrap as W
from geo_bsd import tune as T
from geo_bsd import workloads as WL

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _restore_table():
    T.reset()
    T.mode(False)
    yield
    T.mode(False)
    T.reset()
    T._load_default()


def _bucket32_ms(wl, precision, reps=5):
    H.engine_cont(0, wl, precision=precision)
    return float(np.median([H.engine_cont(0, wl, precision=precision)["stats"]["bucket_ms_2"] for _ in range(reps)]))


@pytest.mark.parametrize("precision", [0, 1])
def test_tuning_mode_sets_the_key_and_keeps_correct_outputs(precision):
    wl = WL.sk_ok_large(0.4)
    ref = H.engine_cont(0, wl, precision=0)
    assert W.solve_variant(32, wl.cov.cov_type, precision) in (W.VARIANT_FOLD, W.VARIANT_QUAD)
    T.mode(True)
    e = H.engine_cont(0, wl, precision=precision)
    T.mode(False)
    assert e["stats"]["bucket_items_2"] >= 20000
    assert W.solve_variant(32, wl.cov.cov_type, precision) != W.VARIANT_DEFAULT
    np.testing.assert_array_equal(e["status"], ref["status"])
    ok = ref["status"] == 0
    tol = 1e-10 if precision == 0 else 1e-6
    assert H.rel_err(e["est"][ok], ref["est"][ok]) <= tol
    assert H.rel_err(e["var"][ok], ref["var"][ok]) <= tol


@pytest.mark.parametrize("precision,variants", [(1, (1, 2, 3, 4, 5, 6)), (0, (1, 3))])
def test_every_variant_meets_the_bound(precision, variants):
    wl = WL.sk_ok_large(0.3)
    ref = H.engine_cont(0, wl, precision=0)
    ok = ref["status"] == 0
    tol = 1e-10 if precision == 0 else 1e-6
    for v in variants:
        for b in (8, 16, 32):
            if b == 32 or v not in (W.VARIANT_TILE, W.VARIANT_TILE_NARROW):
                W.solve_variant(b, wl.cov.cov_type, precision, v)
        for kind in (0, 1):
            r = ref if kind == 0 else H.engine_cont(1, wl, precision=0)
            e = H.engine_cont(kind, wl, precision=precision)
            np.testing.assert_array_equal(e["status"], r["status"])
            okk = r["status"] == 0
            assert H.rel_err(e["est"][okk], r["est"][okk]) <= tol, (v, kind)
            assert H.rel_err(e["var"][okk], r["var"][okk]) <= tol, (v, kind)
    assert ok.any()


@pytest.mark.parametrize("precision", [0, 1])
def test_bucket64_variants_meet_the_bound(precision):
    """The 33-64 bucket's two variants (WIDE, the built-in pick, and FOLD) on
    the clustered Gaussian grid with nugget 1e-3 (k = 64): statuses identical
    and estimates / variances within the precision's bound of the FP64
    built-in pick; escalated FP32 systems are re-solved in FP64."""
    wl = WL.clustered(0.25)
    cov = wl.cov.cov_type
    assert W.solve_variant(64, cov, precision) == W.VARIANT_WIDE
    ref = H.engine_cont(0, wl, precision=0)
    assert ref["stats"]["bucket_items_3"] > 1000
    ok = ref["status"] == 0
    assert ok.any()
    tol = 1e-10 if precision == 0 else 1e-6
    for v in (W.VARIANT_WIDE, W.VARIANT_FOLD):
        W.solve_variant(64, cov, precision, v)
        for kind in (0, 1):
            r = ref if kind == 0 else H.engine_cont(1, wl, precision=0)
            e = H.engine_cont(kind, wl, precision=precision)
            np.testing.assert_array_equal(e["status"], r["status"])
            okk = r["status"] == 0
            assert H.rel_err(e["est"][okk], r["est"][okk]) <= tol, (v, kind)
            assert H.rel_err(e["var"][okk], r["var"][okk]) <= tol, (v, kind)


@pytest.mark.parametrize("precision", [0, 1])
def test_cache_pick_not_slower_than_builtin(precision):
    if not os.path.isfile(T.CACHE):
        pytest.skip("no committed tuning cache")
    T.load_cache(T.CACHE)
    wl = WL.sk_ok_large(0.6)
    cov = wl.cov.cov_type
    picked = W.solve_variant(32, cov, precision)
    t_pick = _bucket32_ms(wl, precision)
    T.reset()
    builtin = W.solve_variant(32, cov, precision)
    t_builtin = _bucket32_ms(wl, precision)
    assert t_pick <= 1.05 * t_builtin, (picked, t_pick, builtin, t_builtin)
