"""The solve-kernel tuning table and its JSON cache, through the C ABI (no GPU).

Keys are (bucket, covariance type, precision); settings come from overrides,
from the cache file the offline tuner writes (geo_bsd/tune_cache.json) or
from timing in tuning mode. Checked here: built-in picks, overrides and their
validity rules, a save / reset / load round trip, the reader's tolerance of the
timing objects, its rejection of invalid entries, and the mode switch.
"""
import json
import os

import pytest

from geo_bsd import hpgl_wrap as W
from geo_bsd import tune as T


@pytest.fixture(autouse=True)
def _restore_table():
    T.reset()
    yield
    T.reset()
    T._load_default()


def test_builtin_picks_and_overrides():
    assert W.solve_variant(32, 1, W.FP32_REFINED) == W.VARIANT_QUAD
    assert W.solve_variant(64, 1, W.FP32_REFINED) == W.VARIANT_WIDE
    assert W.solve_variant(64, 1, W.FP64_PLAIN) == W.VARIANT_WIDE
    assert W.solve_variant(32, 1, W.FP64_PLAIN) == W.VARIANT_FOLD
    assert W.solve_variant(16, 2, W.FP64_PLAIN, W.VARIANT_FOLD_NARROW) == W.VARIANT_DEFAULT
    assert W.solve_variant(16, 2, W.FP64_PLAIN) == W.VARIANT_FOLD_NARROW
    assert W.solve_variant(16, 1, W.FP64_PLAIN) == W.VARIANT_FOLD  # other covariance types keep their pick
    with pytest.raises(ValueError):
        W.solve_variant(32, 1, W.FP64_PLAIN, W.VARIANT_QUAD)  # four rows per lane is FP32 only
    with pytest.raises(ValueError):
        W.solve_variant(64, 1, W.FP32_REFINED, W.VARIANT_QUAD_NARROW)  # bucket 64: WIDE and FOLD only
    assert W.solve_variant(64, 1, W.FP32_REFINED) == W.VARIANT_WIDE
    with pytest.raises(ValueError):
        W.solve_variant(32, 1, W.FP32_REFINED, W.VARIANT_WIDE)
    with pytest.raises(ValueError):
        W.solve_variant(24, 1, W.FP32_REFINED, W.VARIANT_FOLD)  # not a bucket
    with pytest.raises(ValueError):
        W.solve_variant(32, 3, W.FP32_REFINED, W.VARIANT_FOLD)  # not a covariance type


def test_cache_round_trip(tmp_path):
    W.solve_variant(8, 0, W.FP32_REFINED, W.VARIANT_FOLD)
    W.solve_variant(32, 2, W.FP32_REFINED, W.VARIANT_QUAD_NARROW)
    W.solve_variant(16, 1, W.FP64_PLAIN, W.VARIANT_FOLD_NARROW)
    path = str(tmp_path / "cache.json")
    assert T.save_cache(path) == 3
    entries = json.load(open(path))
    assert {(e["np"], e["cov_type"], e["precision"], e["variant"]) for e in entries} == {
        (8, 0, 1, "fold"), (32, 2, 1, "quad_narrow"), (16, 1, 0, "fold_narrow")}
    T.reset()
    assert W.solve_variant(32, 2, W.FP32_REFINED) == W.VARIANT_QUAD
    assert T.load_cache(path) == 3
    assert W.solve_variant(8, 0, W.FP32_REFINED) == W.VARIANT_FOLD
    assert W.solve_variant(32, 2, W.FP32_REFINED) == W.VARIANT_QUAD_NARROW
    assert W.solve_variant(16, 1, W.FP64_PLAIN) == W.VARIANT_FOLD_NARROW


def test_cache_reader_takes_names_numbers_and_timings(tmp_path):
    path = tmp_path / "cache.json"
    path.write_text(json.dumps([
        {"np": 32, "cov_type": 1, "precision": 1, "variant": "quad",
         "ms_per_million": {"fold": 4.8, "quad": 3.9, "fold_narrow": 5.1, "quad_narrow": 4.2}},
        {"precision": 0, "variant": 3, "cov_type": 0, "np": 8},
    ], indent=2))
    assert T.load_cache(str(path)) == 2
    assert W.solve_variant(32, 1, W.FP32_REFINED) == W.VARIANT_QUAD
    assert W.solve_variant(8, 0, W.FP64_PLAIN) == W.VARIANT_FOLD_NARROW


@pytest.mark.parametrize("entry", [
    {"np": 32, "cov_type": 1, "precision": 0, "variant": "quad"},   # FP64 has no four-rows kernel
    {"np": 12, "cov_type": 1, "precision": 1, "variant": "fold"},   # not a bucket
    {"np": 32, "cov_type": 1, "precision": 1, "variant": "fastest"},  # not a variant
    {"np": 32, "cov_type": 1, "variant": "fold"},                   # no precision
])
def test_cache_reader_rejects_invalid_entries(tmp_path, entry):
    path = tmp_path / "bad.json"
    path.write_text(json.dumps([entry]))
    with pytest.raises(RuntimeError):
        T.load_cache(str(path))
    assert "tune_load" in W.last_error()


@pytest.mark.timeout(60)
def test_truncated_cache_is_an_error_and_changes_nothing(tmp_path):
    """A file cut inside an entry's timing object, after a complete entry: an
    error (not a scan that restarts before the cut), and no entry applied."""
    good = {"np": 8, "cov_type": 0, "precision": 0, "variant": "fold_narrow"}
    cut = '{"np": 32, "cov_type": 1, "precision": 1, "variant": "quad", "ms_per_million": {"fold": 4.8'
    path = tmp_path / "cut.json"
    path.write_text("[" + json.dumps(good) + ", " + cut)
    before = W.solve_variant(8, 0, W.FP64_PLAIN)
    with pytest.raises(RuntimeError):
        T.load_cache(str(path))
    assert "tune_load" in W.last_error()
    assert W.solve_variant(8, 0, W.FP64_PLAIN) == before


def test_missing_cache_file_is_an_error(tmp_path):
    with pytest.raises(RuntimeError):
        T.load_cache(str(tmp_path / "absent.json"))


def test_tuning_mode_switch():
    assert T.mode(True) is False
    assert T.mode(False) is True
    assert T.mode(False) is False


def test_committed_cache_loads():
    """The cache shipped beside the package reads back to valid settings."""
    if not os.path.isfile(T.CACHE):
        pytest.skip("no committed tuning cache")
    n = T.load_cache(T.CACHE)
    assert n > 0
    entries = json.load(open(T.CACHE))
    assert len(entries) == n
    for e in entries:
        assert W.solve_variant(e["np"], e["cov_type"], e["precision"]) == [
            k for k, v in W.VARIANT_NAMES.items() if v == e["variant"]][0]
