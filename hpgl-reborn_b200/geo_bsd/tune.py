"""The solve-kernel tuner (no counterpart in HPGL, which makes one LAPACK call
per node).

Every (neighbour-count bucket, covariance type, precision) key of the engine
runs one of the solve kernels' launch shapes (``hpgl_wrap.VARIANT_*``: two or
four rows of the system per lane, 512 / 384 / 256-thread blocks). The engine
starts from built-in picks; this module

* loads and saves the settings as a JSON cache (``load_cache`` /
  ``save_cache``; the package loads ``tune_cache.json`` beside this file at
  import, or the file named by ``HPGL_B200_TUNE_CACHE``, ``none`` for none);
* switches the engine's tuning mode (``mode``), in which the first bucket of
  at least 20000 systems of a key without a setting runs with every variant
  the key can run (each twice, the second run timed) and the fastest becomes
  its setting;
* rebuilds the cache (``autotune``): one synthetic ordinary-kriging grid per
  bucket and covariance type, run in tuning mode for each precision.

Command line: ``python -m geo_bsd.tune [--out PATH] [--scale S]`` (needs a
GPU) rewrites the cache and prints its keys.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os

import numpy as np

from . import hpgl_wrap as W
from . import workloads as WL

CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tune_cache.json")
BUCKETS = (8, 16, 32, 64)
COV_TYPES = (WL.SPHERICAL, WL.EXPONENTIAL, WL.GAUSSIAN)
PRECISIONS = (W.FP64_PLAIN, W.FP32_REFINED)


def load_cache(path: str = CACHE) -> int:
    """Reads a tuning cache (hpgl_b200_tune_load); returns the number of keys."""
    n = W._hpgl_so.hpgl_b200_tune_load(os.fsencode(path))
    if n < 0:
        W.check(n, "tune_load")
    return n


def save_cache(path: str = CACHE) -> int:
    """Writes every key that has a setting (hpgl_b200_tune_save)."""
    n = W._hpgl_so.hpgl_b200_tune_save(os.fsencode(path))
    if n < 0:
        W.check(n, "tune_save")
    return n


def reset() -> None:
    """Every key back to its built-in pick (hpgl_b200_tune_reset)."""
    W._hpgl_so.hpgl_b200_tune_reset()


def mode(on: bool) -> bool:
    """Tuning mode on / off (hpgl_b200_tune_mode); returns the previous mode."""
    return bool(W._hpgl_so.hpgl_b200_tune_mode(1 if on else 0))


def tuning_workload(bucket_np: int, cov_type: int, scale: float = 1.0) -> WL.Workload:
    """A 128x128x64 grid (scaled by `scale` per axis), 1% conditioning cells at
    seeded uniform positions with lognormal(0, 0.5) values, the covariance
    type with ranges (30, 15, 6), azimuth 30, sill 1, nugget 0.05, radiuses
    (30, 15, 6) and max_neighbours = bucket_np, so that nearly every cell's
    system falls in that bucket."""
    rng = np.random.default_rng(100 + 4 * bucket_np + cov_type)
    dims = tuple(max(4, int(round(d * scale))) for d in (128, 128, 64))
    n = dims[0] * dims[1] * dims[2]
    m = max(1, int(n * 0.01))
    idx = rng.choice(n, m, replace=False)
    data = np.full(n, WL.UNDEFINED, np.float32)
    mask = np.zeros(n, np.uint8)
    data[idx] = rng.lognormal(0.0, 0.5, m).astype(np.float32)
    mask[idx] = 1
    cov = WL.CovSpec(cov_type, (30.0, 15.0, 6.0), (30.0, 0.0, 0.0), 1.0, 0.05)
    return WL.Workload(f"tune_np{bucket_np}_cov{cov_type}", dims, data, mask, cov, (30, 15, 6), bucket_np)


def _ordinary_kriging(wl: WL.Workload, precision: int) -> dict:
    dims = (C.c_int * 3)(*wl.dims)
    data = np.ascontiguousarray(wl.data, np.float32)
    mask = np.ascontiguousarray(wl.mask, np.uint8)
    out_d, out_m = data.copy(), mask.copy()
    p = W._HPGL_SK_PARAMS(covariance_type=wl.cov.cov_type, ranges=tuple(wl.cov.ranges),
                          angles=tuple(wl.cov.angles), sill=wl.cov.sill, nugget=wl.cov.nugget,
                          radiuses=tuple(wl.radiuses), max_neighbours=wl.max_neighbours, automatic_mean=1, mean=0.0)
    opt = W._HPGL_B200_OPTIONS(precision=precision, refine_steps=2, flags=W.FLAG_OUT_IS_CLONE, stream=None,
                               estimate64=None, variance=None, status=None, ik_probs=None)
    rc = W._hpgl_so.hpgl_b200_cont_kriging_ex(0, dims, data.ctypes.data, mask.ctypes.data, C.byref(p),
                                              out_d.ctypes.data, out_m.ctypes.data, C.byref(opt))
    W.check(rc, "cont_kriging_ex")
    return W.last_stats()


def autotune(path: str = CACHE, scale: float = 1.0, buckets=BUCKETS, cov_types=COV_TYPES,
             precisions=PRECISIONS) -> list:
    """Times every variant of every key on its synthetic grid (tuning mode,
    buckets in increasing order so each key meets its own grid first) and
    writes the cache. Returns the cache's entries."""
    reset()
    prev = mode(True)
    try:
        for b in buckets:
            for ct in cov_types:
                wl = tuning_workload(b, ct, scale)
                for prec in precisions:
                    _ordinary_kriging(wl, prec)
    finally:
        mode(prev)
    save_cache(path)
    with open(path) as f:
        return json.load(f)


def _load_default() -> None:
    path = os.environ.get("HPGL_B200_TUNE_CACHE", CACHE)
    if path.lower() == "none" or not os.path.isfile(path):
        return
    load_cache(path)


def main() -> None:
    ap = argparse.ArgumentParser(description="rebuild the solve-kernel tuning cache (needs a GPU)")
    ap.add_argument("--out", default=CACHE)
    ap.add_argument("--scale", type=float, default=1.0)
    args = ap.parse_args()
    for e in autotune(args.out, args.scale):
        print(json.dumps(e))


if __name__ == "__main__":
    main()
