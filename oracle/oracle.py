"""TEST INFRASTRUCTURE ONLY — ctypes access to the oracle.

Two checkers, both CPU:

* ``port``: oracle/lib/libkrige_oracle.so, this project's restatement of the
  reference's kriging path (oracle/krige_oracle.cpp);
* ``ref``:  oracle/_ref/libref_harness.so, the reference's own code compiled
  from its sources by oracle/Makefile (present wherever it was built; the
  product never loads either).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "lib", "libkrige_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_harness.so")
REF_API_PATH = os.path.join(HERE, "_ref", "libhpgl.so")

_i = C.POINTER(C.c_int)
_d = C.POINTER(C.c_double)
_f = C.POINTER(C.c_float)
_u8 = C.POINTER(C.c_ubyte)
_u32 = C.POINTER(C.c_uint)

_libs = {}


def _ptr(a, t):
    if a is None:
        return C.cast(None, t)
    return a.ctypes.data_as(t)


def _arr(v, dt):
    return np.ascontiguousarray(np.asarray(v, dtype=dt))


def load(which: str):
    """Load 'port' or 'ref'; raises OSError when the library is absent."""
    if which in _libs:
        return _libs[which]
    path = PORT_PATH if which == "port" else REF_PATH
    lib = C.CDLL(path)
    if which == "port":
        lib.ko_krige_cont.argtypes = [C.c_int, _i, _f, _u8, C.c_int, _d, _d, C.c_double, C.c_double,
                                      _i, C.c_int, C.c_double, _i, C.c_int, _i, _i, _u8, _d, _d,
                                      _f, _i, C.c_int, C.c_int]
        lib.ko_krige_lvm.argtypes = [_i, _f, _u8, _f, C.c_int, _d, _d, C.c_double, C.c_double, _i, C.c_int,
                                     _i, C.c_int, _i, _i, _u8, _d, _d, _f, _i, C.c_int, C.c_int]
        lib.ko_krige_ind.argtypes = [C.c_int, _i, _u8, _u8, C.c_int, C.c_int, _d, _d, C.c_double,
                                     C.c_double, _i, C.c_int, C.c_double, _i, C.c_int, _i, _i, _u8,
                                     _d, _d, _f, _i, C.c_int, C.c_int]
        lib.ko_cont_grid.argtypes = [C.c_int, _i, _f, _u8, C.c_int, _d, _d, C.c_double, C.c_double,
                                     _i, C.c_int, C.c_int, C.c_double, _f, _u8, _d, _d, _i, C.c_int]
        lib.ko_lvm_grid.argtypes = [_i, _f, _u8, _f, C.c_int, _d, _d, C.c_double, C.c_double, _i,
                                    C.c_int, _f, _u8, _d, _d, _i, C.c_int]
        lib.ko_indicator_grid.argtypes = [_i, _u8, _u8, C.c_int, _i, _d, _d, _d, _d, _i, _i, _d,
                                          _u8, _u8, _f, C.c_int]
        lib.ko_median_ik_grid.argtypes = [_i, _u8, _u8, C.c_int, _d, _d, C.c_double, C.c_double,
                                          _i, C.c_int, _d, _u8, _u8, _d, _i, C.c_int]
        lib.ko_sgs.argtypes = [_i, _f, _u8, _u8, _f, _f, C.c_longlong, _f, C.c_int, C.c_int, _d, _d, C.c_double,
                               C.c_double, _i, C.c_int, C.c_longlong, _i]
        lib.ko_sgs_path.argtypes = [C.c_longlong, C.c_longlong, _i, C.c_longlong]
        lib.ko_mt_draws.argtypes = [C.c_longlong, C.c_longlong, _d]
        lib.ko_sis.argtypes = [_i, _u8, _u8, _u8, C.c_int, _i, _d, _d, _d, _d, _i, _i, _d, C.c_void_p,
                               C.c_longlong, _i, C.c_int]
        lib.ko_cokriging.argtypes = [C.c_int, _i, _f, _u8, _f, _u8, C.c_int, _d, _d, C.c_double, C.c_double, C.c_int,
                                     _d, _d, C.c_double, C.c_double, _i, C.c_int, C.c_double, C.c_double,
                                     C.c_double, C.c_double, _f, _u8, _i, C.c_int]
        lib.ko_template.argtypes = [C.c_int, C.c_int, _d, _d, C.c_double, C.c_double, _i, _i,
                                    C.c_int, _i]
        lib.ko_cov.argtypes = [C.c_int, C.c_int, _d, _d, C.c_double, C.c_double, _i, _i, _i]
        lib.ko_cov.restype = C.c_double
        lib.ko_transform.argtypes = [_d, _d, _d]
        lib.ko_sk_weights.argtypes = [_d, _d, _d, _d, C.c_int, C.c_int, _d, _d, C.c_double,
                                      C.c_double, _d, _d]
        lib.ko_sort_check.argtypes = [_u32, C.c_int, _i, _i]
        lib.ko_sort_check.restype = None
        lib.ko_select_check.argtypes = [_u32, C.c_int, C.c_int, _i]
        lib.ko_select_check.restype = None
    else:
        lib.ref_krige_cont.argtypes = [C.c_int, _i, _f, _u8, C.c_int, _d, _d, C.c_double,
                                       C.c_double, _i, C.c_int, C.c_double, _i, C.c_int, _i, _i,
                                       _u8, _d, _d, _f, _i, C.c_int]
        lib.ref_krige_ind.argtypes = [C.c_int, _i, _u8, _u8, C.c_int, C.c_int, _d, _d, C.c_double,
                                      C.c_double, _i, C.c_int, C.c_double, _i, C.c_int, _i, _i,
                                      _u8, _d, _d, _f, _i, C.c_int]
        lib.ref_krige_lvm.argtypes = [_i, _f, _u8, _f, C.c_int, _d, _d, C.c_double, C.c_double, _i, C.c_int,
                                      _i, C.c_int, _i, _i, _u8, _d, _d, _f, _i, C.c_int]
        lib.ref_template.argtypes = [C.c_int, C.c_int, _d, _d, C.c_double, C.c_double, _i, _i,
                                     C.c_int, _i]
        lib.ref_cov.argtypes = [C.c_int, C.c_int, _d, _d, C.c_double, C.c_double, _i, _i, _i]
        lib.ref_cov.restype = C.c_double
        lib.ref_transform.argtypes = [_d, _d, _d]
        lib.ref_sk_weights.argtypes = [_d, _d, _d, _d, C.c_int, C.c_int, _d, _d, C.c_double,
                                       C.c_double, _d, _d]
    _libs[which] = lib
    return lib


def available(which: str) -> bool:
    try:
        load(which)
        return True
    except OSError:
        return False


def krige_nodes(which, kind, dims, data, mask, cov, radiuses, k, mean=0.0, nodes=None,
                ind_value: Optional[int] = None, precision=0, threads=0, want_idx=True, means=None):
    """Per-node kriging at `nodes` (default: every uninformed cell).

    kind 0 = OK (analytic covariance), 1 = SK / IK (truncated table),
    2 = median-IK flavour (truncated field; same values as 1). `means` (one
    float per grid cell) makes it LVM kriging (kind and mean are then unused).
    Returns a dict with idx (n,k; -1 padded), count, path (ref: template path
    flag; port: same), est (f64), var (f64), est_f (f32), status.
    """
    lib = load(which)
    dims_a = _arr(dims, np.int32)
    mask = _arr(mask, np.uint8)
    if nodes is None:
        nodes = np.flatnonzero(mask == 0)
    nodes = _arr(nodes, np.int32)
    n = len(nodes)
    out = {
        "idx": np.full((n, k), -1, np.int32) if want_idx else None,
        "count": np.zeros(n, np.int32),
        "path": np.zeros(n, np.uint8),
        "est": np.zeros(n, np.float64),
        "var": np.zeros(n, np.float64),
        "est_f": np.zeros(n, np.float32),
        "status": np.zeros(n, np.int32),
    }
    ranges = _arr(cov.ranges, np.float64)
    angles = _arr(cov.angles, np.float64)
    rad = _arr(radiuses, np.int32)
    common_tail = [_ptr(nodes, _i), n, _ptr(out["idx"], _i), _ptr(out["count"], _i),
                   _ptr(out["path"], _u8), _ptr(out["est"], _d), _ptr(out["var"], _d),
                   _ptr(out["est_f"], _f), _ptr(out["status"], _i)]
    if means is not None:
        data = _arr(data, np.float32)
        means = _arr(means, np.float32)
        head = [_ptr(dims_a, _i), _ptr(data, _f), _ptr(mask, _u8), _ptr(means, _f), int(cov.cov_type),
                _ptr(ranges, _d), _ptr(angles, _d), float(cov.sill), float(cov.nugget), _ptr(rad, _i), int(k)]
        if which == "port":
            rc = lib.ko_krige_lvm(*head, *common_tail, int(precision), int(threads))
        else:
            rc = lib.ref_krige_lvm(*head, *common_tail, int(threads))
    elif ind_value is None:
        data = _arr(data, np.float32)
        head = [kind, _ptr(dims_a, _i), _ptr(data, _f), _ptr(mask, _u8), int(cov.cov_type),
                _ptr(ranges, _d), _ptr(angles, _d), float(cov.sill), float(cov.nugget),
                _ptr(rad, _i), int(k), float(mean)]
        if which == "port":
            rc = lib.ko_krige_cont(*head, *common_tail, int(precision), int(threads))
        else:
            rc = lib.ref_krige_cont(*head, *common_tail, int(threads))
    else:
        data = _arr(data, np.uint8)
        head = [kind, _ptr(dims_a, _i), _ptr(data, _u8), _ptr(mask, _u8), int(ind_value),
                int(cov.cov_type), _ptr(ranges, _d), _ptr(angles, _d), float(cov.sill),
                float(cov.nugget), _ptr(rad, _i), int(k), float(mean)]
        if which == "port":
            rc = lib.ko_krige_ind(*head, *common_tail, int(precision), int(threads))
        else:
            rc = lib.ref_krige_ind(*head, *common_tail, int(threads))
    if rc != 0:
        raise RuntimeError(f"oracle {which} failed (rc={rc})")
    out["nodes"] = nodes
    return out


def template(which, kind, cov, radiuses, cap=None):
    lib = load(which)
    ranges = _arr(cov.ranges, np.float64)
    angles = _arr(cov.angles, np.float64)
    rad = _arr(radiuses, np.int32)
    if cap is None:
        cap = int((2 * rad[0] + 1) * (2 * rad[1] + 1) * (2 * rad[2] + 1))
    out = np.zeros((cap, 3), np.int32)
    lim = C.c_int(0)
    fn = lib.ko_template if which == "port" else lib.ref_template
    n = fn(kind, int(cov.cov_type), _ptr(ranges, _d), _ptr(angles, _d), float(cov.sill),
           float(cov.nugget), _ptr(rad, _i), _ptr(out, _i), cap, C.byref(lim))
    if n < 0:
        raise RuntimeError("template failed")
    return out[:n].copy(), lim.value


def transform(which, ranges, angles):
    lib = load(which)
    out = np.zeros(9, np.float64)
    fn = lib.ko_transform if which == "port" else lib.ref_transform
    rc = fn(_ptr(_arr(ranges, np.float64), _d), _ptr(_arr(angles, np.float64), _d), _ptr(out, _d))
    if rc != 0:
        raise ValueError("zero range")
    return out


def cov_point(which, kind, cov, radiuses, a, b):
    lib = load(which)
    fn = lib.ko_cov if which == "port" else lib.ref_cov
    return fn(kind, int(cov.cov_type), _ptr(_arr(cov.ranges, np.float64), _d),
              _ptr(_arr(cov.angles, np.float64), _d), float(cov.sill), float(cov.nugget),
              _ptr(_arr(radiuses, np.int32), _i), _ptr(_arr(a, np.int32), _i),
              _ptr(_arr(b, np.int32), _i))


def sk_weights(which, center, xs, ys, zs, cov):
    lib = load(which)
    n = len(xs)
    w = np.zeros(n, np.float64)
    var = C.c_double(0)
    fn = lib.ko_sk_weights if which == "port" else lib.ref_sk_weights
    ok = fn(_ptr(_arr(center, np.float64), _d), _ptr(_arr(xs, np.float64), _d),
            _ptr(_arr(ys, np.float64), _d), _ptr(_arr(zs, np.float64), _d), n, int(cov.cov_type),
            _ptr(_arr(cov.ranges, np.float64), _d), _ptr(_arr(cov.angles, np.float64), _d),
            float(cov.sill), float(cov.nugget), _ptr(w, _d), C.byref(var))
    return (w, var.value) if ok else (None, None)


def cont_grid(kind, dims, data, mask, cov, radiuses, k, mean=None, threads=0):
    """Whole-grid OK (kind 0) / SK (kind 1) with the reference's output rules (port)."""
    lib = load("port")
    data = _arr(data, np.float32)
    mask = _arr(mask, np.uint8)
    out_d = data.copy()
    out_m = mask.copy()
    est = np.zeros(len(data), np.float64)
    var = np.zeros(len(data), np.float64)
    st = np.zeros(len(data), np.int32)
    rc = lib.ko_cont_grid(kind, _ptr(_arr(dims, np.int32), _i), _ptr(data, _f), _ptr(mask, _u8),
                          int(cov.cov_type), _ptr(_arr(cov.ranges, np.float64), _d),
                          _ptr(_arr(cov.angles, np.float64), _d), float(cov.sill),
                          float(cov.nugget), _ptr(_arr(radiuses, np.int32), _i), int(k),
                          1 if mean is None else 0, 0.0 if mean is None else float(mean),
                          _ptr(out_d, _f), _ptr(out_m, _u8), _ptr(est, _d), _ptr(var, _d),
                          _ptr(st, _i), int(threads))
    if rc:
        raise RuntimeError("cont_grid failed")
    return out_d, out_m, est, var, st


def lvm_grid(dims, data, mask, means, cov, radiuses, k, threads=0):
    """Whole-grid LVM kriging with the reference's output rules (port)."""
    lib = load("port")
    data = _arr(data, np.float32)
    mask = _arr(mask, np.uint8)
    means = _arr(means, np.float32)
    out_d = data.copy()
    out_m = mask.copy()
    est = np.zeros(len(data), np.float64)
    var = np.zeros(len(data), np.float64)
    st = np.zeros(len(data), np.int32)
    rc = lib.ko_lvm_grid(_ptr(_arr(dims, np.int32), _i), _ptr(data, _f), _ptr(mask, _u8), _ptr(means, _f),
                         int(cov.cov_type), _ptr(_arr(cov.ranges, np.float64), _d),
                         _ptr(_arr(cov.angles, np.float64), _d), float(cov.sill), float(cov.nugget),
                         _ptr(_arr(radiuses, np.int32), _i), int(k), _ptr(out_d, _f), _ptr(out_m, _u8),
                         _ptr(est, _d), _ptr(var, _d), _ptr(st, _i), int(threads))
    if rc:
        raise RuntimeError("lvm_grid failed")
    return out_d, out_m, est, var, st


def sgs(dims, data, mask, cov, radiuses, k, seed, kind=1, sim_mask=None, cdf=None, means=None):
    """Sequential Gaussian simulation (port). `cov` carries the sill and nugget
    the C++ driver receives (geo_bsd's sgs_simulation normalises them by the
    sill first); `cdf` is (values, probs) or None; `means` makes it LVM SGS.
    Returns (data, mask, status) with the status of each simulated node."""
    lib = load("port")
    data = _arr(data, np.float32).copy()
    mask = _arr(mask, np.uint8).copy()
    st = np.zeros(len(data), np.int32)
    sm = _arr(sim_mask, np.uint8) if sim_mask is not None else None
    cv = _arr(cdf[0], np.float32) if cdf is not None else None
    cp = _arr(cdf[1], np.float32) if cdf is not None else None
    mv = _arr(means, np.float32) if means is not None else None
    rc = lib.ko_sgs(_ptr(_arr(dims, np.int32), _i), _ptr(data, _f), _ptr(mask, _u8), _ptr(sm, _u8), _ptr(cv, _f),
                    _ptr(cp, _f), 0 if cv is None else len(cv), _ptr(mv, _f), int(kind), int(cov.cov_type),
                    _ptr(_arr(cov.ranges, np.float64), _d), _ptr(_arr(cov.angles, np.float64), _d),
                    float(cov.sill), float(cov.nugget), _ptr(_arr(radiuses, np.int32), _i), int(k), int(seed),
                    _ptr(st, _i))
    if rc:
        raise RuntimeError(f"sgs failed (rc={rc})")
    return data, mask, st


class _Shape(C.Structure):
    _fields_ = [("data", C.c_int * 3), ("strides", C.c_int * 3)]


class _Cont(C.Structure):
    _fields_ = [("data", _f), ("mask", _u8), ("shape", _Shape)]


class _SgsP(C.Structure):
    _fields_ = [("t", C.c_int), ("r", C.c_double * 3), ("a", C.c_double * 3), ("sill", C.c_double),
                ("nugget", C.c_double), ("rad", C.c_int * 3), ("k", C.c_int), ("kind", C.c_int), ("seed", C.c_long),
                ("kmin", C.c_int)]


def ref_api():
    """The reference library itself (oracle/_ref/libhpgl.so), its output and
    progress handlers silenced."""
    if "api" in _libs:
        return _libs["api"]
    lib = C.CDLL(REF_API_PATH)
    sink = C.CFUNCTYPE(C.c_int, C.c_char_p, C.c_void_p)(lambda s, p: 0)
    psink = C.CFUNCTYPE(C.c_int, C.c_char_p, C.c_int, C.c_void_p)(lambda s, q, p: 0)
    lib.hpgl_set_output_handler(sink, None)
    lib.hpgl_set_progress_handler(psink, None)
    lib._keep = (sink, psink)
    _libs["api"] = lib
    return lib


class _OkP(C.Structure):
    _fields_ = [("t", C.c_int), ("r", C.c_double * 3), ("a", C.c_double * 3), ("sill", C.c_double),
                ("nugget", C.c_double), ("rad", C.c_int * 3), ("k", C.c_int)]


class _SkP(C.Structure):
    _fields_ = _OkP._fields_ + [("auto", C.c_ubyte), ("mean", C.c_double)]


def ref_cont_api(kind, dims, data, mask, cov, radiuses, k, mean=None, threads=0):
    """The reference library's public kriging entry points on copies of
    data/mask: hpgl_ordinary_kriging (kind 0, api.cpp:253-293) or
    hpgl_simple_kriging (kind 1, automatic mean when `mean` is None,
    api.cpp:323-354), the whole call as geo.ordinary_kriging / simple_kriging
    make it (neighbour lookup construction, per-node kriging under OpenMP).
    `threads` > 0 sets the reference's thread count first (hpgl_set_thread_num).
    Returns (out_data, out_mask)."""
    lib = ref_api()
    if threads > 0:
        lib.hpgl_set_thread_num(int(threads))
    data = _arr(data, np.float32)
    mask = _arr(mask, np.uint8)
    od, om = data.copy(), mask.copy()
    sh = _Shape((C.c_int * 3)(*dims), (C.c_int * 3)(1, dims[0], dims[0] * dims[1]))
    base = (int(cov.cov_type), (C.c_double * 3)(*cov.ranges), (C.c_double * 3)(*cov.angles), float(cov.sill),
            float(cov.nugget), (C.c_int * 3)(*[int(r) for r in radiuses]), int(k))
    if kind == 0:
        a = _Cont(data.ctypes.data_as(_f), mask.ctypes.data_as(_u8), sh)
        b = _Cont(od.ctypes.data_as(_f), om.ctypes.data_as(_u8), sh)
        lib.hpgl_ordinary_kriging(C.byref(a), C.byref(_OkP(*base)), C.byref(b))
    else:
        p = _SkP(*base, 1 if mean is None else 0, 0.0 if mean is None else float(mean))
        lib.hpgl_simple_kriging(data.ctypes.data_as(_f), mask.ctypes.data_as(_u8), C.byref(sh), C.byref(p),
                                od.ctypes.data_as(_f), om.ctypes.data_as(_u8), C.byref(sh))
    return od, om


def ref_sgs(dims, data, mask, cov, radiuses, k, seed, kind=1):
    """The reference's hpgl_sgs_simulation on copies of data/mask (no CDF, no
    simulation mask); `cov` holds the sill and nugget the driver receives."""
    lib = ref_api()
    od = _arr(data, np.float32).copy()
    om = _arr(mask, np.uint8).copy()
    sh = _Shape((C.c_int * 3)(*dims), (C.c_int * 3)(1, dims[0], dims[0] * dims[1]))
    a = _Cont(od.ctypes.data_as(_f), om.ctypes.data_as(_u8), sh)
    p = _SgsP(int(cov.cov_type), (C.c_double * 3)(*cov.ranges), (C.c_double * 3)(*cov.angles), float(cov.sill),
              float(cov.nugget), (C.c_int * 3)(*radiuses), int(k), int(kind), int(seed), 0)
    lib.hpgl_sgs_simulation(C.byref(a), C.byref(p), None, None, None)
    return od, om


def cokriging(mark, dims, pdata, pmask, sdata, smask, cov, radiuses, k, primary_mean, secondary_mean,
              secondary_variance=0.0, corr=0.0, cov2=None, threads=0):
    """Collocated cokriging, Markov model I or II (port). Returns (data, mask, status)."""
    lib = load("port")
    n = int(np.prod(dims))
    od = np.zeros(n, np.float32)
    om = np.zeros(n, np.uint8)
    st = np.zeros(n, np.int32)
    c2 = cov2 if cov2 is not None else cov
    rc = lib.ko_cokriging(int(mark), _ptr(_arr(dims, np.int32), _i), _ptr(_arr(pdata, np.float32), _f),
                          _ptr(_arr(pmask, np.uint8), _u8), _ptr(_arr(sdata, np.float32), _f),
                          _ptr(_arr(smask, np.uint8), _u8), int(cov.cov_type), _ptr(_arr(cov.ranges, np.float64), _d),
                          _ptr(_arr(cov.angles, np.float64), _d), float(cov.sill), float(cov.nugget),
                          int(c2.cov_type), _ptr(_arr(c2.ranges, np.float64), _d),
                          _ptr(_arr(c2.angles, np.float64), _d), float(c2.sill), float(c2.nugget),
                          _ptr(_arr(radiuses, np.int32), _i), int(k), float(primary_mean), float(secondary_mean),
                          float(secondary_variance), float(corr), _ptr(od, _f), _ptr(om, _u8), _ptr(st, _i),
                          int(threads))
    if rc:
        raise RuntimeError(f"cokriging failed (rc={rc})")
    return od, om, st


class _Ind(C.Structure):
    _fields_ = [("data", _u8), ("mask", _u8), ("shape", _Shape), ("indicator_count", C.c_int)]


class _IkP(C.Structure):
    _fields_ = [("t", C.c_int), ("r", C.c_double * 3), ("a", C.c_double * 3), ("sill", C.c_double),
                ("nugget", C.c_double), ("rad", C.c_int * 3), ("k", C.c_int), ("marginal", C.c_double)]


def ref_sis(dims, data, mask, covs, radiuses, ks, marginals, seed):
    """The reference's hpgl_sis_simulation on copies of data/mask (no
    simulation mask); returns the simulated categories and mask."""
    lib = ref_api()
    od = _arr(data, np.uint8).copy()
    om = _arr(mask, np.uint8).copy()
    sh = _Shape((C.c_int * 3)(*dims), (C.c_int * 3)(1, dims[0], dims[0] * dims[1]))
    m = len(covs)
    a = _Ind(od.ctypes.data_as(_u8), om.ctypes.data_as(_u8), sh, m)
    p = (_IkP * m)(*[_IkP(int(c.cov_type), (C.c_double * 3)(*c.ranges), (C.c_double * 3)(*c.angles),
                          float(c.sill), float(c.nugget), (C.c_int * 3)(*radiuses[i]), int(ks[i]),
                          float(marginals[i])) for i, c in enumerate(covs)])
    lib.hpgl_sis_simulation(C.byref(a), p, m, int(seed), None)
    return od, om


class _CovP(C.Structure):
    _fields_ = [("t", C.c_int), ("r", C.c_double * 3), ("a", C.c_double * 3), ("sill", C.c_double),
                ("nugget", C.c_double)]


class _Cok1P(C.Structure):
    _fields_ = [("t", C.c_int), ("r", C.c_double * 3), ("a", C.c_double * 3), ("sill", C.c_double),
                ("nugget", C.c_double), ("rad", C.c_int * 3), ("k", C.c_int), ("pm", C.c_double), ("sm", C.c_double),
                ("sv", C.c_double), ("corr", C.c_double)]


def ref_cokriging_mark1(dims, pdata, pmask, sdata, smask, cov, radiuses, k, pm, sm, sv, corr):
    """The reference's hpgl_simple_cokriging_mark1; returns (data, mask)."""
    lib = ref_api()
    pd = _arr(pdata, np.float32)
    pmk = _arr(pmask, np.uint8)
    sd = _arr(sdata, np.float32)
    smk = _arr(smask, np.uint8)
    od = np.zeros_like(pd)
    om = np.zeros_like(pmk)
    sh = _Shape((C.c_int * 3)(*dims), (C.c_int * 3)(1, dims[0], dims[0] * dims[1]))
    a = _Cont(pd.ctypes.data_as(_f), pmk.ctypes.data_as(_u8), sh)
    b = _Cont(sd.ctypes.data_as(_f), smk.ctypes.data_as(_u8), sh)
    o = _Cont(od.ctypes.data_as(_f), om.ctypes.data_as(_u8), sh)
    p = _Cok1P(int(cov.cov_type), (C.c_double * 3)(*cov.ranges), (C.c_double * 3)(*cov.angles), float(cov.sill),
               float(cov.nugget), (C.c_int * 3)(*radiuses), int(k), float(pm), float(sm), float(sv), float(corr))
    lib.hpgl_simple_cokriging_mark1(C.byref(a), C.byref(b), C.byref(p), C.byref(o))
    return od, om


def sis(dims, data, mask, covs, radiuses, ks, marginals, seed, sim_mask=None, means=None, correlogram=False):
    """Sequential indicator simulation (port): covs / radiuses / ks / marginals per
    category; means (LVM) a list of per-cell float arrays, with `correlogram` the
    correlogram weights. Returns (data, mask, status)."""
    lib = load("port")
    ncat = len(covs)
    data = _arr(data, np.uint8).copy()
    mask = _arr(mask, np.uint8).copy()
    st = np.zeros(len(data), np.int32)
    ct = _arr([c.cov_type for c in covs], np.int32)
    rg = _arr([r for c in covs for r in c.ranges], np.float64)
    an = _arr([a for c in covs for a in c.angles], np.float64)
    si = _arr([c.sill for c in covs], np.float64)
    nu = _arr([c.nugget for c in covs], np.float64)
    rd = _arr([r for rr in radiuses for r in rr], np.int32)
    kk = _arr(ks, np.int32)
    mg = _arr(marginals, np.float64)
    sm = _arr(sim_mask, np.uint8) if sim_mask is not None else None
    mp = None
    keep = []
    if means is not None:
        keep = [_arr(m, np.float32) for m in means]
        mp = (_f * ncat)(*[k.ctypes.data_as(_f) for k in keep])
    rc = lib.ko_sis(_ptr(_arr(dims, np.int32), _i), _ptr(data, _u8), _ptr(mask, _u8), _ptr(sm, _u8), ncat,
                    _ptr(ct, _i), _ptr(rg, _d), _ptr(an, _d), _ptr(si, _d), _ptr(nu, _d), _ptr(rd, _i),
                    _ptr(kk, _i), _ptr(mg, _d), mp, int(seed), _ptr(st, _i),
                    int(bool(correlogram)))
    if rc:
        raise RuntimeError(f"sis failed (rc={rc})")
    return data, mask, st


def mt_draws(seed, n):
    """std::mt19937 + uniform_real_distribution<double>(0, 1) draws (the standard library)."""
    lib = load("port")
    out = np.zeros(n, np.float64)
    lib.ko_mt_draws(int(seed), int(n), _ptr(out, _d))
    return out


def sgs_path(size, seed, count=None):
    lib = load("port")
    count = size if count is None else count
    out = np.zeros(count, np.int32)
    if lib.ko_sgs_path(int(size), int(seed), _ptr(out, _i), int(count)):
        raise RuntimeError("sgs_path failed")
    return out


def indicator_grid(dims, data, mask, covs, radiuses, ks, marginals, threads=0):
    lib = load("port")
    n_cat = len(covs)
    data = _arr(data, np.uint8)
    mask = _arr(mask, np.uint8)
    out_d = data.copy()
    out_m = mask.copy()
    probs = np.zeros((len(data), n_cat), np.float32)
    rc = lib.ko_indicator_grid(
        _ptr(_arr(dims, np.int32), _i), _ptr(data, _u8), _ptr(mask, _u8), n_cat,
        _ptr(_arr([c.cov_type for c in covs], np.int32), _i),
        _ptr(_arr([c.ranges for c in covs], np.float64), _d),
        _ptr(_arr([c.angles for c in covs], np.float64), _d),
        _ptr(_arr([c.sill for c in covs], np.float64), _d),
        _ptr(_arr([c.nugget for c in covs], np.float64), _d),
        _ptr(_arr(radiuses, np.int32), _i), _ptr(_arr(ks, np.int32), _i),
        _ptr(_arr(marginals, np.float64), _d), _ptr(out_d, _u8), _ptr(out_m, _u8),
        _ptr(probs, _f), int(threads))
    if rc:
        raise RuntimeError("indicator_grid failed")
    return out_d, out_m, probs


def median_ik_grid(dims, data, mask, cov, radiuses, k, marginal_probs, threads=0):
    lib = load("port")
    data = _arr(data, np.uint8)
    mask = _arr(mask, np.uint8)
    out_d = data.copy()
    out_m = mask.copy()
    prob = np.zeros(len(data), np.float64)
    st = np.zeros(len(data), np.int32)
    rc = lib.ko_median_ik_grid(
        _ptr(_arr(dims, np.int32), _i), _ptr(data, _u8), _ptr(mask, _u8), int(cov.cov_type),
        _ptr(_arr(cov.ranges, np.float64), _d), _ptr(_arr(cov.angles, np.float64), _d),
        float(cov.sill), float(cov.nugget), _ptr(_arr(radiuses, np.int32), _i), int(k),
        _ptr(_arr(marginal_probs, np.float64), _d), _ptr(out_d, _u8), _ptr(out_m, _u8),
        _ptr(prob, _d), _ptr(st, _i), int(threads))
    if rc:
        raise RuntimeError("median_ik_grid failed")
    return out_d, out_m, prob, st


def sort_check(keys):
    lib = load("port")
    keys = _arr(keys, np.uint32)
    a = np.zeros(len(keys), np.int32)
    b = np.zeros(len(keys), np.int32)
    lib.ko_sort_check(_ptr(keys, _u32), len(keys), _ptr(a, _i), _ptr(b, _i))
    return a, b


def select_check(keys, k):
    lib = load("port")
    keys = _arr(keys, np.uint32)
    out = C.c_int(0)
    lib.ko_select_check(_ptr(keys, _u32), len(keys), int(k), C.byref(out))
    return bool(out.value)
