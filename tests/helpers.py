"""Shared helpers: run the engine through its C ABI and the oracle on one workload."""
import ctypes as C

import numpy as np

from geo_bsd import hpgl_wrap as W


def sk_params(cov, radiuses, k, mean=None):
    return W._HPGL_SK_PARAMS(covariance_type=cov.cov_type, ranges=tuple(cov.ranges), angles=tuple(cov.angles),
                             sill=cov.sill, nugget=cov.nugget, radiuses=tuple(int(r) for r in radiuses),
                             max_neighbours=int(k), automatic_mean=1 if mean is None else 0,
                             mean=0.0 if mean is None else float(mean))


def engine_cont(kind, wl, precision=0, refine_steps=2, mean=None, cov=None, radiuses=None, k=None, flags=0):
    """Whole-grid OK (kind 0) / SK (kind 1) through hpgl_b200_cont_kriging_ex with host buffers."""
    cov = cov or wl.cov
    radiuses = radiuses or wl.radiuses
    k = k or wl.max_neighbours
    n = wl.n_cells
    dims = (C.c_int * 3)(*wl.dims)
    data = np.ascontiguousarray(wl.data, np.float32)
    mask = np.ascontiguousarray(wl.mask, np.uint8)
    out_d = data.copy()
    out_m = mask.copy()
    est = np.full(n, np.nan)
    var = np.full(n, np.nan)
    st = np.zeros(n, np.int8)
    opt = W._HPGL_B200_OPTIONS(precision=precision, refine_steps=refine_steps, flags=W.FLAG_OUT_IS_CLONE | flags,
                               stream=None, estimate64=est.ctypes.data, variance=var.ctypes.data,
                               status=st.ctypes.data, ik_probs=None)
    p = sk_params(cov, radiuses, k, mean)
    rc = W._hpgl_so.hpgl_b200_cont_kriging_ex(kind, dims, data.ctypes.data, mask.ctypes.data, C.byref(p),
                                              out_d.ctypes.data, out_m.ctypes.data, C.byref(opt))
    W.check(rc, "cont_kriging_ex")
    return {"data": out_d, "mask": out_m, "est": est, "var": var, "status": st, "stats": W.last_stats()}


def ok_params(cov, radiuses, k):
    return W._HPGL_OK_PARAMS(covariance_type=cov.cov_type, ranges=tuple(cov.ranges), angles=tuple(cov.angles),
                             sill=cov.sill, nugget=cov.nugget, radiuses=tuple(int(r) for r in radiuses),
                             max_neighbours=int(k))


def engine_lvm(wl, means, precision=0, refine_steps=2, flags=0):
    """Whole-grid LVM kriging through hpgl_b200_lvm_kriging_ex with host buffers."""
    n = wl.n_cells
    dims = (C.c_int * 3)(*wl.dims)
    data = np.ascontiguousarray(wl.data, np.float32)
    mask = np.ascontiguousarray(wl.mask, np.uint8)
    means = np.ascontiguousarray(means, np.float32)
    out_d = data.copy()
    out_m = mask.copy()
    est = np.full(n, np.nan)
    var = np.full(n, np.nan)
    st = np.zeros(n, np.int8)
    opt = W._HPGL_B200_OPTIONS(precision=precision, refine_steps=refine_steps, flags=W.FLAG_OUT_IS_CLONE | flags,
                               stream=None, estimate64=est.ctypes.data, variance=var.ctypes.data,
                               status=st.ctypes.data, ik_probs=None)
    p = ok_params(wl.cov, wl.radiuses, wl.max_neighbours)
    rc = W._hpgl_so.hpgl_b200_lvm_kriging_ex(dims, data.ctypes.data, mask.ctypes.data, means.ctypes.data, C.byref(p),
                                             out_d.ctypes.data, out_m.ctypes.data, C.byref(opt))
    W.check(rc, "lvm_kriging_ex")
    return {"data": out_d, "mask": out_m, "est": est, "var": var, "status": st, "stats": W.last_stats()}


def sgs_params(cov, radiuses, k, kind, seed):
    return W._HPGL_SGS_PARAMS(covariance_type=cov.cov_type, ranges=tuple(cov.ranges), angles=tuple(cov.angles),
                              sill=cov.sill, nugget=cov.nugget, radiuses=tuple(int(r) for r in radiuses),
                              max_neighbours=int(k), kriging_kind=int(kind), seed=int(seed), min_neighbours=0)


def engine_sgs(dims, data, mask, cov, radiuses, k, seed, kind=1, sim_mask=None, cdf=None, means=None):
    """SGS through hpgl_b200_sgs_ex with host buffers; returns data, mask, status, stats."""
    n = int(np.prod(dims))
    d = np.ascontiguousarray(data, np.float32).copy()
    m = np.ascontiguousarray(mask, np.uint8).copy()
    st = np.zeros(n, np.int8)
    keep = []
    c = None
    if cdf is not None:
        cv = np.ascontiguousarray(cdf[0], np.float32)
        cp = np.ascontiguousarray(cdf[1], np.float32)
        keep += [cv, cp]
        c = W._HPGL_NON_PARAMETRIC_CDF(values=cv.ctypes.data_as(C.POINTER(C.c_float)),
                                       probs=cp.ctypes.data_as(C.POINTER(C.c_float)), size=len(cv))
    sm = np.ascontiguousarray(sim_mask, np.uint8) if sim_mask is not None else None
    mv = np.ascontiguousarray(means, np.float32) if means is not None else None
    opt = W._HPGL_B200_OPTIONS(precision=0, refine_steps=0, flags=0, stream=None, estimate64=None, variance=None,
                               status=st.ctypes.data, ik_probs=None)
    p = sgs_params(cov, radiuses, k, kind, seed)
    rc = W._hpgl_so.hpgl_b200_sgs_ex((C.c_int * 3)(*dims), d.ctypes.data, m.ctypes.data,
                                     sm.ctypes.data if sm is not None else None, C.byref(c) if c is not None else None,
                                     mv.ctypes.data if mv is not None else None, C.byref(p), C.byref(opt))
    W.check(rc, "sgs_ex")
    return {"data": d, "mask": m, "status": st, "stats": W.last_stats()}


def engine_neighbours(kind, wl, nodes, cov=None, radiuses=None, k=None, mask=None):
    cov = cov or wl.cov
    radiuses = radiuses or wl.radiuses
    k = k or wl.max_neighbours
    dims = (C.c_int * 3)(*wl.dims)
    mask = np.ascontiguousarray(wl.mask if mask is None else mask, np.uint8)
    nodes = np.ascontiguousarray(nodes, np.int32)
    idx = np.full((len(nodes), k), -1, np.int32)
    cnt = np.zeros(len(nodes), np.int32)
    path = np.zeros(len(nodes), np.uint8)
    p = sk_params(cov, radiuses, k)
    rc = W._hpgl_so.hpgl_b200_find_neighbours(kind, dims, mask.ctypes.data, C.byref(p), nodes.ctypes.data,
                                              len(nodes), idx.ctypes.data, cnt.ctypes.data, path.ctypes.data)
    W.check(rc, "find_neighbours")
    return idx, cnt, path


def ik_params(covs, radiuses, ks, marginals):
    m = len(covs)
    arr = (W._HPGL_IK_PARAMS * m)()
    for i in range(m):
        c = covs[i]
        arr[i] = W._HPGL_IK_PARAMS(covariance_type=c.cov_type, ranges=tuple(c.ranges), angles=tuple(c.angles),
                                   sill=c.sill, nugget=c.nugget, radiuses=tuple(int(r) for r in radiuses[i]),
                                   max_neighbours=int(ks[i]), marginal_prob=float(marginals[i]))
    return arr


def engine_indicator(wl, covs, radiuses, ks, marginals, precision=0):
    n = wl.n_cells
    m = len(covs)
    dims = (C.c_int * 3)(*wl.dims)
    data = np.ascontiguousarray(wl.data, np.uint8)
    mask = np.ascontiguousarray(wl.mask, np.uint8)
    out_d = data.copy()
    out_m = mask.copy()
    probs = np.zeros((n, m), np.float32)
    opt = W._HPGL_B200_OPTIONS(precision=precision, refine_steps=2, flags=W.FLAG_OUT_IS_CLONE, stream=None,
                               estimate64=None, variance=None, status=None, ik_probs=probs.ctypes.data)
    arr = ik_params(covs, radiuses, ks, marginals)
    rc = W._hpgl_so.hpgl_b200_indicator_kriging_ex(dims, data.ctypes.data, mask.ctypes.data, arr, m,
                                                   out_d.ctypes.data, out_m.ctypes.data, C.byref(opt))
    W.check(rc, "indicator_kriging_ex")
    return out_d, out_m, probs


def engine_median_ik(wl, cov, radiuses, k, marginal_probs, precision=0):
    n = wl.n_cells
    dims = (C.c_int * 3)(*wl.dims)
    data = np.ascontiguousarray(wl.data, np.uint8)
    mask = np.ascontiguousarray(wl.mask, np.uint8)
    out_d = data.copy()
    out_m = mask.copy()
    prob = np.zeros(n, np.float32)
    opt = W._HPGL_B200_OPTIONS(precision=precision, refine_steps=2, flags=W.FLAG_OUT_IS_CLONE, stream=None,
                               estimate64=None, variance=None, status=None, ik_probs=prob.ctypes.data)
    p = W._HPGL_MEDIAN_IK_PARAMS(covariance_type=cov.cov_type, ranges=tuple(cov.ranges), angles=tuple(cov.angles),
                                 sill=cov.sill, nugget=cov.nugget, radiuses=tuple(int(r) for r in radiuses),
                                 max_neighbours=int(k), marginal_probs=tuple(marginal_probs))
    rc = W._hpgl_so.hpgl_b200_median_ik_ex(dims, data.ctypes.data, mask.ctypes.data, C.byref(p),
                                           out_d.ctypes.data, out_m.ctypes.data, C.byref(opt))
    W.check(rc, "median_ik_ex")
    return out_d, out_m, prob


def rel_err(a, ref):
    """Normwise relative error max|a - ref| / max|ref| over the compared cells."""
    a = np.asarray(a, np.float64)
    ref = np.asarray(ref, np.float64)
    if a.size == 0:
        return 0.0
    return float(np.max(np.abs(a - ref)) / max(np.max(np.abs(ref)), 1e-300))


def engine_sis(dims, data, mask, covs, radiuses, ks, marginals, seed, sim_mask=None, means=None, corr=False):
    """SIS through hpgl_b200_sis_ex with host buffers; returns data, mask, status, stats."""
    n = int(np.prod(dims))
    d = np.ascontiguousarray(data, np.uint8).copy()
    m = np.ascontiguousarray(mask, np.uint8).copy()
    st = np.zeros(n, np.int8)
    sm = np.ascontiguousarray(sim_mask, np.uint8) if sim_mask is not None else None
    keep = []
    mp = None
    if means is not None:
        keep = [np.ascontiguousarray(v, np.float32) for v in means]
        mp = (C.c_void_p * len(keep))(*[v.ctypes.data for v in keep])
    opt = W._HPGL_B200_OPTIONS(precision=0, refine_steps=0, flags=0, stream=None, estimate64=None, variance=None,
                               status=st.ctypes.data, ik_probs=None)
    arr = ik_params(covs, radiuses, ks, marginals)
    rc = W._hpgl_so.hpgl_b200_sis_ex((C.c_int * 3)(*dims), d.ctypes.data, m.ctypes.data,
                                     sm.ctypes.data if sm is not None else None, arr, len(covs),
                                     C.cast(mp, C.c_void_p) if mp is not None else None, int(seed), int(bool(corr)),
                                     C.byref(opt))
    W.check(rc, "sis_ex")
    return {"data": d, "mask": m, "status": st, "stats": W.last_stats()}
