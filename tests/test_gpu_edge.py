"""GPU edge cases and the Python API: empty and tiny inputs, path selection
extremes, device-pointer mode on a caller's stream, determinism, and the
full-size benchmark grid's size-independent properties."""
import ctypes as C

import numpy as np
import pytest

import helpers as H
import oracle as O
import geo_bsd
from geo_bsd import hpgl_wrap as W
from geo_bsd import workloads as WL

pytestmark = pytest.mark.gpu


def _wl(dims, informed, values, cov, rad, k):
    n = dims[0] * dims[1] * dims[2]
    data = np.full(n, -99.0, np.float32)
    mask = np.zeros(n, np.uint8)
    data[informed] = values
    mask[informed] = 1
    return WL.Workload("edge", dims, data, mask, cov, rad, k)


SPH = WL.CovSpec(WL.SPHERICAL, (6.0, 6.0, 3.0), (0.0, 0.0, 0.0), 1.0, 0.1)
EXP = WL.CovSpec(WL.EXPONENTIAL, (8.0, 4.0, 3.0), (30.0, 0.0, 0.0), 1.0, 0.05)


def _check_against_oracle(wl, kind, tol=1e-10):
    od, om, oest, ovar, ost = O.cont_grid(kind, wl.dims, wl.data, wl.mask, wl.cov, wl.radiuses, wl.max_neighbours)
    e = H.engine_cont(kind, wl, precision=0)
    unk = wl.mask == 0
    np.testing.assert_array_equal(e["status"][unk], ost[unk].astype(np.int8))
    np.testing.assert_array_equal(e["mask"], om)
    ok = unk & (ost == 0)
    if ok.any():
        assert H.rel_err(e["est"][ok], oest[ok]) <= tol
    fail = unk & (ost != 0)
    if kind == 0:
        np.testing.assert_array_equal(e["data"][fail], wl.data[fail])  # left as the input clone
    return e


@pytest.mark.parametrize("kind", [0, 1])
def test_no_conditioning_data(kind):
    wl = _wl((12, 9, 5), np.array([], np.int64), np.array([], np.float32), SPH, (3, 3, 2), 8)
    e = _check_against_oracle(wl, kind)
    assert np.all(e["status"] == 1)


@pytest.mark.parametrize("kind", [0, 1])
def test_single_point_and_k1(kind):
    wl = _wl((15, 11, 6), np.array([300]), np.array([2.5], np.float32), SPH, (4, 4, 2), 1)
    _check_against_oracle(wl, kind)


@pytest.mark.parametrize("kind", [0, 1])
def test_all_cells_informed(kind):
    n = 6 * 5 * 4
    wl = _wl((6, 5, 4), np.arange(n), np.arange(n, dtype=np.float32), SPH, (2, 2, 2), 4)
    e = H.engine_cont(kind, wl)
    np.testing.assert_array_equal(e["data"], wl.data)
    assert np.all(e["mask"] == 1)


@pytest.mark.parametrize("kind", [0, 1])
def test_radius_larger_than_grid_and_template_everywhere(kind):
    rng = np.random.default_rng(2)
    dims = (20, 14, 7)
    idx = rng.choice(20 * 14 * 7, 300, replace=False)  # dense: every bin overflows -> template path
    wl = _wl(dims, idx, rng.standard_normal(300).astype(np.float32), EXP, (25, 25, 9), 10)
    _check_against_oracle(wl, kind)


@pytest.mark.parametrize("kind", [0, 1])
def test_k_above_candidates_and_large_k(kind):
    rng = np.random.default_rng(3)
    dims = (30, 30, 8)
    idx = rng.choice(30 * 30 * 8, 90, replace=False)
    wl = _wl(dims, idx, rng.standard_normal(90).astype(np.float32), EXP, (8, 6, 3), 80)  # > 64: large-n kernel
    _check_against_oracle(wl, kind, tol=1e-9)


def test_ties_and_duplicated_geometry():
    """A lattice of equally spaced points makes many equal keys: tie groups straddle the k-th slot."""
    dims = (24, 24, 4)
    # spacing 6 keeps every bin under the clusterizer limit, so cells take the bin path
    xs, ys, zs = np.meshgrid(np.arange(0, 24, 6), np.arange(0, 24, 6), np.arange(0, 4, 2), indexing="ij")
    idx = (xs + 24 * ys + 576 * zs).ravel()
    wl = _wl(dims, idx, np.sin(idx).astype(np.float32), WL.CovSpec(WL.EXPONENTIAL, (9.0, 9.0, 9.0), (0, 0, 0), 1.0,
                                                                   0.0), (9, 9, 3), 7)
    for kind in (0, 1):
        e = _check_against_oracle(wl, kind)
        assert e["stats"]["tie_cells"] > 0
        nodes = np.flatnonzero(wl.mask == 0)
        idx_e, cnt, _ = H.engine_neighbours(kind, wl, nodes)
        r = O.krige_nodes("port", kind, wl.dims, wl.data, wl.mask, wl.cov, wl.radiuses, wl.max_neighbours,
                          nodes=nodes)
        np.testing.assert_array_equal(cnt, r["count"])
        assert all(set(a[a >= 0]) == set(b[b >= 0]) for a, b in zip(idx_e, r["idx"]))


def test_python_api_shapes_and_variance():
    wl = WL.ok_small(0.3)
    grid = geo_bsd.SugarboxGrid(*wl.dims)
    prop = geo_bsd.ContProperty(wl.data.reshape(wl.dims, order="F"), wl.mask.reshape(wl.dims, order="F"))
    cm = geo_bsd.CovarianceModel(type=wl.cov.cov_type, ranges=wl.cov.ranges, angles=wl.cov.angles, sill=wl.cov.sill,
                                 nugget=wl.cov.nugget)
    out, var = geo_bsd.ordinary_kriging(prop, grid, wl.radiuses, wl.max_neighbours, cm, return_variance=True)
    assert out.data.shape == wl.dims and out.data.flags["F"]
    assert var.shape == wl.dims
    e = H.engine_cont(0, wl)
    np.testing.assert_array_equal(out.data.reshape(-1, order="F"), e["data"])
    out32 = geo_bsd.ordinary_kriging(prop, grid, wl.radiuses, wl.max_neighbours, cm, precision="fp32_refined")
    assert np.abs(out32.data - out.data).max() <= 1e-5
    sk = geo_bsd.simple_kriging((prop.data, prop.mask), grid, wl.radiuses, wl.max_neighbours, cm, mean=0.5)
    assert sk.mask.all() or sk.mask.sum() >= out.mask.sum()
    w = geo_bsd.simple_kriging_weights((1, 1, 1), [0, 2], [0, 2], [0, 2], ranges=(5, 5, 5))
    assert w.shape == (2,) and np.isfinite(w).all()


def test_two_category_indicator_dispatches_to_median_ik():
    wl = WL.indicator(0.12)
    data = (wl.data >= 2).astype(np.uint8)
    grid = geo_bsd.SugarboxGrid(*wl.dims)
    prop = geo_bsd.IndProperty(data, wl.mask, 2)
    c = wl.cat_covs[2]
    cm = geo_bsd.CovarianceModel(type=c.cov_type, ranges=c.ranges, angles=c.angles, sill=c.sill, nugget=c.nugget)
    spec = [{"cov_model": cm, "radiuses": wl.cat_radiuses[2], "max_neighbours": 24} for _ in range(2)]
    out = geo_bsd.indicator_kriging(prop, grid, spec, [0.7, 0.3])
    od, om, prob, st = O.median_ik_grid(wl.dims, data, wl.mask, c, wl.cat_radiuses[2], 24, (0.7, 0.3))
    np.testing.assert_array_equal(out.data.reshape(-1)[st == 0], od[st == 0])


def test_device_pointers_on_a_caller_stream_and_determinism():
    import torch
    wl = WL.sk_ok_large(0.25)
    dev = torch.device("cuda", 0)
    d = torch.from_numpy(wl.data).to(dev)
    m = torch.from_numpy(wl.mask).to(dev)
    s = torch.cuda.Stream()
    outs = []
    for _ in range(2):
        od, om = d.clone(), m.clone()
        est = torch.full((wl.n_cells,), float("nan"), dtype=torch.float64, device=dev)
        o = W._HPGL_B200_OPTIONS(precision=1, refine_steps=3, flags=W.FLAG_DEVICE_POINTERS | W.FLAG_OUT_IS_CLONE,
                                 stream=s.cuda_stream, estimate64=est.data_ptr(), variance=None, status=None,
                                 ik_probs=None)
        p = H.sk_params(wl.cov, wl.radiuses, wl.max_neighbours)
        rc = W._hpgl_so.hpgl_b200_cont_kriging_ex(0, (C.c_int * 3)(*wl.dims), d.data_ptr(), m.data_ptr(),
                                                  C.byref(p), od.data_ptr(), om.data_ptr(), C.byref(o))
        W.check(rc, "device call")
        s.synchronize()
        outs.append((od.cpu().numpy(), est.cpu().numpy()))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    host = H.engine_cont(0, wl, precision=1, refine_steps=3)
    np.testing.assert_array_equal(outs[0][0], host["data"])


def test_pageable_pinned_and_device_buffers_agree():
    """Inputs and outputs above the staging threshold (4 MB) in pageable numpy
    arrays (copied through page-locked areas by host threads), in page-locked
    buffers from hpgl_b200_host_alloc (copied directly) and on the device give
    bit-identical outputs; a second pageable call into fresh arrays too."""
    import torch
    wl = WL.sk_ok_large(0.55)
    n = wl.n_cells
    assert n * 4 >= 4 << 20
    a = H.engine_cont(0, wl, precision=1)
    b = H.engine_cont(0, wl, precision=1)
    np.testing.assert_array_equal(a["data"], b["data"])
    np.testing.assert_array_equal(a["var"], b["var"])
    lib = W._hpgl_so
    sizes = (n * 4, n, n * 4, n, n * 8)
    ptrs = [lib.hpgl_b200_host_alloc(sz) for sz in sizes]
    try:
        hd, hm, ho, hom, hv = ptrs
        C.memmove(hd, np.ascontiguousarray(wl.data, np.float32).ctypes.data, n * 4)
        C.memmove(hm, np.ascontiguousarray(wl.mask, np.uint8).ctypes.data, n)
        o = W._HPGL_B200_OPTIONS(precision=1, refine_steps=2, flags=W.FLAG_OUT_IS_CLONE, stream=None,
                                 estimate64=None, variance=hv, status=None, ik_probs=None)
        p = H.sk_params(wl.cov, wl.radiuses, wl.max_neighbours)
        rc = lib.hpgl_b200_cont_kriging_ex(0, (C.c_int * 3)(*wl.dims), hd, hm, C.byref(p), ho, hom, C.byref(o))
        W.check(rc, "pinned call")
        out = np.ctypeslib.as_array((C.c_float * n).from_address(ho)).copy()
        omask = np.ctypeslib.as_array((C.c_ubyte * n).from_address(hom)).copy()
        var = np.ctypeslib.as_array((C.c_double * n).from_address(hv)).copy()
    finally:
        for q in ptrs:
            lib.hpgl_b200_host_free(q)
    np.testing.assert_array_equal(out, a["data"])
    np.testing.assert_array_equal(omask, a["mask"])
    np.testing.assert_array_equal(var, a["var"])
    dev = torch.device("cuda", 0)
    d = torch.from_numpy(np.ascontiguousarray(wl.data)).to(dev)
    m = torch.from_numpy(np.ascontiguousarray(wl.mask)).to(dev)
    od, om = d.clone(), m.clone()
    o = W._HPGL_B200_OPTIONS(precision=1, refine_steps=2, flags=W.FLAG_DEVICE_POINTERS | W.FLAG_OUT_IS_CLONE,
                             stream=None, estimate64=None, variance=None, status=None, ik_probs=None)
    rc = lib.hpgl_b200_cont_kriging_ex(0, (C.c_int * 3)(*wl.dims), d.data_ptr(), m.data_ptr(), C.byref(p),
                                       od.data_ptr(), om.data_ptr(), C.byref(o))
    W.check(rc, "device call")
    torch.cuda.synchronize()
    np.testing.assert_array_equal(od.cpu().numpy(), a["data"])


def test_full_size_benchmark_grid_properties():
    """256x256x128 OK, k=32: FP32-refined agrees with FP64 plain to 1e-6, variances are
    non-negative, every uninformed cell is kriged, and repeated runs are bit-identical."""
    wl = WL.sk_ok_large(1.0)
    a = H.engine_cont(0, wl, precision=0)
    b = H.engine_cont(0, wl, precision=1, refine_steps=3)
    c = H.engine_cont(0, wl, precision=1, refine_steps=3)
    unk = wl.mask == 0
    ok = unk & (a["status"] == 0)
    assert ok.sum() >= 0.99 * unk.sum()
    assert H.rel_err(b["est"][ok], a["est"][ok]) <= 1e-6
    assert np.all(a["var"][ok] >= 0) and np.all(b["var"][ok] >= 0)
    np.testing.assert_array_equal(b["data"], c["data"])
    np.testing.assert_array_equal(b["est"], c["est"])
    # at every kriged cell the OK estimate lies within the range of the data
    v = wl.data[wl.mask == 1]
    assert a["data"][ok].min() >= v.min() - 3 * v.std() and a["data"][ok].max() <= v.max() + 3 * v.std()
