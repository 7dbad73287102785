"""LVM kriging (kriging with a locally varying mean) on the GPU.

Bars: the float grid and mask that the reference's hpgl_lvm_kriging writes
reproduced through the engine's entry point of the same signature to float
rounding; FP64-plain estimates and variances within 1e-10 relative of the
oracle's FP64 path and FP32-refined within 1e-6, with per-cell status
identical; failed cells hold their own mean; a constant mean field gives SK
with that mean.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import geo_bsd
import golden_io as G
import helpers as H
import oracle as O
from geo_bsd import hpgl_wrap as W
from geo_bsd import workloads as WL

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_TOL = 1e-6


@pytest.mark.parametrize("case", ["ok_small_s030", "gauss_cv_s020"])
def test_lvm_grid_matches_reference_api(case):
    g = G.load(case)
    lv = G.load("lvm")
    wl = G.as_workload(g, case)
    means = lv[f"{case}_means"]
    data = np.ascontiguousarray(wl.data).reshape(wl.dims, order="F")
    mask = np.ascontiguousarray(wl.mask).reshape(wl.dims, order="F")
    m3 = means.reshape(wl.dims, order="F")
    out_d, out_m = data.copy(order="F"), mask.copy(order="F")
    sh = W._HPGL_SHAPE(data=wl.dims, strides=(1, wl.dims[0], wl.dims[0] * wl.dims[1]))
    p = H.ok_params(wl.cov, wl.radiuses, wl.max_neighbours)
    W._hpgl_so.hpgl_lvm_kriging(data, mask, C.byref(sh), m3, C.byref(sh), C.byref(p), out_d, out_m, C.byref(sh))
    assert W.last_stats()["kriged_cells"] > 0
    np.testing.assert_array_equal(out_m.reshape(-1, order="F"), lv[f"{case}_grid_mask"])
    ref = lv[f"{case}_grid_data"]
    assert np.abs(out_d.reshape(-1, order="F") - ref).max() <= 1e-6 * max(np.abs(ref).max(), 1.0)


@pytest.mark.parametrize("case", ["ok_small_s030", "gauss_cv_s020"])
@pytest.mark.parametrize("precision", [0, 1])
def test_lvm_estimates_match_reference_per_node(case, precision):
    """FP64 estimates and variances of the reference's own LVM instantiation."""
    g = G.load(case)
    lv = G.load("lvm")
    wl = G.as_workload(g, case)
    e = H.engine_lvm(wl, lv[f"{case}_means"], precision=precision)
    nodes = lv[f"{case}_nodes"]
    st = e["status"][nodes]
    np.testing.assert_array_equal(st, lv[f"{case}_status"].astype(np.int8))
    ok = st == 0
    tol = FP64_TOL if precision == 0 else FP32_TOL
    assert H.rel_err(e["est"][nodes][ok], lv[f"{case}_est"][ok]) <= tol
    assert H.rel_err(e["var"][nodes][ok], lv[f"{case}_var"][ok]) <= tol


@pytest.mark.parametrize("name,scale", [("ok_small", 0.6), ("sk_ok_large", 0.3), ("gauss_cv", 0.35),
                                        ("clustered", 0.2)])
def test_lvm_against_oracle(name, scale):
    wl = WL.ALL[name](scale)
    means = WL.lvm_means(wl.dims, seed=11)
    od, om, oest, ovar, ost = O.lvm_grid(wl.dims, wl.data, wl.mask, means, wl.cov, wl.radiuses, wl.max_neighbours)
    unk = wl.mask == 0
    for precision in (0, 1):
        e = H.engine_lvm(wl, means, precision=precision)
        np.testing.assert_array_equal(e["status"][unk], ost[unk].astype(np.int8))
        np.testing.assert_array_equal(e["mask"], om)
        ok = unk & (ost == 0)
        tol = FP64_TOL if precision == 0 else FP32_TOL
        if name == "clustered":
            tol = max(tol, 1e-8)
        assert H.rel_err(e["est"][ok], oest[ok]) <= tol, (precision, H.rel_err(e["est"][ok], oest[ok]))
        assert H.rel_err(e["var"][ok], ovar[ok]) <= tol
        assert np.abs(e["data"][ok] - od[ok]).max() <= 1e-6 * max(np.abs(od[ok]).max(), 1.0)
        failed = unk & (ost != 0)
        np.testing.assert_array_equal(e["data"][failed], means[failed])
        np.testing.assert_array_equal(e["data"][~unk], wl.data[~unk])


def test_lvm_failures_take_the_cell_mean():
    wl = WL.ok_small(0.3)
    means = WL.lvm_means(wl.dims)
    e = H.engine_lvm(wl, means)
    failed = (wl.mask == 0) & (e["status"] != 0)
    assert failed.sum() > 0
    np.testing.assert_array_equal(e["data"][failed], means[failed])
    assert np.all(e["mask"] == 1)


@pytest.mark.parametrize("precision", [0, 1])
def test_constant_mean_field_is_simple_kriging(precision):
    wl = WL.sk_ok_large(0.25)
    mean = np.float32(0.37)
    lvm = H.engine_lvm(wl, np.full(wl.n_cells, mean, np.float32), precision=precision)
    sk = H.engine_cont(1, wl, precision=precision, mean=float(mean))
    np.testing.assert_array_equal(lvm["status"], sk["status"])
    np.testing.assert_array_equal(lvm["est"], sk["est"])
    np.testing.assert_array_equal(lvm["var"], sk["var"])
    np.testing.assert_array_equal(lvm["data"], sk["data"])


def test_lvm_device_pointers_match_host_buffers():
    wl = WL.gauss_cv(0.35)
    means = WL.lvm_means(wl.dims)
    host = H.engine_lvm(wl, means)
    dev = torch.device("cuda")
    d_data = torch.from_numpy(np.ascontiguousarray(wl.data, np.float32)).to(dev)
    d_mask = torch.from_numpy(np.ascontiguousarray(wl.mask, np.uint8)).to(dev)
    d_means = torch.from_numpy(means).to(dev)
    d_out = d_data.clone()
    d_om = d_mask.clone()
    d_est = torch.empty(wl.n_cells, dtype=torch.float64, device=dev)
    opt = W._HPGL_B200_OPTIONS(precision=0, refine_steps=2, flags=W.FLAG_DEVICE_POINTERS | W.FLAG_OUT_IS_CLONE,
                               stream=None, estimate64=d_est.data_ptr(), variance=None, status=None, ik_probs=None)
    p = H.ok_params(wl.cov, wl.radiuses, wl.max_neighbours)
    rc = W._hpgl_so.hpgl_b200_lvm_kriging_ex((C.c_int * 3)(*wl.dims), d_data.data_ptr(), d_mask.data_ptr(),
                                             d_means.data_ptr(), C.byref(p), d_out.data_ptr(), d_om.data_ptr(),
                                             C.byref(opt))
    W.check(rc, "lvm_kriging_ex")
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_out.cpu().numpy(), host["data"])
    np.testing.assert_array_equal(d_om.cpu().numpy(), host["mask"])
    ok = host["status"] == 0
    np.testing.assert_array_equal(d_est.cpu().numpy()[ok], host["est"][ok])


def test_geo_lvm_kriging_api():
    wl = WL.gauss_cv(0.2)
    grid = geo_bsd.SugarboxGrid(*wl.dims)
    prop = geo_bsd.ContProperty(wl.data.reshape(wl.dims, order="F").copy(order="F"),
                                wl.mask.reshape(wl.dims, order="F").copy(order="F"))
    cm = geo_bsd.CovarianceModel(type=wl.cov.cov_type, ranges=wl.cov.ranges, angles=wl.cov.angles, sill=wl.cov.sill,
                                 nugget=wl.cov.nugget)
    means = WL.lvm_means(wl.dims).reshape(wl.dims, order="F")
    out, var = geo_bsd.lvm_kriging(prop, grid, means, wl.radiuses, wl.max_neighbours, cm, return_variance=True)
    od, om, oest, ovar, ost = O.lvm_grid(wl.dims, wl.data, wl.mask, means.reshape(-1, order="F"), wl.cov,
                                         wl.radiuses, wl.max_neighbours)
    flat = out.data.reshape(-1, order="F")
    assert np.abs(flat - od).max() <= 1e-6 * max(np.abs(od).max(), 1.0)
    ok = (wl.mask == 0) & (ost == 0)
    assert H.rel_err(var.reshape(-1, order="F")[ok], ovar[ok]) <= FP64_TOL
    # float64 means are narrowed to float32 as the reference does
    out2 = geo_bsd.lvm_kriging(prop, grid, means.astype(np.float64), wl.radiuses, wl.max_neighbours, cm)
    np.testing.assert_array_equal(out2.data, out.data)
    with pytest.raises(ValueError):
        geo_bsd.lvm_kriging(prop, grid, list(means.reshape(-1)), wl.radiuses, wl.max_neighbours, cm)
    with pytest.raises(C.ArgumentError):  # ndpointer(flags='F') rejects a C-ordered 3-D array
        geo_bsd.lvm_kriging(prop, grid, np.ascontiguousarray(means), wl.radiuses, wl.max_neighbours, cm)
    with pytest.raises(RuntimeError):
        geo_bsd.lvm_kriging(prop, grid, means.reshape(-1, order="F")[:-1], wl.radiuses, wl.max_neighbours, cm)
