"""Simple collocated cokriging (Markov models I and II) on the GPU.

Bars: masks identical to the reference's (golden fixtures) and per-cell status
identical to the oracle's; values bit-identical to the reference's on at least
99% of the cells and within 1e-5 relative everywhere (the weights come from a
Cholesky factorisation and a Schur complement, not the reference's Gaussian
elimination; the float result is the reference's per-term rounding of a
double accumulation); failed cells exactly pm + sv - sm.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import geo_bsd
import golden_io as G
import oracle as O
from geo_bsd import hpgl_wrap as W
from geo_bsd import workloads as WL

pytestmark = pytest.mark.gpu

BIT_FRAC = 0.99
REL_TOL = 1e-5


def _close(got, ref, what):
    same = got.view(np.uint32) == ref.view(np.uint32)
    diff = np.abs(got.astype(np.float64) - ref.astype(np.float64))
    scale = max(1.0, float(np.abs(ref).max()))
    assert same.mean() >= BIT_FRAC, (what, float(same.mean()), float(diff.max()))
    assert diff.max() <= REL_TOL * scale, (what, float(same.mean()), float(diff.max()))


def _params(x, mark):
    c = x["cov"]
    if mark == 1:
        return W._HPGL_COK_M1_PARAMS(covariance_type=c.cov_type, ranges=c.ranges, angles=c.angles, sill=c.sill,
                                     nugget=c.nugget, radiuses=x["rad"], max_neighbours=x["k"], primary_mean=x["pm"],
                                     secondary_mean=x["sm"], secondary_variance=x["sv"], correlation_coef=x["corr"])
    c2 = x["cov2"]
    cp = W._HPGL_COV_PARAMS(covariance_type=c.cov_type, ranges=c.ranges, angles=c.angles, sill=c.sill, nugget=c.nugget)
    cs = W._HPGL_COV_PARAMS(covariance_type=c2.cov_type, ranges=c2.ranges, angles=c2.angles, sill=c2.sill,
                            nugget=c2.nugget)
    return W._HPGL_COK_M2_PARAMS(primary_cov_params=cp, secondary_cov_params=cs, radiuses=x["rad"],
                                 max_neighbours=x["k"], primary_mean=x["pm"], secondary_mean=x["sm"],
                                 correlation_coef=x["corr"])


def _run_ex(x, mark, flags=0, arrays=None):
    n = int(np.prod(x["dims"]))
    out = np.zeros(n, np.float32)
    om = np.zeros(n, np.uint8)
    st = np.zeros(n, np.int8)
    p = _params(x, mark)
    opt = W._HPGL_B200_OPTIONS(precision=0, refine_steps=0, flags=flags, stream=None, estimate64=None,
                               variance=None, status=st.ctypes.data, ik_probs=None)
    pd, pm, sd, sm = (np.ascontiguousarray(x["pdata"], np.float32), np.ascontiguousarray(x["pmask"], np.uint8),
                      np.ascontiguousarray(x["sdata"], np.float32), np.ascontiguousarray(x["smask"], np.uint8))
    rc = W._hpgl_so.hpgl_b200_cokriging_ex(mark, (C.c_int * 3)(*x["dims"]), pd.ctypes.data, pm.ctypes.data,
                                           sd.ctypes.data, sm.ctypes.data, C.byref(p) if mark == 1 else None,
                                           C.byref(p) if mark == 2 else None, out.ctypes.data, om.ctypes.data,
                                           C.byref(opt))
    W.check(rc, "cokriging_ex")
    return out, om, st


def _oracle(x, mark):
    return O.cokriging(mark, x["dims"], x["pdata"], x["pmask"], x["sdata"], x["smask"], x["cov"], x["rad"], x["k"],
                       x["pm"], x["sm"], secondary_variance=x["sv"], corr=x["corr"], cov2=x["cov2"])


@pytest.mark.parametrize("case", [c[0] for c in G.COK_CASES])
def test_cokriging_matches_reference(case):
    """Through the entry points of the reference's signatures."""
    _, base, mark = next(c for c in G.COK_CASES if c[0] == case)
    ref = G.load("cok")
    x = G.cok_inputs(G.load(base), mark, (ref[f"{base}_sdata"], ref[f"{base}_smask"]))
    n = int(np.prod(x["dims"]))
    sh = W._HPGL_SHAPE(data=x["dims"], strides=(1, x["dims"][0], x["dims"][0] * x["dims"][1]))
    fp, up = C.POINTER(C.c_float), C.POINTER(C.c_ubyte)
    pd, pm = x["pdata"].copy(), x["pmask"].copy()
    sd, sm = np.ascontiguousarray(x["sdata"]), np.ascontiguousarray(x["smask"])
    out, om = np.zeros(n, np.float32), np.zeros(n, np.uint8)
    a = W._HPGL_CONT_MASKED_ARRAY(pd.ctypes.data_as(fp), pm.ctypes.data_as(up), sh)
    b = W._HPGL_CONT_MASKED_ARRAY(sd.ctypes.data_as(fp), sm.ctypes.data_as(up), sh)
    o = W._HPGL_CONT_MASKED_ARRAY(out.ctypes.data_as(fp), om.ctypes.data_as(up), sh)
    p = _params(x, mark)
    fn = W._hpgl_so.hpgl_simple_cokriging_mark1 if mark == 1 else W._hpgl_so.hpgl_simple_cokriging_mark2
    fn(C.byref(a), C.byref(b), C.byref(p), C.byref(o))
    assert W.last_stats()["kriged_cells"] > 0
    np.testing.assert_array_equal(om, ref[f"{case}_mask"])
    _close(out, ref[f"{case}_data"], case)


def _scaled(name, scale, mark):
    wl = WL.ALL[name](scale)
    g = {"dims": np.array(wl.dims), "informed": np.flatnonzero(wl.mask == 1), "values": wl.data[wl.mask == 1],
         "cov_type": wl.cov.cov_type, "ranges": np.array(wl.cov.ranges), "angles": np.array(wl.cov.angles),
         "sill": wl.cov.sill, "nugget": wl.cov.nugget, "radiuses": np.array(wl.radiuses), "k": wl.max_neighbours}
    return G.cok_inputs(g, mark)


@pytest.mark.parametrize("name,scale,mark", [("sk_ok_large", 0.3, 1), ("sk_ok_large", 0.3, 2), ("gauss_cv", 0.5, 2),
                                             ("ok_small", 0.6, 1), ("clustered", 0.2, 1)])
def test_cokriging_against_oracle(name, scale, mark):
    """Larger grids (clustered has k = 64: the block-per-target solve)."""
    x = _scaled(name, scale, mark)
    od, om, ost = _oracle(x, mark)
    out, mk, st = _run_ex(x, mark)
    np.testing.assert_array_equal(mk, om)
    np.testing.assert_array_equal(st, ost.astype(np.int8))
    _close(out, od, name)
    failed = st > 0
    sv = np.where(x["smask"] == 1, x["sdata"], np.float32(x["sm"])).astype(np.float32)
    fb = (np.float32(x["pm"]) + sv) - np.float32(x["sm"])
    np.testing.assert_array_equal(out[failed], fb[failed])


@pytest.mark.parametrize("k", [80, 24])
def test_template_scan_and_selection_paths(k):
    """k > 64 takes the template scan over the informed-cell bitmap, k <= 64 the
    binned selection keyed by template position; both give the oracle's cells."""
    x = _scaled("gauss_cv", 0.3, 1)
    x = dict(x, k=k)
    od, om, ost = _oracle(x, 1)
    out, mk, st = _run_ex(x, 1)
    np.testing.assert_array_equal(mk, om)
    np.testing.assert_array_equal(st, ost.astype(np.int8))
    _close(out, od, f"k={k}")


def test_device_pointers_match_host_buffers():
    x = _scaled("gauss_cv", 0.35, 1)
    host, hm, hs = _run_ex(x, 1)
    dev = torch.device("cuda")
    t = {k: torch.from_numpy(np.ascontiguousarray(x[k])).to(dev) for k in ("pdata", "pmask", "sdata", "smask")}
    out = torch.zeros_like(t["pdata"])
    om = torch.zeros_like(t["pmask"])
    p = _params(x, 1)
    opt = W._HPGL_B200_OPTIONS(precision=0, refine_steps=0, flags=W.FLAG_DEVICE_POINTERS, stream=None,
                               estimate64=None, variance=None, status=None, ik_probs=None)
    rc = W._hpgl_so.hpgl_b200_cokriging_ex(1, (C.c_int * 3)(*x["dims"]), t["pdata"].data_ptr(), t["pmask"].data_ptr(),
                                           t["sdata"].data_ptr(), t["smask"].data_ptr(), C.byref(p), None,
                                           out.data_ptr(), om.data_ptr(), C.byref(opt))
    W.check(rc, "cokriging_ex")
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), host)
    np.testing.assert_array_equal(om.cpu().numpy(), hm)


def test_geo_cokriging_api():
    x = _scaled("gauss_cv", 0.3, 2)
    dims = x["dims"]
    grid = geo_bsd.SugarboxGrid(*dims)
    prop = geo_bsd.ContProperty(x["pdata"].reshape(dims, order="F").copy(order="F"),
                                x["pmask"].reshape(dims, order="F").copy(order="F"))
    sec = geo_bsd.ContProperty(x["sdata"].reshape(dims, order="F").copy(order="F"),
                               x["smask"].reshape(dims, order="F").copy(order="F"))
    c = x["cov"]
    cm = geo_bsd.CovarianceModel(type=c.cov_type, ranges=c.ranges, angles=c.angles, sill=c.sill, nugget=c.nugget)
    c2 = x["cov2"]
    cm2 = geo_bsd.CovarianceModel(type=c2.cov_type, ranges=c2.ranges, angles=c2.angles, sill=c2.sill,
                                  nugget=c2.nugget)
    out1 = geo_bsd.simple_cokriging_markI(prop, grid, sec, x["pm"], x["sm"], x["sv"], x["corr"], x["rad"], x["k"], cm)
    od1, _, _ = _oracle(x, 1)
    _close(out1.data.reshape(-1, order="F"), od1, "geo mark I")
    assert np.all(out1.mask == 1)
    out2 = geo_bsd.simple_cokriging_markII(grid, {"data": prop, "mean": x["pm"], "cov_model": cm},
                                           {"data": sec, "mean": x["sm"], "cov_model": cm2}, x["corr"], x["rad"],
                                           x["k"])
    od2, _, _ = _oracle(x, 2)
    _close(out2.data.reshape(-1, order="F"), od2, "geo mark II")
    with pytest.raises(geo_bsd.CriticalValidationError):
        geo_bsd.simple_cokriging_markI(prop, grid, sec, x["pm"], x["sm"], x["sv"], 1.5, x["rad"], x["k"], cm)
    with pytest.raises(geo_bsd.CriticalValidationError):
        geo_bsd.simple_cokriging_markI(prop, grid, sec, x["pm"], x["sm"], -1.0, x["corr"], x["rad"], x["k"], cm)
