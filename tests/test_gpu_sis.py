"""Sequential indicator simulation on the GPU.

Bars: simulated categories and masks identical to the reference's (golden
fixtures) and to the oracle's at larger sizes; per-node status identical to
the oracle's. The categories come from double probabilities through one draw
per node: the weights come from a different Cholesky than LAPACK's, so a pick
could in principle move where a draw lands within an ulp of a category
boundary; none does on these cases and the tests hold them to exact equality.
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


def _run(x, **kw):
    return H.engine_sis(x["dims"], x["data"], x["mask"], x["covs"], x["rads"], x["ks"], x["marginals"],
                        kw.get("seed", x["seed"]), sim_mask=x["sim_mask"], means=x["means"], corr=x["corr"])


def _oracle(x, seed=None):
    return O.sis(x["dims"], x["data"], x["mask"], x["covs"], x["rads"], x["ks"], x["marginals"],
                 x["seed"] if seed is None else seed, sim_mask=x["sim_mask"], means=x["means"],
                 correlogram=x["corr"])


def _same_as_oracle(e, od, om, ost, mask_in):
    np.testing.assert_array_equal(e["mask"], om)
    np.testing.assert_array_equal(e["data"], od)
    sim = ost >= 0
    np.testing.assert_array_equal(e["status"][sim], ost[sim].astype(np.int8))
    # cells not simulated: -1 informed, 3 left out by the simulation mask
    np.testing.assert_array_equal(e["status"][~sim], np.where(np.asarray(mask_in)[~sim] == 1, -1, 3))


@pytest.mark.parametrize("case", [c[0] for c in G.SIS_CASES])
def test_sis_matches_reference(case):
    opts = next(c[1] for c in G.SIS_CASES if c[0] == case)
    x = G.sis_inputs(G.load("indicator_s015"), opts)
    ref = G.load("sis")
    e = _run(x)
    np.testing.assert_array_equal(e["mask"], ref[f"{case}_mask"])
    np.testing.assert_array_equal(e["data"], ref[f"{case}_data"])
    _same_as_oracle(e, *_oracle(x), x["mask"])
    assert e["stats"]["sgs_levels"] > 0 and e["stats"]["sgs_flops"] > 0


def _ind_struct(d, m, dims, ncat):
    up = C.POINTER(C.c_ubyte)
    sh = W._HPGL_SHAPE(data=dims, strides=(1, dims[0], dims[0] * dims[1]))
    return W._HPGL_IND_MASKED_ARRAY(d.ctypes.data_as(up), m.ctypes.data_as(up), sh, ncat)


def test_reference_entry_points_match_ex():
    """hpgl_sis_simulation / hpgl_sis_simulation_lvm (the reference's signatures, in place) give the _ex result."""
    for case in ("sis5_mask", "sis5_lvm_corr"):
        opts = next(c[1] for c in G.SIS_CASES if c[0] == case)
        x = G.sis_inputs(G.load("indicator_s015"), opts)
        e = _run(x)
        d = x["data"].copy()
        m = x["mask"].copy()
        ncat = len(x["covs"])
        arr = _ind_struct(d, m, x["dims"], ncat)
        params = H.ik_params(x["covs"], x["rads"], x["ks"], x["marginals"])
        sh = W._HPGL_SHAPE(data=x["dims"], strides=(1, x["dims"][0], x["dims"][0] * x["dims"][1]))
        sm = None
        if x["sim_mask"] is not None:
            smv = np.ascontiguousarray(x["sim_mask"], np.uint8)
            sm = W._HPGL_UBYTE_ARRAY(smv.ctypes.data_as(C.POINTER(C.c_ubyte)), sh)
        if x["means"] is None:
            W._hpgl_so.hpgl_sis_simulation(C.byref(arr), params, ncat, x["seed"], C.byref(sm) if sm else None)
        else:
            keep = [np.ascontiguousarray(v, np.float32) for v in x["means"]]
            fa = (W._HPGL_FLOAT_ARRAY * ncat)(*[W._HPGL_FLOAT_ARRAY(v.ctypes.data_as(C.POINTER(C.c_float)), sh)
                                                for v in keep])
            W._hpgl_so.hpgl_sis_simulation_lvm(C.byref(arr), params, fa, ncat, x["seed"],
                                               C.byref(sm) if sm else None, int(x["corr"]))
        np.testing.assert_array_equal(d, e["data"])
        np.testing.assert_array_equal(m, e["mask"])


def _scaled(scale, k, seed=41, **opts):
    wl = WL.indicator(scale)
    data = np.where(wl.mask == 1, wl.data, 0).astype(np.uint8)
    covs, rads, marg = list(wl.cat_covs), list(wl.cat_radiuses), list(wl.marginals)
    if opts.get("two"):
        data = ((data >= 2).astype(np.uint8) * wl.mask).astype(np.uint8)
        covs, rads, marg = covs[1:3], rads[1:3], [0.45, 0.55]
    x = {"dims": wl.dims, "data": data, "mask": wl.mask.copy(), "covs": covs, "rads": rads, "ks": [k] * len(covs),
         "marginals": marg, "seed": seed, "sim_mask": None, "means": None, "corr": bool(opts.get("corr"))}
    if "sim_mask" in opts:
        x["sim_mask"] = (np.random.default_rng(8).random(wl.n_cells) < opts["sim_mask"]).astype(np.uint8)
    if opts.get("lvm"):
        t = WL.lvm_means(wl.dims)
        t = (t - t.min()) / max(float(t.max() - t.min()), 1e-6)
        x["means"] = [(np.float32(marg[c]) * (0.75 + 0.5 * t)).astype(np.float32) for c in range(len(covs))]
    return x


@pytest.mark.parametrize("scale,k,opts", [(0.3, 12, {}),
                                          (0.4, 24, {"sim_mask": 0.5}),
                                          (0.25, 32, {"lvm": True, "corr": True}),
                                          (0.3, 16, {"lvm": True}),
                                          (0.35, 20, {"two": True})])
def test_sis_against_oracle(scale, k, opts):
    """Larger grids: 62k-256k cells, k up to 32, masks, LVM with and without correlograms, median SIS."""
    x = _scaled(scale, k, **opts)
    e = _run(x)
    _same_as_oracle(e, *_oracle(x), x["mask"])


@pytest.mark.parametrize("dims", [(1, 1, 1), (3, 1, 1), (5, 2, 1), (5, 3, 2), (7, 5, 3)])
def test_small_grids(dims):
    n = int(np.prod(dims))
    rng = np.random.default_rng(n)
    data = rng.integers(0, 3, n).astype(np.uint8)
    mask = (rng.random(n) < 0.3).astype(np.uint8)
    data *= mask
    covs = [WL.CovSpec(WL.SPHERICAL, (4.0, 4.0, 4.0), (0.0, 0.0, 0.0), 1.0, 0.1)] * 3
    rads = [(3, 3, 3)] * 3
    for seed in (0, 13):
        od, om, ost = O.sis(dims, data, mask, covs, rads, [8] * 3, [0.3, 0.3, 0.4], seed)
        e = H.engine_sis(dims, data, mask, covs, rads, [8] * 3, [0.3, 0.3, 0.4], seed)
        _same_as_oracle(e, od, om, ost, mask)


def test_rejected_arguments():
    cov = WL.CovSpec(WL.SPHERICAL, (4.0, 4.0, 4.0), (0.0, 0.0, 0.0), 1.0, 0.1)
    dims = (6, 5, 4)
    n = 120
    data = np.zeros(n, np.uint8)
    mask = np.zeros(n, np.uint8)
    # a walk that does not visit every node (4 cells), more than 32 neighbours,
    # more than 16 categories, one category
    for d, ncat, k in (((2, 2, 1), 3, 8), (dims, 3, 33), (dims, 17, 8), (dims, 1, 8)):
        nn = int(np.prod(d))
        with pytest.raises(RuntimeError):
            H.engine_sis(d, data[:nn], mask[:nn], [cov] * ncat, [(3, 3, 3)] * ncat, [k] * ncat,
                         [1.0 / ncat] * ncat, 5)


def test_deterministic_and_seeded():
    x = _scaled(0.3, 12)
    a = _run(x, seed=2024)
    b = _run(x, seed=2024)
    c = _run(x, seed=2025)
    np.testing.assert_array_equal(a["data"], b["data"])
    assert (a["data"] != c["data"]).mean() > 0.3


def test_device_pointers_on_a_caller_stream():
    x = _scaled(0.3, 16, lvm=True, corr=True, sim_mask=0.7)
    host = _run(x)
    dev = torch.device("cuda")
    d = torch.from_numpy(x["data"]).to(dev)
    m = torch.from_numpy(x["mask"]).to(dev)
    sm = torch.from_numpy(x["sim_mask"]).to(dev)
    means = [torch.from_numpy(v).to(dev) for v in x["means"]]
    mp = (C.c_void_p * len(means))(*[v.data_ptr() for v in means])
    stt = torch.empty(d.numel(), dtype=torch.int8, device=dev)
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    opt = W._HPGL_B200_OPTIONS(precision=0, refine_steps=0, flags=W.FLAG_DEVICE_POINTERS, stream=s.cuda_stream,
                               estimate64=None, variance=None, status=stt.data_ptr(), ik_probs=None)
    params = H.ik_params(x["covs"], x["rads"], x["ks"], x["marginals"])
    rc = W._hpgl_so.hpgl_b200_sis_ex((C.c_int * 3)(*x["dims"]), d.data_ptr(), m.data_ptr(), sm.data_ptr(), params,
                                     len(x["covs"]), C.cast(mp, C.c_void_p), x["seed"], 1, C.byref(opt))
    W.check(rc, "sis_ex")
    s.synchronize()
    np.testing.assert_array_equal(d.cpu().numpy(), host["data"])
    np.testing.assert_array_equal(m.cpu().numpy(), host["mask"])
    np.testing.assert_array_equal(stt.cpu().numpy(), host["status"])


def test_geo_sis_simulation_api():
    x = _scaled(0.3, 12)
    dims = x["dims"]
    grid = geo_bsd.SugarboxGrid(*dims)
    f = lambda a: a.reshape(dims, order="F").copy(order="F")  # noqa: E731
    prop = geo_bsd.IndProperty(f(x["data"]), f(x["mask"]), 5)
    data = [{"cov_model": geo_bsd.CovarianceModel(type=c.cov_type, ranges=c.ranges, angles=c.angles, sill=c.sill,
                                                  nugget=c.nugget),
             "radiuses": r, "max_neighbours": 12} for c, r in zip(x["covs"], x["rads"])]
    out = geo_bsd.sis_simulation(prop, grid, data, 41, x["marginals"])
    od, om, _ = _oracle(x)
    np.testing.assert_array_equal(out.data.reshape(-1, order="F"), od)
    assert np.all(out.mask == 1) and out.indicator_count == 5
    assert data[0]["marginal_prob"] == x["marginals"][0]
    # use_harddata=False simulates every cell unconditioned
    out2 = geo_bsd.sis_simulation(prop, grid, data, 41, x["marginals"], use_harddata=False)
    z = dict(x, data=np.zeros_like(x["data"]), mask=np.zeros_like(x["mask"]))
    np.testing.assert_array_equal(out2.data.reshape(-1, order="F"), _oracle(z)[0])
    # mean arrays select LVM with correlogram weights (the default); a mask leaves the other cells alone
    y = _scaled(0.3, 12, lvm=True, corr=True)
    sm = np.zeros(dims, np.uint8, order="F")
    sm[:, :, : dims[2] // 2] = 1
    out3 = geo_bsd.sis_simulation(prop, grid, data, 41, [f(v) for v in y["means"]], mask=sm)
    y["sim_mask"] = sm.reshape(-1, order="F")
    od3, om3, _ = _oracle(y)
    np.testing.assert_array_equal(out3.mask.reshape(-1, order="F"), om3)
    np.testing.assert_array_equal(out3.data.reshape(-1, order="F"), od3)
    assert data[0]["marginal_prob"] == 0
    out4 = geo_bsd.sis_simulation(prop, grid, data, 41, [f(v) for v in y["means"]], use_correlogram=False, mask=sm)
    y["corr"] = False
    np.testing.assert_array_equal(out4.data.reshape(-1, order="F"), _oracle(y)[0])
