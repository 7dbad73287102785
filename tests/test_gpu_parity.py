"""GPU parity: the engine (through its C ABI) against the reference's golden
vectors and the oracle.

Bars: neighbour sets bit-exact (node indices), and the order position by
position except inside groups of equal covariance keys (the reference orders
candidates with an unstable std::sort, so the order inside such a group is
libstdc++'s permutation; the set of a group that straddles slot k is still
exact); FP64-plain estimates and variances within 1e-10 relative of the
reference's FP64 path; FP32-refined within 1e-6; per-cell status identical;
the float grid the reference's public API writes reproduced to float
rounding; indicator probabilities within 2e-6 and categories identical.
"""
import ctypes as C

import numpy as np
import pytest

import golden_io as G
import helpers as H
import oracle as O
from geo_bsd import hpgl_wrap as W
from geo_bsd import workloads as WL

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_TOL = 1e-6


def _sets_equal(a, b):
    return all(set(x[x >= 0].tolist()) == set(y[y >= 0].tolist()) for x, y in zip(a, b))


def _xyz(node, dims):
    return [node % dims[0], (node // dims[0]) % dims[1], node // (dims[0] * dims[1])]


def _order_matches(nodes, idx, ref_idx, dims, kind, cov, radiuses):
    """Position-by-position order of each neighbour list against the
    reference's, where runs of equal covariance keys (from the pinned CPU
    restatement of the reference's covariance) compare as sets. Returns the
    number of positions compared exactly."""
    which = "ref" if O.available("ref") else "port"
    cache = {}  # the key depends on the displacement only

    def key(c, p):
        d = tuple(b - a for a, b in zip(c, p))
        if d not in cache:
            cache[d] = O.cov_point(which, kind, cov, radiuses, [0, 0, 0], list(d))
        return cache[d]

    exact = 0
    for node, mine, ref in zip(nodes, idx, ref_idx):
        ref = ref[ref >= 0]
        mine = mine[: len(ref)]
        c = _xyz(int(node), dims)
        keys = [key(c, _xyz(int(p), dims)) for p in ref]
        i = 0
        while i < len(ref):
            j = i + 1
            while j < len(ref) and keys[j] == keys[i]:
                j += 1
            if j - i == 1:
                assert mine[i] == ref[i], (node, i)
                exact += 1
            else:
                assert set(mine[i:j].tolist()) == set(ref[i:j].tolist()), (node, i, j)
            i = j
    return exact


@pytest.mark.parametrize("case", G.CONT_CASES)
@pytest.mark.parametrize("tag,kind", [("ok", 0), ("sk", 1)])
def test_neighbour_order_matches_reference(case, tag, kind):
    g = G.load(case)
    wl = G.as_workload(g, case)
    nodes = g["nodes"]
    idx, cnt, _ = H.engine_neighbours(kind, wl, nodes)
    np.testing.assert_array_equal(cnt, g[f"{tag}_count"])
    exact = _order_matches(nodes, idx, g[f"{tag}_idx"], wl.dims, kind, wl.cov, wl.radiuses)
    assert exact > 0


@pytest.mark.parametrize("case", G.CONT_CASES)
@pytest.mark.parametrize("tag,kind", [("ok", 0), ("sk", 1)])
def test_neighbours_match_reference(case, tag, kind):
    g = G.load(case)
    wl = G.as_workload(g, case)
    idx, cnt, path = H.engine_neighbours(kind, wl, g["nodes"])
    np.testing.assert_array_equal(cnt, g[f"{tag}_count"])
    np.testing.assert_array_equal(path, g[f"{tag}_path"])
    assert _sets_equal(idx, g[f"{tag}_idx"])


@pytest.mark.parametrize("case", G.CONT_CASES)
@pytest.mark.parametrize("tag,kind", [("ok", 0), ("sk", 1)])
@pytest.mark.parametrize("precision", [0, 1])
def test_estimates_match_reference(case, tag, kind, precision):
    g = G.load(case)
    wl = G.as_workload(g, case)
    e = H.engine_cont(kind, wl, precision=precision, mean=None)
    nodes = g["nodes"]
    st = e["status"][nodes]
    np.testing.assert_array_equal(st, g[f"{tag}_status"].astype(np.int8))
    ok = st == 0
    tol = FP64_TOL if precision == 0 else FP32_TOL
    if case.startswith("clustered"):
        tol = max(tol, 1e-8)  # nugget 1e-3 Gaussian: cond(A) * eps of the reference's own LAPACK path
    assert H.rel_err(e["est"][nodes][ok], g[f"{tag}_est"][ok]) <= tol
    assert H.rel_err(e["var"][nodes][ok], g[f"{tag}_var"][ok]) <= tol


@pytest.mark.parametrize("case", ["ok_small_s030", "gauss_cv_s020"])
@pytest.mark.parametrize("tag,kind", [("ok", 0), ("sk", 1)])
def test_grid_output_matches_reference_api(case, tag, kind):
    """The float grid and mask that the reference's hpgl_ordinary_kriging /
    hpgl_simple_kriging write, reproduced through the engine's compatible entry points."""
    g = G.load(case)
    wl = G.as_workload(g, case)
    n = wl.n_cells
    data = np.ascontiguousarray(wl.data)
    mask = np.ascontiguousarray(wl.mask)
    out_d, out_m = data.copy(), mask.copy()
    sh = W._HPGL_SHAPE(data=wl.dims, strides=(1, wl.dims[0], wl.dims[0] * wl.dims[1]))
    fp = C.POINTER(C.c_float)
    up = C.POINTER(C.c_ubyte)
    if kind == 0:
        p = W._HPGL_OK_PARAMS(covariance_type=wl.cov.cov_type, ranges=wl.cov.ranges, angles=wl.cov.angles,
                              sill=wl.cov.sill, nugget=wl.cov.nugget, radiuses=wl.radiuses,
                              max_neighbours=wl.max_neighbours)
        a = W._HPGL_CONT_MASKED_ARRAY(data.ctypes.data_as(fp), mask.ctypes.data_as(up), sh)
        b = W._HPGL_CONT_MASKED_ARRAY(out_d.ctypes.data_as(fp), out_m.ctypes.data_as(up), sh)
        W._hpgl_so.hpgl_ordinary_kriging(C.byref(a), C.byref(p), C.byref(b))
    else:
        p = W._HPGL_SK_PARAMS(covariance_type=wl.cov.cov_type, ranges=wl.cov.ranges, angles=wl.cov.angles,
                              sill=wl.cov.sill, nugget=wl.cov.nugget, radiuses=wl.radiuses,
                              max_neighbours=wl.max_neighbours, automatic_mean=1, mean=0.0)
        d3 = data.reshape(wl.dims, order="F")
        m3 = mask.reshape(wl.dims, order="F")
        o3 = out_d.reshape(wl.dims, order="F")
        om3 = out_m.reshape(wl.dims, order="F")
        W._hpgl_so.hpgl_simple_kriging(d3, m3, C.byref(sh), C.byref(p), o3, om3, C.byref(sh))
    assert W.last_error() == "" or W.last_stats()["kriged_cells"] > 0
    np.testing.assert_array_equal(out_m, g[f"{tag}_grid_mask"])
    ref = g[f"{tag}_grid_data"]
    assert np.abs(out_d - ref).max() <= 1e-6 * max(np.abs(ref).max(), 1.0)
    assert n == len(ref)


def _order_relations(probs):
    """correct_order_relations (indicator_kriging.h:34-59) on float
    probabilities: clamp to [0, 1], then one left-to-right pass replacing a
    decreasing pair by its average (formed in double, stored as float)."""
    p = np.clip(np.asarray(probs, np.float32), 0.0, 1.0)
    for i in range(p.shape[1] - 1):
        sel = p[:, i] > p[:, i + 1]
        avg = ((p[sel, i].astype(np.float64) + p[sel, i + 1].astype(np.float64)) / 2.0).astype(np.float32)
        p[sel, i] = avg
        p[sel, i + 1] = avg
    return p


@pytest.mark.parametrize("precision", [0, 1])
def test_indicator_probabilities_match_reference(precision):
    """Corrected per-category probabilities at the golden nodes against the
    reference's own per-category SK results (its float estimate, the marginal
    where kriging failed: indicator_kriging.h:125-153), corrected as it does."""
    g = G.load("indicator_s015")
    dims, data, mask = G.grid_inputs(g, dtype=np.uint8)
    wl = WL.Workload("ik", dims, data, mask, None, None, 24)
    covs, rads, ks = [], [], []
    for c in range(5):
        cov, rad, k = G.cov_of(g, f"c{c}_")
        covs.append(cov)
        rads.append(rad)
        ks.append(k)
    marg = list(g["marginals"])
    _, _, probs = H.engine_indicator(wl, covs, rads, ks, marg, precision=precision)
    nodes = g["nodes"]
    raw = np.stack([np.where(g[f"c{c}_status"] == 0, g[f"c{c}_est_f"], np.float32(marg[c])) for c in range(5)], 1)
    ref = _order_relations(raw)
    assert np.abs(probs[nodes] - ref).max() <= 2e-6


@pytest.mark.parametrize("precision", [0, 1])
def test_indicator_kriging_wide_systems_against_oracle(precision):
    """IK with 40 to 64 neighbours per category (the 33-64 bucket's one-warp
    kernels writing per-category probabilities): corrected probabilities
    within 1e-5 of the CPU oracle's and categories identical wherever the
    oracle's largest probability is not within that of the runner-up."""
    wl = WL.indicator(0.3)
    covs, rads = wl.cat_covs, wl.cat_radiuses
    ks = [40, 48, 56, 64, 48]
    od, om, op = O.indicator_grid(wl.dims, wl.data, wl.mask, covs, rads, ks, wl.marginals)
    out_d, out_m, probs = H.engine_indicator(wl, covs, rads, ks, wl.marginals, precision=precision)
    np.testing.assert_array_equal(out_m, om)
    assert np.abs(probs - op).max() <= 1e-5
    top2 = np.sort(op, axis=1)[:, -2:]
    clear = (top2[:, 1] - top2[:, 0]) > 1e-5
    np.testing.assert_array_equal(out_d[clear], od[clear])
    _, cnt, _ = H.engine_neighbours(1, wl, np.flatnonzero(wl.mask == 0)[::97], cov=covs[3], radiuses=rads[3],
                                    k=ks[3])
    assert (cnt > 32).mean() > 0.5  # the wide kernels carry most systems


@pytest.mark.parametrize("precision", [0, 1])
def test_indicator_kriging_matches_reference(precision):
    g = G.load("indicator_s015")
    dims, data, mask = G.grid_inputs(g, dtype=np.uint8)
    wl = WL.Workload("ik", dims, data, mask, None, None, 24)
    covs, rads, ks = [], [], []
    for c in range(5):
        cov, rad, k = G.cov_of(g, f"c{c}_")
        covs.append(cov)
        rads.append(rad)
        ks.append(k)
    out_d, out_m, probs = H.engine_indicator(wl, covs, rads, ks, list(g["marginals"]), precision=precision)
    np.testing.assert_array_equal(out_d, g["ik_grid"])
    assert np.all(out_m == 1)
    for c in range(5):
        nodes = g["nodes"]
        idx, cnt, path = H.engine_neighbours(1, wl, nodes, cov=covs[c], radiuses=rads[c], k=ks[c])
        assert _sets_equal(idx, g[f"c{c}_idx"])
        np.testing.assert_array_equal(path, g[f"c{c}_path"])


@pytest.mark.parametrize("precision", [0, 1])
def test_median_ik_matches_reference(precision):
    g = G.load("indicator_s015")
    dims, data, mask = G.grid_inputs(g, "mik_values", dtype=np.uint8)
    wl = WL.Workload("mik", dims, data, mask, None, None, 24)
    cov, rad, _ = G.cov_of(g, "c2_")
    out_d, out_m, prob = H.engine_median_ik(wl, cov, rad, 24, list(g["mik_marginals"]), precision=precision)
    # cells where the reference's kriging failed hold an uninitialised decision there
    _, _, _, st = O.median_ik_grid(dims, data, mask, cov, rad, 24, list(g["mik_marginals"]))
    ok = st == 0
    np.testing.assert_array_equal(out_d[ok], g["mik_grid"][ok])


def test_known_answers():
    """Constant field 42 -> 42 and zeros -> 0 (reference test_edge_cases.py:368-392, 487-511)."""
    g = dict(np.load(G.GOLDEN + "/known_answers.npz"))
    for name, val in (("const42", 42.0), ("zeros", 0.0)):
        wl = WL.Workload(name, (10, 10, 5), g[f"{name}_data"], g[f"{name}_mask"],
                         WL.CovSpec(WL.SPHERICAL, (10.0, 10.0, 10.0), (0.0, 0.0, 0.0), 1.0, 0.0), (5, 5, 5), 12)
        for precision in (0, 1):
            e = H.engine_cont(0, wl, precision=precision)
            np.testing.assert_array_equal(e["mask"], g[f"{name}_outmask"])
            assert np.abs(e["data"] - g[f"{name}_out"]).max() <= 1e-4
            assert np.abs(e["data"][e["mask"] == 1] - val).max() <= 0.1


@pytest.mark.parametrize("name,scale", [("ok_small", 0.6), ("sk_ok_large", 0.3), ("gauss_cv", 0.35),
                                        ("clustered", 0.2)])
@pytest.mark.parametrize("kind", [0, 1])
def test_larger_grids_against_oracle(name, scale, kind):
    wl = WL.ALL[name](scale)
    od, om, oest, ovar, ost = O.cont_grid(kind, wl.dims, wl.data, wl.mask, wl.cov, wl.radiuses, wl.max_neighbours)
    unk = wl.mask == 0
    for precision in (0, 1):
        e = H.engine_cont(kind, wl, precision=precision)
        np.testing.assert_array_equal(e["status"][unk], ost[unk].astype(np.int8))
        np.testing.assert_array_equal(e["mask"], om)
        ok = unk & (ost == 0)
        tol = FP64_TOL if precision == 0 else FP32_TOL
        if name == "clustered":
            tol = max(tol, 1e-8)
        assert H.rel_err(e["est"][ok], oest[ok]) <= tol, (precision, H.rel_err(e["est"][ok], oest[ok]))
        assert H.rel_err(e["var"][ok], ovar[ok]) <= tol
    rng = np.random.default_rng(1)
    nodes = np.sort(rng.choice(np.flatnonzero(unk), 2000, replace=False))
    idx, cnt, path = H.engine_neighbours(kind, wl, nodes)
    r = O.krige_nodes("port", kind, wl.dims, wl.data, wl.mask, wl.cov, wl.radiuses, wl.max_neighbours,
                      nodes=nodes)
    np.testing.assert_array_equal(cnt, r["count"])
    np.testing.assert_array_equal(path, r["path"])
    assert _sets_equal(idx, r["idx"])


@pytest.mark.parametrize("name,scale,kind", [("sk_ok_large", 1.0, 0), ("sk_ok_large", 0.5, 1),
                                             ("gauss_cv", 0.5, 0), ("clustered", 0.35, 1), ("ok_small", 1.0, 0)])
def test_float_prefilter_selects_the_exact_neighbours(name, scale, kind):
    """The float distance prefilter changes no neighbour set: FP64 estimates and variances
    are bit-identical to a search by exact ranks over every candidate, at full size."""
    wl = WL.ALL[name](scale)
    a = H.engine_cont(kind, wl, precision=0)
    b = H.engine_cont(kind, wl, precision=0, flags=W.FLAG_EXACT_SEARCH)
    assert b["stats"]["prefilter_active"] == 0.0
    np.testing.assert_array_equal(a["status"], b["status"])
    np.testing.assert_array_equal(a["est"], b["est"])
    np.testing.assert_array_equal(a["var"], b["var"])
    np.testing.assert_array_equal(a["data"], b["data"])
    assert a["stats"]["tie_cells"] == b["stats"]["tie_cells"]
    if name == "sk_ok_large" and kind == 0:
        # the benchmark model passes the host monotonicity check; most cells are decided in float
        assert a["stats"]["prefilter_active"] == 1.0
        assert a["stats"]["prefilter_exact_cells"] <= 0.25 * a["stats"]["kriged_cells"]


def test_simple_kriging_weights_entry():
    rng = np.random.default_rng(4)
    for cov in (WL.CovSpec(WL.EXPONENTIAL, (10.0, 10.0, 10.0), (0.0, 0.0, 0.0), 1.0, 0.0),
                WL.CovSpec(WL.GAUSSIAN, (20.0, 10.0, 5.0), (30.0, 0.0, 0.0), 1.0, 0.1)):
        xs, ys, zs = (rng.uniform(0, 10, 12).astype(np.float32) for _ in range(3))
        centre = np.array([5.0, 5.0, 5.0], np.float32)
        covp = W._HPGL_COV_PARAMS(covariance_type=cov.cov_type, ranges=cov.ranges, angles=cov.angles,
                                  sill=cov.sill, nugget=cov.nugget)
        w = np.zeros(12, np.float32)
        rc = W._hpgl_so.hpgl_simple_kriging_weights((C.c_float * 3)(*centre), xs, ys, zs, 12, C.byref(covp), w)
        assert rc == 0
        ref, _ = O.sk_weights("port", centre.astype(np.float64), xs.astype(np.float64), ys.astype(np.float64),
                              zs.astype(np.float64), cov)
        assert np.abs(w - ref).max() <= 1e-5 * max(1.0, np.abs(ref).max())
