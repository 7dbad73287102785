"""GPU parity at the full sizes of the benchmark configurations, on sampled cells.

The engine runs the whole grid (through its C ABI); the reference's own
per-node code (the harness over the reference's templates, oracle/_ref) or,
where that build is absent, the pinned CPU restatement krige the same sampled
cells of the same grid. Compared per sampled cell: neighbour counts, search
paths and sets, status, FP64 estimate and variance (FP64 plain within 1e-10,
FP32-refined within 1e-6 relative, normwise; 1e-8 on the nugget-1e-3 Gaussian
grid, whose cond(A) eps bounds the reference's own LAPACK result); for
indicator kriging the corrected probabilities (within 2e-6) and categories,
for median IK the decisions wherever the reference defines them.

Workloads (seeded, geo_bsd.workloads): ordinary / simple kriging of the
256x256x128 grid, k = 32; the clustered 512x512x64 grid, Gaussian model with
nugget 1e-3, k = 64; full and median IK of the 200x200x100 five-category grid,
k = 24.
"""
import numpy as np
import pytest

import helpers as H
import oracle as O
from geo_bsd import workloads as WL

pytestmark = pytest.mark.gpu

WHICH = "ref" if O.available("ref") else "port"
SAMPLE = 20000


def _sample(mask, n, seed):
    rng = np.random.default_rng(seed)
    cand = np.flatnonzero(mask == 0)
    return np.sort(rng.choice(cand, min(n, len(cand)), replace=False)).astype(np.int32)


def _sets_equal(a, b):
    return all(set(x[x >= 0].tolist()) == set(y[y >= 0].tolist()) for x, y in zip(a, b))


@pytest.mark.parametrize("name,kind,sample", [("sk_ok_large", 0, SAMPLE), ("sk_ok_large", 1, SAMPLE),
                                              ("clustered", 0, 8000)])
def test_full_size_sampled_cells(name, kind, sample):
    wl = WL.ALL[name](1.0)
    nodes = _sample(wl.mask, sample, 7 + kind)
    # SK: the reference's automatic mean over the informed cells (calc_mean.cpp:6-30), as the engine forms it
    mean = 0.0 if kind == 0 else float(wl.data[wl.mask == 1].astype(np.float64).mean())
    ref = O.krige_nodes(WHICH, kind, wl.dims, wl.data, wl.mask, wl.cov, wl.radiuses, wl.max_neighbours,
                        mean=mean, nodes=nodes, threads=0)
    idx, cnt, path = H.engine_neighbours(kind, wl, nodes)
    np.testing.assert_array_equal(cnt, ref["count"])
    np.testing.assert_array_equal(path, ref["path"])
    assert _sets_equal(idx, ref["idx"])
    for precision in (0, 1):
        e = H.engine_cont(kind, wl, precision=precision)
        st = e["status"][nodes]
        np.testing.assert_array_equal(st, ref["status"].astype(np.int8))
        ok = st == 0
        tol = 1e-10 if precision == 0 else 1e-6
        if name == "clustered":
            tol = max(tol, 1e-8)
        assert H.rel_err(e["est"][nodes][ok], ref["est"][ok]) <= tol, precision
        assert H.rel_err(e["var"][nodes][ok], ref["var"][ok]) <= tol, precision
        del e


def _order_relations(probs):
    """correct_order_relations (indicator_kriging.h:34-59) on float probabilities."""
    p = np.clip(np.asarray(probs, np.float32), 0.0, 1.0)
    for i in range(p.shape[1] - 1):
        sel = p[:, i] > p[:, i + 1]
        avg = ((p[sel, i].astype(np.float64) + p[sel, i + 1].astype(np.float64)) / 2.0).astype(np.float32)
        p[sel, i] = avg
        p[sel, i + 1] = avg
    return p


@pytest.mark.parametrize("precision", [0, 1])
def test_full_size_indicator_kriging_sampled_cells(precision):
    """Full IK (indicator_kriging.h:88-161): every cell, informed ones included,
    is kriged per category around its marginal; failures take the marginal."""
    wl = WL.indicator(1.0)
    m = len(wl.cat_covs)
    ks = [wl.max_neighbours] * m
    out_d, out_m, probs = H.engine_indicator(wl, wl.cat_covs, wl.cat_radiuses, ks, list(wl.marginals),
                                             precision=precision)
    assert np.all(out_m == 1)
    rng = np.random.default_rng(9)
    nodes = np.sort(rng.choice(wl.n_cells, SAMPLE, replace=False)).astype(np.int32)
    raw = np.zeros((len(nodes), m), np.float32)
    for c in range(m):
        r = O.krige_nodes(WHICH, 1, wl.dims, wl.data, wl.mask, wl.cat_covs[c], wl.cat_radiuses[c], ks[c],
                          mean=float(np.float32(wl.marginals[c])), nodes=nodes, ind_value=c, want_idx=False)
        raw[:, c] = np.where(r["status"] == 0, r["est_f"], np.float32(wl.marginals[c]))
    ref = _order_relations(raw)
    assert np.abs(probs[nodes] - ref).max() <= 2e-6
    # most_probable_category (cdf_utils.cpp:11-27): the first maximum
    np.testing.assert_array_equal(out_d[nodes], np.argmax(ref, axis=1).astype(np.uint8))


@pytest.mark.parametrize("precision", [0, 1])
def test_full_size_median_ik_sampled_cells(precision):
    """Median IK (median_ik.cpp:24-89) with category 2's model on the indicator
    (category >= 2), marginals (0.6, 0.4): the SK probability and the
    decision prob > 0.5 wherever the reference's kriging succeeds."""
    wl0 = WL.indicator(1.0)
    data = (wl0.data >= 2).astype(np.uint8)
    wl = WL.Workload("mik", wl0.dims, data, wl0.mask, None, None, wl0.max_neighbours)
    cov, rad, k, mp = wl0.cat_covs[2], wl0.cat_radiuses[2], wl0.max_neighbours, (0.6, 0.4)
    out_d, out_m, prob = H.engine_median_ik(wl, cov, rad, k, list(mp), precision=precision)
    rng = np.random.default_rng(10)
    nodes = np.sort(rng.choice(wl.n_cells, SAMPLE, replace=False)).astype(np.int32)
    r = O.krige_nodes(WHICH, 2, wl.dims, data, wl.mask, cov, rad, k, mean=float(np.float32(mp[1])), nodes=nodes,
                      ind_value=1, want_idx=False)
    ok = r["status"] == 0
    assert ok.mean() > 0.9
    assert np.abs(prob[nodes][ok] - r["est_f"][ok]).max() <= 2e-6
    decided = ok & (np.abs(r["est_f"] - 0.5) > 1e-5)
    np.testing.assert_array_equal(out_d[nodes][decided], (r["est_f"][decided] > 0.5).astype(np.uint8))
