"""The oracle (CPU restatement, oracle/krige_oracle.cpp) against golden vectors
produced by the reference itself (tests/golden/make_golden.py)."""
import numpy as np
import pytest

import golden_io as G
import oracle as O


@pytest.mark.parametrize("case", G.CONT_CASES)
@pytest.mark.parametrize("tag,kind", [("ok", 0), ("sk", 1)])
def test_oracle_matches_reference_per_node(case, tag, kind):
    g = G.load(case)
    wl = G.as_workload(g, case)
    r = O.krige_nodes("port", kind, wl.dims, wl.data, wl.mask, wl.cov, wl.radiuses, wl.max_neighbours,
                      mean=float(g["sk_mean"]), nodes=g["nodes"], threads=4)
    # neighbour indices: identical, in the reference's order
    np.testing.assert_array_equal(r["idx"], g[f"{tag}_idx"])
    np.testing.assert_array_equal(r["count"], g[f"{tag}_count"])
    np.testing.assert_array_equal(r["path"], g[f"{tag}_path"])
    np.testing.assert_array_equal(r["status"], g[f"{tag}_status"])
    ok = g[f"{tag}_status"] == 0
    tol = 1e-8 if case.startswith("clustered") else 1e-12  # LAPACK vs own Cholesky, cond(A) * eps
    scale = max(np.abs(g[f"{tag}_est"][ok]).max(), 1.0)
    assert np.abs(r["est"][ok] - g[f"{tag}_est"][ok]).max() <= tol * scale
    assert np.abs(r["var"][ok] - g[f"{tag}_var"][ok]).max() <= tol * max(np.abs(g[f"{tag}_var"][ok]).max(), 1.0)
    # float estimate the drivers store: same float accumulation, at most a few ulp apart
    assert np.abs(r["est_f"][ok] - g[f"{tag}_est_f"][ok]).max() <= 4e-7 * scale


@pytest.mark.parametrize("case", ["ok_small_s030", "gauss_cv_s020"])
@pytest.mark.parametrize("tag,kind", [("ok", 0), ("sk", 1)])
def test_oracle_whole_grid_matches_reference_api(case, tag, kind):
    g = G.load(case)
    wl = G.as_workload(g, case)
    od, om, _, _, _ = O.cont_grid(kind, wl.dims, wl.data, wl.mask, wl.cov, wl.radiuses, wl.max_neighbours, threads=4)
    np.testing.assert_array_equal(om, g[f"{tag}_grid_mask"])
    ref = g[f"{tag}_grid_data"]
    assert np.abs(od - ref).max() <= 4e-7 * max(np.abs(ref).max(), 1.0)


@pytest.mark.parametrize("case", ["ok_small_s030", "gauss_cv_s020"])
def test_oracle_lvm_matches_reference_api(case):
    """LVM kriging: the restatement's grid against hpgl_lvm_kriging's output."""
    g = G.load(case)
    lv = G.load("lvm")
    wl = G.as_workload(g, case)
    means = lv[f"{case}_means"]
    od, om, _, _, st = O.lvm_grid(wl.dims, wl.data, wl.mask, means, wl.cov, wl.radiuses, wl.max_neighbours,
                                  threads=4)
    np.testing.assert_array_equal(om, lv[f"{case}_grid_mask"])
    ref = lv[f"{case}_grid_data"]
    assert np.abs(od - ref).max() <= 4e-7 * max(np.abs(ref).max(), 1.0)
    failed = (wl.mask == 0) & (st != 0)
    np.testing.assert_array_equal(ref[failed], means[failed])  # mean_on_failure


@pytest.mark.parametrize("case", ["ok_small_s030", "gauss_cv_s020"])
def test_oracle_lvm_matches_reference_per_node(case):
    g = G.load(case)
    lv = G.load("lvm")
    wl = G.as_workload(g, case)
    r = O.krige_nodes("port", 1, wl.dims, wl.data, wl.mask, wl.cov, wl.radiuses, wl.max_neighbours,
                      nodes=lv[f"{case}_nodes"], threads=4, means=lv[f"{case}_means"])
    for key in ("idx", "count", "path", "status"):
        np.testing.assert_array_equal(r[key], lv[f"{case}_{key}"])
    ok = lv[f"{case}_status"] == 0
    ref = lv[f"{case}_est"][ok]
    assert np.abs(r["est"][ok] - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1.0)
    assert np.abs(r["var"][ok] - lv[f"{case}_var"][ok]).max() <= 1e-12
    assert np.abs(r["est_f"][ok] - lv[f"{case}_est_f"][ok]).max() <= 4e-7 * max(np.abs(ref).max(), 1.0)


@pytest.mark.parametrize("case", [c[0] for c in G.SGS_CASES])
def test_oracle_sgs_matches_reference(case):
    """SGS: the restatement reproduces the reference's hpgl_sgs_simulation output bit for bit."""
    _, base, kind, seed, opts = next(c for c in G.SGS_CASES if c[0] == case)
    x = G.sgs_inputs(G.load(base), opts)
    ref = G.load("sgs")
    d, m, _ = O.sgs(x["dims"], x["data"], x["mask"], x["cov"], x["rad"], x["k"], seed, kind=kind,
                    sim_mask=x["sim_mask"], cdf=x["cdf"], means=x["means"])
    np.testing.assert_array_equal(m, ref[f"{case}_mask"])
    np.testing.assert_array_equal(d.view(np.uint32), ref[f"{case}_data"].view(np.uint32))


@pytest.mark.parametrize("size", [1, 2, 4, 6, 7, 8, 9, 12, 30, 64, 1000, 4096, 12345, 65536])
def test_sgs_walk_visits_every_node_once(size):
    """The simulation path (path_random_generator.cpp) is a permutation exactly when
    its increment (the largest prime <= size/3 not dividing size, else 2) is
    coprime to the size: every size but a few small ones (2, 4, 6, 8, 12)."""
    def isprime(q):
        return q > 1 and all(q % d for d in range(2, int(q ** 0.5) + 1))
    inc = next((q for q in range(size // 3, 2, -1) if isprime(q) and size % q), 2)
    for seed in (0, 5, 123456789):
        p = O.sgs_path(size, seed)
        assert p[0] == seed % size
        assert (len(np.unique(p)) == size) == (size % inc != 0 or size == 1)
    assert (size % inc != 0 or size == 1) == (size not in (2, 4, 6, 8, 12))


def test_oracle_indicator_matches_reference():
    g = G.load("indicator_s015")
    dims, data, mask = G.grid_inputs(g, dtype=np.uint8)
    covs, rads, ks = [], [], []
    for c in range(5):
        cov, rad, k = G.cov_of(g, f"c{c}_")
        covs.append(cov)
        rads.append(rad)
        ks.append(k)
        r = O.krige_nodes("port", 1, dims, data, mask, cov, rad, k, mean=float(np.float32(g["marginals"][c])),
                          nodes=g["nodes"], ind_value=c, threads=4)
        np.testing.assert_array_equal(r["idx"], g[f"c{c}_idx"])
        np.testing.assert_array_equal(r["path"], g[f"c{c}_path"])
        ok = g[f"c{c}_status"] == 0
        assert np.abs(r["est_f"][ok] - g[f"c{c}_est_f"][ok]).max() <= 4e-7
    od, om, probs = O.indicator_grid(dims, data, mask, covs, rads, ks, list(g["marginals"]), threads=4)
    np.testing.assert_array_equal(od, g["ik_grid"])
    dims, mdata, mask = G.grid_inputs(g, "mik_values", dtype=np.uint8)
    cov, rad, _ = G.cov_of(g, "c2_")
    od, om, prob, st = O.median_ik_grid(dims, mdata, mask, cov, rad, 24, list(g["mik_marginals"]), threads=4)
    defined = st == 0  # the reference leaves failed cells undefined (median_ik.cpp:65-76)
    np.testing.assert_array_equal(od[defined], g["mik_grid"][defined])


def test_oracle_known_answers():
    """Constant field -> OK returns the constant; zeros -> 0 (reference test_edge_cases.py:368-392, 487-511)."""
    g = dict(np.load(G.GOLDEN + "/known_answers.npz"))
    from geo_bsd import workloads as WL
    cov = WL.CovSpec(WL.SPHERICAL, (10.0, 10.0, 10.0), (0.0, 0.0, 0.0), 1.0, 0.0)
    for name, val in (("const42", 42.0), ("zeros", 0.0)):
        od, om, _, _, _ = O.cont_grid(0, (10, 10, 5), g[f"{name}_data"], g[f"{name}_mask"], cov, (5, 5, 5), 12)
        np.testing.assert_array_equal(om, g[f"{name}_outmask"])
        assert np.abs(od - g[f"{name}_out"]).max() <= 1e-4
        assert np.abs(od[om == 1] - val).max() <= 0.1


def test_introsort_restatement_matches_std_sort():
    rng = np.random.default_rng(5)
    for trial in range(400):
        n = int(rng.integers(0, 3000 if trial % 10 == 0 else 200))
        distinct = int(rng.integers(1, 50))
        keys = rng.integers(0, distinct, n).astype(np.uint32)
        a, b = O.sort_check(keys)
        np.testing.assert_array_equal(a, b)


def test_introselect_matches_std_sort_first_k():
    """The O(n) tie resolver used for straddling cells picks the same first-k set as std::sort."""
    rng = np.random.default_rng(8)
    for trial in range(600):
        n = int(rng.integers(1, 3000 if trial % 7 == 0 else 300))
        distinct = int(rng.integers(1, 40))
        keys = rng.integers(0, distinct, n).astype(np.uint32)
        if trial % 5 == 0:
            keys = np.sort(keys)[::-1].copy()  # descending runs
        k = int(rng.integers(1, n + 1))
        assert O.select_check(keys, k), (n, k, distinct)


@pytest.mark.parametrize("case", [c[0] for c in G.COK_CASES])
def test_oracle_cokriging_matches_reference(case):
    """Collocated cokriging: the restatement reproduces hpgl_simple_cokriging_mark1/2 bit for bit."""
    _, base, mark = next(c for c in G.COK_CASES if c[0] == case)
    ref = G.load("cok")
    x = G.cok_inputs(G.load(base), mark, (ref[f"{base}_sdata"], ref[f"{base}_smask"]))
    d, m, st = O.cokriging(mark, x["dims"], x["pdata"], x["pmask"], x["sdata"], x["smask"], x["cov"], x["rad"], x["k"],
                           x["pm"], x["sm"], secondary_variance=x["sv"], corr=x["corr"], cov2=x["cov2"], threads=4)
    np.testing.assert_array_equal(m, ref[f"{case}_mask"])
    np.testing.assert_array_equal(d.view(np.uint32), ref[f"{case}_data"].view(np.uint32))


@pytest.mark.parametrize("case", [c[0] for c in G.SIS_CASES])
def test_oracle_sis_matches_reference(case):
    """SIS: the restatement reproduces the reference's hpgl_sis_simulation(_lvm) output exactly."""
    opts = next(c[1] for c in G.SIS_CASES if c[0] == case)
    x = G.sis_inputs(G.load("indicator_s015"), opts)
    ref = G.load("sis")
    d, m, _ = O.sis(x["dims"], x["data"], x["mask"], x["covs"], x["rads"], x["ks"], x["marginals"], x["seed"],
                    sim_mask=x["sim_mask"], means=x["means"], correlogram=x["corr"])
    np.testing.assert_array_equal(m, ref[f"{case}_mask"])
    np.testing.assert_array_equal(d, ref[f"{case}_data"])
