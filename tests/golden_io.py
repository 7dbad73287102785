"""Loading of the committed golden fixtures (tests/golden/*.npz)."""
import os

import numpy as np

from geo_bsd import workloads as WL

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CONT_CASES = ["ok_small_s030", "sk_ok_large_s016", "gauss_cv_s020", "clustered_s010"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def grid_inputs(g, values_key="values", dtype=np.float32, undefined=-99.0):
    dims = tuple(int(v) for v in g["dims"])
    n = dims[0] * dims[1] * dims[2]
    data = np.full(n, undefined, dtype)
    mask = np.zeros(n, np.uint8)
    data[g["informed"]] = g[values_key]
    mask[g["informed"]] = 1
    return dims, data, mask


def cov_of(g, prefix=""):
    cov = WL.CovSpec(int(g[prefix + "cov_type"]), tuple(float(v) for v in g[prefix + "ranges"]),
                     tuple(float(v) for v in g[prefix + "angles"]), float(g[prefix + "sill"]),
                     float(g[prefix + "nugget"]))
    return cov, tuple(int(v) for v in g[prefix + "radiuses"]), int(g[prefix + "k"])


def as_workload(g, name="golden", values_key="values", dtype=np.float32, prefix=""):
    dims, data, mask = grid_inputs(g, values_key, dtype, undefined=-99.0 if dtype == np.float32 else 0)
    cov, rad, k = cov_of(g, prefix)
    return WL.Workload(name, dims, data, mask, cov, rad, k)


def empirical_cdf(values):
    """calc_cdf (cdf.py:8-40) of a set of values: distinct values without the
    largest, with the running sum of their frequencies."""
    v, c = np.unique(np.asarray(values, np.float32), return_counts=True)
    size = v.size - 1 if v.size > 1 else v.size
    return v[:size].astype(np.float32), np.cumsum(c[:size] / float(len(values))).astype(np.float32)


SGS_CASES = [
    # name, base fixture, kind, seed, options
    ("sk_plain", "gauss_cv_s020", 1, 1234, {}),
    ("ok_cdf", "gauss_cv_s020", 0, 7, {"cdf": True}),
    ("sk_mask", "gauss_cv_s020", 1, 99, {"sim_mask": 0.7}),
    ("lvm_cdf", "gauss_cv_s020", 1, 5, {"lvm": 0.5, "cdf": True}),
    ("sk_nohard", "ok_small_s030", 1, 3, {"nohard": True}),
    ("ok_plain", "ok_small_s030", 0, 11, {}),
]


def sgs_inputs(g, opts):
    """Inputs of an SGS golden case from its base fixture: data, mask, sim mask,
    cdf, means (the sill/nugget normalisation of sgs.py:108 applied to cov)."""
    dims = tuple(int(v) for v in g["dims"])
    n = dims[0] * dims[1] * dims[2]
    data = np.full(n, -99.0, np.float32)
    mask = np.zeros(n, np.uint8)
    data[g["informed"]] = g["values"]
    mask[g["informed"]] = 1
    cov = WL.CovSpec(int(g["cov_type"]), tuple(float(v) for v in g["ranges"]), tuple(float(v) for v in g["angles"]),
                     1.0, float(g["nugget"]) / float(g["sill"]))
    out = {"dims": dims, "data": data, "mask": mask, "cov": cov, "rad": tuple(int(v) for v in g["radiuses"]),
           "k": int(g["k"]), "sim_mask": None, "cdf": None, "means": None}
    if "sim_mask" in opts:
        out["sim_mask"] = (np.random.default_rng(3).random(n) < opts["sim_mask"]).astype(np.uint8)
    if opts.get("cdf"):
        out["cdf"] = empirical_cdf(g["values"])
    if "lvm" in opts:
        out["means"] = (WL.lvm_means(dims) * np.float32(opts["lvm"])).astype(np.float32)
    if opts.get("nohard"):
        out["data"] = np.zeros(n, np.float32)
        out["mask"] = np.zeros(n, np.uint8)
    return out


COK_CASES = [
    # name, base fixture, mark
    ("m1_gauss", "gauss_cv_s020", 1),
    ("m2_gauss", "gauss_cv_s020", 2),
    ("m1_small", "ok_small_s030", 1),
]
COK_SECONDARY_COV = WL.CovSpec(WL.EXPONENTIAL, (20.0, 20.0, 5.0), (10.0, 0.0, 0.0), 1.5, 0.1)


def cok_inputs(g, mark, secondary=None):
    """Inputs of a cokriging golden case from its base fixture: the primary
    data, a secondary field (from the fixture when given, else made: 0.6 times
    the primary values plus seeded noise, informed on half of the cells) and
    the parameters (primary mean of the data, secondary mean of the field)."""
    dims, pdata, pmask = grid_inputs(g)
    n = len(pdata)
    if secondary is None:
        rng = np.random.default_rng(4)
        sdata = (0.6 * np.where(pmask == 1, pdata, 0) + rng.normal(size=n)).astype(np.float32)
        smask = (rng.random(n) < 0.5).astype(np.uint8)
    else:
        sdata, smask = secondary
    cov, rad, k = cov_of(g)
    return {"dims": dims, "pdata": pdata, "pmask": pmask, "sdata": sdata, "smask": smask, "cov": cov, "rad": rad,
            "k": k, "pm": float(pdata[pmask == 1].astype(np.float64).mean()),
            "sm": float(sdata[smask == 1].astype(np.float64).mean()), "sv": 0.9, "corr": 0.6,
            "cov2": COK_SECONDARY_COV if mark == 2 else None}


SIS_CASES = [
    # name, options: seed, categories (5 = the fixture's, 2 = median SIS on category >= 2), mask, LVM,
    # correlogram weights (LVM)
    ("sis5", {"seed": 17}),
    ("sis5_mask", {"seed": 5, "sim_mask": 0.6}),
    ("sis2_median", {"seed": 9, "two": True}),
    ("sis5_lvm", {"seed": 23, "lvm": True}),
    ("sis5_lvm_corr", {"seed": 31, "lvm": True, "corr": True}),
]


def sis_inputs(g, opts):
    """Inputs of a SIS golden case from the indicator fixture: its categories,
    per-category models, radiuses and marginals (k = 12 per category); a
    seeded simulation mask; LVM means from a smooth trend per category."""
    dims, data, mask = grid_inputs(g, dtype=np.uint8)
    n = len(data)
    data = np.where(mask == 1, data, 0).astype(np.uint8)
    covs, rads = [], []
    for c in range(5):
        cov, rad, _ = cov_of(g, f"c{c}_")
        covs.append(cov)
        rads.append(rad)
    marg = [float(v) for v in g["marginals"]]
    if opts.get("two"):
        data = (data >= 2).astype(np.uint8) * mask
        covs, rads = covs[2:4], rads[2:4]
        marg = [0.6, 0.4]
    ks = [12] * len(covs)
    x = {"dims": dims, "data": data, "mask": mask.copy(), "covs": covs, "rads": rads, "ks": ks, "marginals": marg,
         "seed": opts["seed"], "sim_mask": None, "means": None, "corr": bool(opts.get("corr"))}
    if "sim_mask" in opts:
        x["sim_mask"] = (np.random.default_rng(6).random(n) < opts["sim_mask"]).astype(np.uint8)
    if opts.get("lvm"):
        t = WL.lvm_means(dims)
        t = (t - t.min()) / max(float(t.max() - t.min()), 1e-6)
        base = np.array(marg, np.float64)
        x["means"] = [((0.5 * base[c] + 0.5 * base[c] * (0.5 + t)) / 1.0).astype(np.float32) for c in range(5)]
    return x
