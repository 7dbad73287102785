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
