"""Generates tests/golden/*.npz from the reference itself.

Run here, where the reference sources are present and oracle/Makefile has built
oracle/_ref/ (the reference's unmodified library, libhpgl.so, and the white-box
harness libref_harness.so around its own templates):

    make -C oracle REF=<reference checkout> && python tests/golden/make_golden.py   (all fixtures)
                      python tests/golden/make_golden.py lvm    (lvm.npz only)
                      python tests/golden/make_golden.py sgs    (sgs.npz only)
                      python tests/golden/make_golden.py cok    (cok.npz only)
                      python tests/golden/make_golden.py sis    (sis.npz only)

Inputs are the seeded workloads of geo_bsd.workloads at reduced scale (the
conditioning cells are stored in each file, so the fixtures do not depend on
the generator). Outputs per sampled node: the reference's neighbour indices in
its own order, the search path taken, the FP64 estimate and variance of
kriging_interpolation with result_t = double, the float estimate the drivers
store, and the status code. Whole-grid outputs of the reference's public C API
(hpgl_ordinary_kriging, hpgl_simple_kriging, hpgl_lvm_kriging,
hpgl_indicator_kriging, hpgl_median_ik, hpgl_sgs_simulation,
hpgl_sgs_lvm_simulation, hpgl_simple_cokriging_mark1/2, hpgl_sis_simulation(_lvm)) are stored for the small grids, plus the known-answer cases
of the reference's test suite (constant field 42, all zeros).
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "hpgl-reborn_b200"))

import oracle as O  # noqa: E402
sys.path.insert(0, os.path.dirname(HERE))
from golden_io import COK_CASES, SGS_CASES, SIS_CASES, cok_inputs, sgs_inputs, sis_inputs  # noqa: E402
from geo_bsd import workloads as WL  # noqa: E402  (pure python module)

SAMPLE = 1200


def _api():
    lib = C.CDLL(O.REF_API_PATH)
    sink = C.CFUNCTYPE(C.c_int, C.c_char_p, C.c_void_p)(lambda s, p: 0)
    psink = C.CFUNCTYPE(C.c_int, C.c_char_p, C.c_int, C.c_void_p)(lambda s, q, p: 0)
    lib.hpgl_set_output_handler(sink, None)
    lib.hpgl_set_progress_handler(psink, None)
    lib._keep = (sink, psink)
    return lib


class Shape(C.Structure):
    _fields_ = [("data", C.c_int * 3), ("strides", C.c_int * 3)]


class Cont(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("mask", C.POINTER(C.c_ubyte)), ("shape", Shape)]


class Ind(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_ubyte)), ("mask", C.POINTER(C.c_ubyte)), ("shape", Shape),
                ("indicator_count", C.c_int)]


class OkP(C.Structure):
    _fields_ = [("t", C.c_int), ("r", C.c_double * 3), ("a", C.c_double * 3), ("sill", C.c_double),
                ("nugget", C.c_double), ("rad", C.c_int * 3), ("k", C.c_int)]


class SkP(C.Structure):
    _fields_ = OkP._fields_ + [("auto", C.c_ubyte), ("mean", C.c_double)]


class IkP(C.Structure):
    _fields_ = OkP._fields_ + [("marginal", C.c_double)]


class MikP(C.Structure):
    _fields_ = OkP._fields_ + [("marginals", C.c_double * 2)]


def _shape(dims):
    return Shape((C.c_int * 3)(*dims), (C.c_int * 3)(1, dims[0], dims[0] * dims[1]))


def api_cont(lib, kind, dims, data, mask, cov, rad, k, mean=None):
    data = np.ascontiguousarray(data, np.float32)
    mask = np.ascontiguousarray(mask, np.uint8)
    od, om = data.copy(), mask.copy()
    fp = C.POINTER(C.c_float)
    up = C.POINTER(C.c_ubyte)
    if kind == 0:
        p = OkP(cov.cov_type, (C.c_double * 3)(*cov.ranges), (C.c_double * 3)(*cov.angles), cov.sill, cov.nugget,
                (C.c_int * 3)(*rad), k)
        a = Cont(data.ctypes.data_as(fp), mask.ctypes.data_as(up), _shape(dims))
        b = Cont(od.ctypes.data_as(fp), om.ctypes.data_as(up), _shape(dims))
        lib.hpgl_ordinary_kriging(C.byref(a), C.byref(p), C.byref(b))
    else:
        p = SkP(cov.cov_type, (C.c_double * 3)(*cov.ranges), (C.c_double * 3)(*cov.angles), cov.sill, cov.nugget,
                (C.c_int * 3)(*rad), k, 1 if mean is None else 0, 0.0 if mean is None else mean)
        sh = _shape(dims)
        lib.hpgl_simple_kriging(data.ctypes.data_as(fp), mask.ctypes.data_as(up), C.byref(sh), C.byref(p),
                                od.ctypes.data_as(fp), om.ctypes.data_as(up), C.byref(sh))
    return od, om


def api_lvm(lib, dims, data, mask, means, cov, rad, k):
    data = np.ascontiguousarray(data, np.float32)
    mask = np.ascontiguousarray(mask, np.uint8)
    means = np.ascontiguousarray(means, np.float32)
    od, om = data.copy(), mask.copy()
    fp = C.POINTER(C.c_float)
    up = C.POINTER(C.c_ubyte)
    p = OkP(cov.cov_type, (C.c_double * 3)(*cov.ranges), (C.c_double * 3)(*cov.angles), cov.sill, cov.nugget,
            (C.c_int * 3)(*rad), k)
    sh = _shape(dims)
    lib.hpgl_lvm_kriging(data.ctypes.data_as(fp), mask.ctypes.data_as(up), C.byref(sh), means.ctypes.data_as(fp),
                         C.byref(sh), C.byref(p), od.ctypes.data_as(fp), om.ctypes.data_as(up), C.byref(sh))
    return od, om


class SgsP(C.Structure):
    _fields_ = [("t", C.c_int), ("r", C.c_double * 3), ("a", C.c_double * 3), ("sill", C.c_double),
                ("nugget", C.c_double), ("rad", C.c_int * 3), ("k", C.c_int), ("kind", C.c_int), ("seed", C.c_long),
                ("kmin", C.c_int)]


class NpCdf(C.Structure):
    _fields_ = [("values", C.POINTER(C.c_float)), ("probs", C.POINTER(C.c_float)), ("size", C.c_longlong)]


class FloatArr(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_float)), ("shape", Shape)]


class UbyteArr(C.Structure):
    _fields_ = [("data", C.POINTER(C.c_ubyte)), ("shape", Shape)]


def api_sgs(lib, dims, data, mask, cov, rad, k, seed, kind=1, sim_mask=None, cdf=None, means=None):
    """The reference's hpgl_sgs_simulation / hpgl_sgs_lvm_simulation; `cov` holds the
    sill and nugget as the driver receives them. Returns the output data and mask."""
    od = np.ascontiguousarray(data, np.float32).copy()
    om = np.ascontiguousarray(mask, np.uint8).copy()
    fp = C.POINTER(C.c_float)
    up = C.POINTER(C.c_ubyte)
    a = Cont(od.ctypes.data_as(fp), om.ctypes.data_as(up), _shape(dims))
    p = SgsP(cov.cov_type, (C.c_double * 3)(*cov.ranges), (C.c_double * 3)(*cov.angles), cov.sill, cov.nugget,
             (C.c_int * 3)(*rad), k, kind, seed, 0)
    keep = []
    c = None
    if cdf is not None:
        cv = np.ascontiguousarray(cdf[0], np.float32)
        cp = np.ascontiguousarray(cdf[1], np.float32)
        keep += [cv, cp]
        c = C.byref(NpCdf(cv.ctypes.data_as(fp), cp.ctypes.data_as(fp), len(cv)))
    sm = None
    if sim_mask is not None:
        smv = np.ascontiguousarray(sim_mask, np.uint8)
        keep.append(smv)
        sm = C.byref(UbyteArr(smv.ctypes.data_as(up), _shape(dims)))
    if means is None:
        lib.hpgl_sgs_simulation(C.byref(a), C.byref(p), c, None, sm)
    else:
        mv = np.ascontiguousarray(means, np.float32)
        keep.append(mv)
        lib.hpgl_sgs_lvm_simulation(C.byref(a), C.byref(p), c, C.byref(FloatArr(mv.ctypes.data_as(fp), _shape(dims))),
                                    sm)
    return od, om


class CovP(C.Structure):
    _fields_ = [("t", C.c_int), ("r", C.c_double * 3), ("a", C.c_double * 3), ("sill", C.c_double),
                ("nugget", C.c_double)]


class Cok1P(C.Structure):
    _fields_ = [("t", C.c_int), ("r", C.c_double * 3), ("a", C.c_double * 3), ("sill", C.c_double),
                ("nugget", C.c_double), ("rad", C.c_int * 3), ("k", C.c_int), ("pm", C.c_double), ("sm", C.c_double),
                ("sv", C.c_double), ("corr", C.c_double)]


class Cok2P(C.Structure):
    _fields_ = [("pc", CovP), ("sc", CovP), ("rad", C.c_int * 3), ("k", C.c_int), ("pm", C.c_double),
                ("sm", C.c_double), ("corr", C.c_double)]


def _covp(c):
    return CovP(c.cov_type, (C.c_double * 3)(*c.ranges), (C.c_double * 3)(*c.angles), c.sill, c.nugget)


def api_cokriging(lib, mark, dims, pdata, pmask, sdata, smask, cov, rad, k, pm, sm, sv=0.0, corr=0.0, cov2=None):
    """The reference's hpgl_simple_cokriging_mark1 / _mark2; returns the output data and mask."""
    fp = C.POINTER(C.c_float)
    up = C.POINTER(C.c_ubyte)
    pd = np.ascontiguousarray(pdata, np.float32)
    pmk = np.ascontiguousarray(pmask, np.uint8)
    sd = np.ascontiguousarray(sdata, np.float32)
    smk = np.ascontiguousarray(smask, np.uint8)
    od = np.zeros_like(pd)
    om = np.zeros_like(pmk)
    a = Cont(pd.ctypes.data_as(fp), pmk.ctypes.data_as(up), _shape(dims))
    b = Cont(sd.ctypes.data_as(fp), smk.ctypes.data_as(up), _shape(dims))
    o = Cont(od.ctypes.data_as(fp), om.ctypes.data_as(up), _shape(dims))
    if mark == 1:
        p = Cok1P(cov.cov_type, (C.c_double * 3)(*cov.ranges), (C.c_double * 3)(*cov.angles), cov.sill, cov.nugget,
                  (C.c_int * 3)(*rad), k, pm, sm, sv, corr)
        lib.hpgl_simple_cokriging_mark1(C.byref(a), C.byref(b), C.byref(p), C.byref(o))
    else:
        p = Cok2P(_covp(cov), _covp(cov2), (C.c_int * 3)(*rad), k, pm, sm, corr)
        lib.hpgl_simple_cokriging_mark2(C.byref(a), C.byref(b), C.byref(p), C.byref(o))
    return od, om


def api_sis(lib, dims, data, mask, covs, rads, ks, marginals, seed, sim_mask=None, means=None, corr=False):
    """The reference's hpgl_sis_simulation / hpgl_sis_simulation_lvm (correlogram
    weights with `corr`); returns the output data and mask."""
    od = np.ascontiguousarray(data, np.uint8).copy()
    om = np.ascontiguousarray(mask, np.uint8).copy()
    up = C.POINTER(C.c_ubyte)
    m = len(covs)
    arr = (IkP * m)()
    for i, c in enumerate(covs):
        arr[i] = IkP(c.cov_type, (C.c_double * 3)(*c.ranges), (C.c_double * 3)(*c.angles), c.sill, c.nugget,
                     (C.c_int * 3)(*rads[i]), ks[i], marginals[i])
    a = Ind(od.ctypes.data_as(up), om.ctypes.data_as(up), _shape(dims), m)
    keep = []
    sm = None
    if sim_mask is not None:
        smv = np.ascontiguousarray(sim_mask, np.uint8)
        keep.append(smv)
        sm = C.byref(UbyteArr(smv.ctypes.data_as(up), _shape(dims)))
    if means is None:
        lib.hpgl_sis_simulation(C.byref(a), arr, m, seed, sm)
    else:
        fa = (FloatArr * m)()
        for i, mv in enumerate(means):
            mv = np.ascontiguousarray(mv, np.float32)
            keep.append(mv)
            fa[i] = FloatArr(mv.ctypes.data_as(C.POINTER(C.c_float)), _shape(dims))
        lib.hpgl_sis_simulation_lvm(C.byref(a), arr, fa, m, seed, sm, int(bool(corr)))
    return od, om


def api_ik(lib, dims, data, mask, covs, rads, ks, marginals):
    data = np.ascontiguousarray(data, np.uint8)
    mask = np.ascontiguousarray(mask, np.uint8)
    od, om = data.copy(), mask.copy()
    up = C.POINTER(C.c_ubyte)
    m = len(covs)
    arr = (IkP * m)()
    for i, c in enumerate(covs):
        arr[i] = IkP(c.cov_type, (C.c_double * 3)(*c.ranges), (C.c_double * 3)(*c.angles), c.sill, c.nugget,
                     (C.c_int * 3)(*rads[i]), ks[i], marginals[i])
    a = Ind(data.ctypes.data_as(up), mask.ctypes.data_as(up), _shape(dims), m)
    b = Ind(od.ctypes.data_as(up), om.ctypes.data_as(up), _shape(dims), m)
    lib.hpgl_indicator_kriging(C.byref(a), C.byref(b), arr, m)
    return od, om


def api_mik(lib, dims, data, mask, cov, rad, k, mp):
    data = np.ascontiguousarray(data, np.uint8)
    mask = np.ascontiguousarray(mask, np.uint8)
    od, om = data.copy(), mask.copy()
    up = C.POINTER(C.c_ubyte)
    p = MikP(cov.cov_type, (C.c_double * 3)(*cov.ranges), (C.c_double * 3)(*cov.angles), cov.sill, cov.nugget,
             (C.c_int * 3)(*rad), k, (C.c_double * 2)(*mp))
    a = Ind(data.ctypes.data_as(up), mask.ctypes.data_as(up), _shape(dims), 2)
    b = Ind(od.ctypes.data_as(up), om.ctypes.data_as(up), _shape(dims), 2)
    lib.hpgl_median_ik(C.byref(a), C.byref(p), C.byref(b))
    return od, om


def cov_fields(prefix, cov, rad, k):
    return {f"{prefix}cov_type": cov.cov_type, f"{prefix}ranges": np.array(cov.ranges),
            f"{prefix}angles": np.array(cov.angles), f"{prefix}sill": cov.sill, f"{prefix}nugget": cov.nugget,
            f"{prefix}radiuses": np.array(rad, np.int32), f"{prefix}k": k}


def cont_case(lib, wl, name, kinds=(0, 1), sample=SAMPLE, grid_api=False):
    rng = np.random.default_rng(7)
    unk = np.flatnonzero(wl.mask == 0)
    nodes = np.sort(rng.choice(unk, min(sample, len(unk)), replace=False)).astype(np.int32)
    informed = np.flatnonzero(wl.mask == 1).astype(np.int32)
    out = {"dims": np.array(wl.dims, np.int32), "informed": informed, "values": wl.data[informed],
           "nodes": nodes, **cov_fields("", wl.cov, wl.radiuses, wl.max_neighbours)}
    mean = float(wl.data[informed].astype(np.float64).mean())
    out["sk_mean"] = mean
    for kind in kinds:
        r = O.krige_nodes("ref", kind, wl.dims, wl.data, wl.mask, wl.cov, wl.radiuses, wl.max_neighbours,
                          mean=mean, nodes=nodes, threads=8)
        tag = "ok" if kind == 0 else "sk"
        for key in ("idx", "count", "path", "est", "var", "est_f", "status"):
            out[f"{tag}_{key}"] = r[key]
        if grid_api:
            od, om = api_cont(lib, kind, wl.dims, wl.data, wl.mask, wl.cov, wl.radiuses, wl.max_neighbours,
                              mean=None)
            out[f"{tag}_grid_data"] = od
            out[f"{tag}_grid_mask"] = om
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("wrote", name, {k: v.shape for k, v in out.items() if hasattr(v, "shape") and v.size > 3})


def lvm_cases(lib):
    """LVM kriging on the small grids with a smooth trend as the mean: the whole
    grid through hpgl_lvm_kriging and per-node results of the reference's
    templates instantiated as lvm_kriging does; the inputs are those of the
    OK/SK fixtures of the same names."""
    out = {}
    for name, wl in (("ok_small_s030", WL.ok_small(0.3)), ("gauss_cv_s020", WL.gauss_cv(0.2))):
        m = WL.lvm_means(wl.dims)
        od, om = api_lvm(lib, wl.dims, wl.data, wl.mask, m, wl.cov, wl.radiuses, wl.max_neighbours)
        out[f"{name}_means"] = m
        out[f"{name}_grid_data"] = od
        out[f"{name}_grid_mask"] = om
        rng = np.random.default_rng(7)
        unk = np.flatnonzero(wl.mask == 0)
        nodes = np.sort(rng.choice(unk, min(SAMPLE, len(unk)), replace=False)).astype(np.int32)
        r = O.krige_nodes("ref", 1, wl.dims, wl.data, wl.mask, wl.cov, wl.radiuses, wl.max_neighbours, nodes=nodes,
                          threads=8, means=m)
        out[f"{name}_nodes"] = nodes
        for key in ("idx", "count", "path", "est", "var", "est_f", "status"):
            out[f"{name}_{key}"] = r[key]
    np.savez_compressed(os.path.join(HERE, "lvm.npz"), **out)
    print("wrote lvm")


def sgs_cases(lib):
    """The reference's hpgl_sgs_simulation / hpgl_sgs_lvm_simulation outputs."""
    out = {}
    for name, base, kind, seed, opts in SGS_CASES:
        g = dict(np.load(os.path.join(HERE, base + ".npz")))
        x = sgs_inputs(g, opts)
        od, om = api_sgs(lib, x["dims"], x["data"], x["mask"], x["cov"], x["rad"], x["k"], seed, kind=kind,
                         sim_mask=x["sim_mask"], cdf=x["cdf"], means=x["means"])
        out[f"{name}_data"] = od
        out[f"{name}_mask"] = om
    np.savez_compressed(os.path.join(HERE, "sgs.npz"), **out)
    print("wrote sgs")


def cok_cases(lib):
    """The reference's hpgl_simple_cokriging_mark1 / _mark2 outputs, with the
    secondary fields they were given."""
    out = {}
    for name, base, mark in COK_CASES:
        g = dict(np.load(os.path.join(HERE, base + ".npz")))
        x = cok_inputs(g, mark)
        od, om = api_cokriging(lib, mark, x["dims"], x["pdata"], x["pmask"], x["sdata"], x["smask"], x["cov"],
                               x["rad"], x["k"], x["pm"], x["sm"], sv=x["sv"], corr=x["corr"], cov2=x["cov2"])
        out[f"{base}_sdata"] = x["sdata"]
        out[f"{base}_smask"] = x["smask"]
        out[f"{name}_data"] = od
        out[f"{name}_mask"] = om
    np.savez_compressed(os.path.join(HERE, "cok.npz"), **out)
    print("wrote cok")


def sis_cases(lib):
    """The reference's SIS outputs (inputs: the indicator fixture; see golden_io.sis_inputs)."""
    out = {}
    for name, opts in SIS_CASES:
        x = sis_inputs(dict(np.load(os.path.join(HERE, "indicator_s015.npz"))), opts)
        od, om = api_sis(lib, x["dims"], x["data"], x["mask"], x["covs"], x["rads"], x["ks"], x["marginals"],
                         x["seed"], sim_mask=x["sim_mask"], means=x["means"], corr=x["corr"])
        out[f"{name}_data"] = od
        out[f"{name}_mask"] = om
    np.savez_compressed(os.path.join(HERE, "sis.npz"), **out)
    print("wrote sis")


def main(only=None):
    lib = _api()
    if only == "sis":
        sis_cases(lib)
        return
    if only == "cok":
        cok_cases(lib)
        return
    if only == "lvm":
        lvm_cases(lib)
        return
    if only == "sgs":
        sgs_cases(lib)
        return
    lvm_cases(lib)
    sgs_cases(lib)
    cok_cases(lib)
    sis_cases(lib)
    cont_case(lib, WL.ok_small(0.3), "ok_small_s030", grid_api=True)
    cont_case(lib, WL.sk_ok_large(0.16), "sk_ok_large_s016")
    cont_case(lib, WL.gauss_cv(0.2), "gauss_cv_s020", grid_api=True)
    cont_case(lib, WL.clustered(0.1), "clustered_s010")

    # indicator: per-category SK probabilities (reference float results) and the
    # public API's full IK / median IK outputs on the whole small grid
    wl = WL.indicator(0.15)
    rng = np.random.default_rng(11)
    nodes = np.sort(rng.choice(wl.n_cells, min(SAMPLE, wl.n_cells), replace=False)).astype(np.int32)
    informed = np.flatnonzero(wl.mask == 1).astype(np.int32)
    out = {"dims": np.array(wl.dims, np.int32), "informed": informed, "values": wl.data[informed], "nodes": nodes,
           "marginals": np.array(wl.marginals)}
    ks = [wl.max_neighbours] * 5
    for c in range(5):
        out.update(cov_fields(f"c{c}_", wl.cat_covs[c], wl.cat_radiuses[c], ks[c]))
        r = O.krige_nodes("ref", 1, wl.dims, wl.data, wl.mask, wl.cat_covs[c], wl.cat_radiuses[c], ks[c],
                          mean=float(np.float32(wl.marginals[c])), nodes=nodes, ind_value=c, threads=8)
        for key in ("idx", "count", "path", "est_f", "status"):
            out[f"c{c}_{key}"] = r[key]
    od, om = api_ik(lib, wl.dims, wl.data, wl.mask, wl.cat_covs, wl.cat_radiuses, ks, wl.marginals)
    out["ik_grid"] = od
    mik_data = (wl.data >= 2).astype(np.uint8)
    out["mik_values"] = mik_data[informed]
    mp = (0.6, 0.4)
    od, om = api_mik(lib, wl.dims, mik_data, wl.mask, wl.cat_covs[2], wl.cat_radiuses[2], 24, mp)
    out["mik_grid"] = od
    out["mik_marginals"] = np.array(mp)
    np.savez_compressed(os.path.join(HERE, "indicator_s015.npz"), **out)
    print("wrote indicator_s015")

    # known answers pinned by the reference's tests (test_edge_cases.py:368-392, :487-511)
    kat = {}
    dims = (10, 10, 5)
    n = 500
    rng = np.random.default_rng(3)
    idx = rng.choice(n, 60, replace=False)
    for name, val in (("const42", 42.0), ("zeros", 0.0)):
        data = np.full(n, -99.0, np.float32)
        mask = np.zeros(n, np.uint8)
        data[idx] = val
        mask[idx] = 1
        cov = WL.CovSpec(WL.SPHERICAL, (10.0, 10.0, 10.0), (0.0, 0.0, 0.0), 1.0, 0.0)
        od, om = api_cont(lib, 0, dims, data, mask, cov, (5, 5, 5), 12)
        kat[f"{name}_data"] = data
        kat[f"{name}_mask"] = mask
        kat[f"{name}_out"] = od
        kat[f"{name}_outmask"] = om
    np.savez_compressed(os.path.join(HERE, "known_answers.npz"), **kat)
    print("wrote known_answers")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
