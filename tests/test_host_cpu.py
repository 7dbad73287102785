"""Host-side pieces of the engine, runnable without a GPU: the C ABI library
loads and exports every entry point of include/hpgl_b200.h, its struct layouts
agree with the header, and its covariance / template / transform code is
bit-identical to the oracle (and so to the reference)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import oracle as O
from geo_bsd import hpgl_wrap as W
from geo_bsd import workloads as WL

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hpgl_b200.h")

MODELS = [
    WL.CovSpec(WL.SPHERICAL, (10.0, 10.0, 5.0), (0.0, 0.0, 0.0), 1.0, 0.1),
    WL.CovSpec(WL.EXPONENTIAL, (30.0, 15.0, 6.0), (30.0, 0.0, 0.0), 1.0, 0.05),
    WL.CovSpec(WL.GAUSSIAN, (18.0, 18.0, 6.0), (0.0, 0.0, 0.0), 1.0, 0.05),
    WL.CovSpec(WL.GAUSSIAN, (12.0, 7.0, 3.0), (45.0, 10.0, 5.0), 2.5, 0.3),
    WL.CovSpec(WL.SPHERICAL, (8.0, 5.0, 4.0), (120.0, 30.0, 60.0), 1.0, 0.0),
]
RADII = [(10, 10, 5), (30, 15, 6), (18, 18, 6), (9, 6, 3), (6, 4, 3)]


def header_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(hpgl_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_header_function():
    names = header_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(W._hpgl_so, name), name
    assert set(W.EXPORTS) <= set(names)


def test_struct_layouts_match_header():
    fields = {
        "hpgl_shape_t": (W._HPGL_SHAPE, ["m_data", "m_strides"]),
        "hpgl_cont_masked_array_t": (W._HPGL_CONT_MASKED_ARRAY, ["m_data", "m_mask", "m_shape"]),
        "hpgl_ind_masked_array_t": (W._HPGL_IND_MASKED_ARRAY, ["m_data", "m_mask", "m_shape", "m_indicator_count"]),
        "hpgl_ok_params_t": (W._HPGL_OK_PARAMS, ["m_covariance_type", "m_ranges", "m_angles", "m_sill", "m_nugget",
                                                 "m_radiuses", "m_max_neighbours"]),
        "hpgl_sk_params_t": (W._HPGL_SK_PARAMS, ["m_covariance_type", "m_ranges", "m_angles", "m_sill", "m_nugget",
                                                 "m_radiuses", "m_max_neighbours", "m_automatic_mean", "m_mean"]),
        "hpgl_cov_params_t": (W._HPGL_COV_PARAMS, ["m_covariance_type", "m_ranges", "m_angles", "m_sill",
                                                   "m_nugget"]),
        "hpgl_median_ik_params_t": (W._HPGL_MEDIAN_IK_PARAMS, ["m_covariance_type", "m_ranges", "m_angles", "m_sill",
                                                               "m_nugget", "m_radiuses", "m_max_neighbours",
                                                               "m_marginal_probs"]),
        "hpgl_ik_params_t": (W._HPGL_IK_PARAMS, ["m_covariance_type", "m_ranges", "m_angles", "m_sill", "m_nugget",
                                                 "m_radiuses", "m_max_neighbours", "m_marginal_prob"]),
        "hpgl_b200_options_t": (W._HPGL_B200_OPTIONS, ["precision", "refine_steps", "flags", "stream", "estimate64",
                                                       "variance", "status", "ik_probs", "tolerance"]),
        "hpgl_float_array_t": (W._HPGL_FLOAT_ARRAY, ["m_data", "m_shape"]),
        "hpgl_ubyte_array_t": (W._HPGL_UBYTE_ARRAY, ["m_data", "m_shape"]),
        "hpgl_sgs_params_t": (W._HPGL_SGS_PARAMS, ["m_covariance_type", "m_ranges", "m_angles", "m_sill", "m_nugget",
                                                   "m_radiuses", "m_max_neighbours", "m_kriging_kind", "m_seed",
                                                   "m_min_neighbours"]),
        "hpgl_non_parametric_cdf_t": (W._HPGL_NON_PARAMETRIC_CDF, ["m_values", "m_probs", "m_size"]),
        "hpgl_cokriging_m1_params_t": (W._HPGL_COK_M1_PARAMS, ["m_covariance_type", "m_ranges", "m_angles", "m_sill",
                                                             "m_nugget", "m_radiuses", "m_max_neighbours",
                                                             "m_primary_mean", "m_secondary_mean",
                                                             "m_secondary_variance", "m_correlation_coef"]),
        "hpgl_cokriging_m2_params_t": (W._HPGL_COK_M2_PARAMS, ["m_primary_cov_params", "m_secondary_cov_params",
                                                             "m_radiuses", "m_max_neighbours", "m_primary_mean",
                                                             "m_secondary_mean", "m_correlation_coef"]),
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for s, (_, fl) in fields.items():
        lines.append(f'printf("{s} %zu\\n", sizeof(struct {s}));')
        for f in fl:
            lines.append(f'printf("{s}.{f} %zu\\n", offsetof(struct {s}, {f}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["/usr/bin/gcc", src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(l.split() for l in out if l.strip())
    for s, (ct, fl) in fields.items():
        assert int(got[s]) == C.sizeof(ct), s
        for f, (cname, _) in zip(fl, ct._fields_):
            assert int(got[f"{s}.{f}"]) == getattr(ct, cname).offset, f"{s}.{f}"


def _covp(cov):
    return W._HPGL_COV_PARAMS(covariance_type=cov.cov_type, ranges=cov.ranges, angles=cov.angles, sill=cov.sill,
                              nugget=cov.nugget)


@pytest.mark.parametrize("mi", range(len(MODELS)))
def test_transform_template_and_covariance_bit_identical(mi):
    cov, rad = MODELS[mi], RADII[mi]
    lib = W._hpgl_so
    t = (C.c_double * 9)()
    assert lib.hpgl_b200_transform((C.c_double * 3)(*cov.ranges), (C.c_double * 3)(*cov.angles), t) == 0
    np.testing.assert_array_equal(np.array(list(t)), O.transform("port", cov.ranges, cov.angles))
    cap = (2 * rad[0] + 1) * (2 * rad[1] + 1) * (2 * rad[2] + 1)
    # the key table behind the template is built by a team of host threads (the
    # first half of the block evaluated, the mirrors copied): the same at any size
    saved = lib.hpgl_get_thread_num()
    try:
        for threads in (1, 3, 16):
            lib.hpgl_set_thread_num(threads)
            for kind in (0, 1):
                out = np.zeros((cap, 3), np.int32)
                lim = C.c_int(0)
                n = lib.hpgl_b200_template(kind, C.byref(_covp(cov)), (C.c_int * 3)(*rad), out.ctypes.data, cap,
                                           C.byref(lim))
                ref, rlim = O.template("port", kind, cov, rad)
                assert n == len(ref) and lim.value == rlim
                np.testing.assert_array_equal(out[:n], ref)
    finally:
        lib.hpgl_set_thread_num(saved)
    rng = np.random.default_rng(mi)
    for _ in range(300):
        a = rng.integers(0, 60, 3).astype(np.int32)
        b = (a + rng.integers(-2 * max(rad), 2 * max(rad) + 1, 3)).astype(np.int32)
        for kind in (0, 1):
            v = lib.hpgl_b200_covariance(kind, C.byref(_covp(cov)), (C.c_int * 3)(*rad), (C.c_int * 3)(*a),
                                         (C.c_int * 3)(*b))
            assert v == O.cov_point("port", kind, cov, rad, a, b)


def _template(lib, mi, kind=0):
    cov, rad = MODELS[mi], RADII[mi]
    cap = (2 * rad[0] + 1) * (2 * rad[1] + 1) * (2 * rad[2] + 1)
    out = np.zeros((cap, 3), np.int32)
    lim = C.c_int(0)
    n = lib.hpgl_b200_template(kind, C.byref(_covp(cov)), (C.c_int * 3)(*rad), out.ctypes.data, cap, C.byref(lim))
    return out[:n].copy(), lim.value


@pytest.mark.timeout(300)
def test_key_tables_built_from_several_threads_at_once():
    """The key table's host workers serve one build at a time; builds that find
    them busy start threads of their own. Concurrent builds from six Python
    threads (ctypes calls release the GIL) all equal the oracle's template."""
    import threading

    lib = W._hpgl_so
    want = {mi: O.template("port", 0, MODELS[mi], RADII[mi]) for mi in range(len(MODELS))}
    errors = []

    def worker(seed):
        rng = np.random.default_rng(seed)
        for mi in rng.integers(0, len(MODELS), 8):
            got, lim = _template(lib, int(mi))
            ref, rlim = want[int(mi)]
            if lim != rlim or not np.array_equal(got, ref):
                errors.append(int(mi))

    saved = lib.hpgl_get_thread_num()
    lib.hpgl_set_thread_num(4)
    try:
        ts = [threading.Thread(target=worker, args=(s,)) for s in range(6)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
    finally:
        lib.hpgl_set_thread_num(saved)
    assert not errors, errors


@pytest.mark.timeout(300)
@pytest.mark.filterwarnings("ignore:This process .* is multi-threaded:DeprecationWarning")
def test_key_table_in_a_forked_child():
    """A child forked after the workers started builds with workers of its own
    (the library's own locks are free at the fork; the wait for the child is
    bounded all the same)."""
    import time

    lib = W._hpgl_so
    ref, rlim = O.template("port", 0, MODELS[1], RADII[1])
    got, lim = _template(lib, 1)  # the workers exist in this process now
    assert lim == rlim and np.array_equal(got, ref)
    pid = os.fork()
    if pid == 0:
        code = 1
        try:
            g, l = _template(lib, 1)
            code = 0 if (l == rlim and np.array_equal(g, ref)) else 2
        finally:
            os._exit(code)
    deadline = time.time() + 120
    status = None
    while time.time() < deadline:
        done, status = os.waitpid(pid, os.WNOHANG)
        if done:
            break
        time.sleep(0.05)
    else:
        os.kill(pid, 9)
        os.waitpid(pid, 0)
        pytest.fail("the forked child did not finish its key table")
    assert os.WIFEXITED(status) and os.WEXITSTATUS(status) == 0, status


def test_zero_range_is_an_error_not_an_abort():
    lib = W._hpgl_so
    out = (C.c_double * 9)()
    assert lib.hpgl_b200_transform((C.c_double * 3)(10, 0, 5), (C.c_double * 3)(0, 0, 0), out) != 0
    assert "non-zero" in W.last_error()


def test_kriging_without_gpu_reports_an_error():
    """On a machine without a usable GPU the C ABI returns an error code (never a CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    wl = WL.ok_small(0.2)
    dims = (C.c_int * 3)(*wl.dims)
    p = W._HPGL_SK_PARAMS(covariance_type=0, ranges=wl.cov.ranges, angles=wl.cov.angles, sill=1.0, nugget=0.1,
                          radiuses=wl.radiuses, max_neighbours=12, automatic_mean=1, mean=0.0)
    out = wl.data.copy()
    om = wl.mask.copy()
    rc = W._hpgl_so.hpgl_b200_cont_kriging_ex(0, dims, wl.data.ctypes.data, wl.mask.ctypes.data, C.byref(p),
                                              out.ctypes.data, om.ctypes.data, None)
    assert rc == -2
    np.testing.assert_array_equal(out, wl.data)


def test_lvm_entry_argument_checks():
    """LVM: a missing mean array is EINVAL before any device work; without a GPU the
    call returns ECUDA and leaves the output untouched."""
    wl = WL.ok_small(0.2)
    dims = (C.c_int * 3)(*wl.dims)
    p = W._HPGL_OK_PARAMS(covariance_type=0, ranges=wl.cov.ranges, angles=wl.cov.angles, sill=1.0, nugget=0.1,
                          radiuses=wl.radiuses, max_neighbours=12)
    out = wl.data.copy()
    om = wl.mask.copy()
    fn = W._hpgl_so.hpgl_b200_lvm_kriging_ex
    assert fn(dims, wl.data.ctypes.data, wl.mask.ctypes.data, None, C.byref(p), out.ctypes.data, om.ctypes.data,
              None) == W.EINVAL
    import torch
    if torch.cuda.is_available():
        return
    means = WL.lvm_means(wl.dims)
    assert fn(dims, wl.data.ctypes.data, wl.mask.ctypes.data, means.ctypes.data, C.byref(p), out.ctypes.data,
              om.ctypes.data, None) == W.ECUDA
    np.testing.assert_array_equal(out, wl.data)


def test_sgs_entry_argument_checks():
    """SGS limits are checked before any device work: more than 10,000,000 cells
    and max_neighbours above 160 are ELIMIT, a seed with a negative remainder EINVAL."""
    dims = (C.c_int * 3)(2000, 2000, 3)
    p = W._HPGL_SGS_PARAMS(covariance_type=0, ranges=(10.0, 10.0, 10.0), angles=(0.0, 0.0, 0.0), sill=1.0,
                           nugget=0.0, radiuses=(5, 5, 5), max_neighbours=12, kriging_kind=1, seed=1,
                           min_neighbours=0)
    fn = W._hpgl_so.hpgl_b200_sgs_ex
    assert fn(dims, None, None, None, None, None, C.byref(p), None) == W.EINVAL  # null arrays
    d = np.zeros(8, np.float32)
    m = np.zeros(8, np.uint8)
    assert fn(dims, d.ctypes.data, m.ctypes.data, None, None, None, C.byref(p), None) == W.ELIMIT
    small = (C.c_int * 3)(2, 2, 2)
    p.max_neighbours = 161
    assert fn(small, d.ctypes.data, m.ctypes.data, None, None, None, C.byref(p), None) == W.ELIMIT
    p.max_neighbours = 12
    p.seed = -3
    assert fn(small, d.ctypes.data, m.ctypes.data, None, None, None, C.byref(p), None) == W.EINVAL
    assert "seed" in W.last_error()


def test_calc_cdf_matches_the_reference_loop():
    """calc_cdf against a loop restatement of cdf.py:8-40 (dict of counts, sorted
    keys without the largest, running sums)."""
    import geo_bsd
    rng = np.random.default_rng(2)
    data = np.round(rng.normal(size=(6, 5, 4)), 1).astype(np.float32)
    mask = (rng.random((6, 5, 4)) < 0.6).astype(np.uint8)
    got = geo_bsd.calc_cdf(geo_bsd.ContProperty(data, mask))
    counts, full = {}, 0
    for x in range(6):
        for y in range(5):
            for z in range(4):
                if mask[x, y, z]:
                    counts[data[x, y, z]] = counts.get(data[x, y, z], 0) + 1
                    full += 1
    values = np.sort(list(counts.keys()))[: len(counts) - 1]
    probs, last = np.zeros(values.shape), 0.0
    for i in range(values.size):
        probs[i] = last + counts[values[i]] / float(full)
        last = probs[i]
    np.testing.assert_array_equal(got.values, values.astype(np.float32))
    np.testing.assert_array_equal(got.probs, probs.astype(np.float32))


@pytest.mark.parametrize("seed", [0, 1, 42, 4357, 2**31 + 5, 2**32 + 7, -5])
def test_sgs_draws_equal_the_standard_library(seed):
    """The simulation's uniform draws (the engine's own MT19937 and canonical
    double) are bit-identical to std::mt19937 + std::uniform_real_distribution."""
    n = 5000
    got = np.zeros(n)
    assert W._hpgl_so.hpgl_b200_sgs_draws(seed, n, got.ctypes.data) == 0
    np.testing.assert_array_equal(got.view(np.uint64), O.mt_draws(seed, n).view(np.uint64))


def test_cokriging_entry_argument_checks():
    """A mark other than 1 or 2, or one without its parameters, is EINVAL before any device work."""
    fn = W._hpgl_so.hpgl_b200_cokriging_ex
    m1 = W._HPGL_COK_M1_PARAMS(covariance_type=0, ranges=(5.0, 5.0, 5.0), angles=(0.0, 0.0, 0.0), sill=1.0,
                               nugget=0.0, radiuses=(3, 3, 3), max_neighbours=8, primary_mean=0.0, secondary_mean=0.0,
                               secondary_variance=1.0, correlation_coef=0.5)
    dims = (C.c_int * 3)(2, 2, 2)
    assert fn(3, dims, None, None, None, None, C.byref(m1), None, None, None, None) == W.EINVAL
    assert fn(2, dims, None, None, None, None, C.byref(m1), None, None, None, None) == W.EINVAL
    assert fn(1, dims, None, None, None, None, C.byref(m1), None, None, None, None) == W.EINVAL  # null arrays



def _sis_params(m, k=8):
    arr = (W._HPGL_IK_PARAMS * m)()
    for i in range(m):
        arr[i] = W._HPGL_IK_PARAMS(covariance_type=0, ranges=(4.0, 4.0, 4.0), angles=(0.0, 0.0, 0.0), sill=1.0,
                                   nugget=0.1, radiuses=(3, 3, 3), max_neighbours=k, marginal_prob=1.0 / m)
    return arr


def test_sis_entry_argument_checks():
    """SIS limits are checked before any device work: null arrays and fewer than
    two categories are EINVAL, more than 16 categories, more than 32 neighbours
    and more than 10,000,000 cells ELIMIT, a walk that misses nodes EINVAL."""
    fn = W._hpgl_so.hpgl_b200_sis_ex
    dims = (C.c_int * 3)(6, 5, 4)
    d = np.zeros(120, np.uint8)
    m = np.zeros(120, np.uint8)
    assert fn(dims, None, None, None, _sis_params(3), 3, None, 1, 0, None) == W.EINVAL
    assert fn(dims, d.ctypes.data, m.ctypes.data, None, _sis_params(1), 1, None, 1, 0, None) == W.EINVAL
    assert fn(dims, d.ctypes.data, m.ctypes.data, None, _sis_params(17), 17, None, 1, 0, None) == W.ELIMIT
    assert fn(dims, d.ctypes.data, m.ctypes.data, None, _sis_params(3, 33), 3, None, 1, 0, None) == W.ELIMIT
    big = (C.c_int * 3)(2000, 2000, 3)
    assert fn(big, d.ctypes.data, m.ctypes.data, None, _sis_params(3), 3, None, 1, 0, None) == W.ELIMIT
    four = (C.c_int * 3)(2, 2, 1)
    assert fn(four, d.ctypes.data, m.ctypes.data, None, _sis_params(3), 3, None, 1, 0, None) == W.EINVAL
    assert "visit" in W.last_error()


def test_geo_sis_simulation_validation():
    """geo_bsd.sis_simulation validates as the reference's sis.py does before calling the library."""
    import geo_bsd
    from geo_bsd.validation import CriticalValidationError, ParameterValidator
    ParameterValidator.validate_probability_sum([0.3, 0.3, 0.405])
    with pytest.raises(CriticalValidationError):
        ParameterValidator.validate_probability_sum([0.3, 0.3, 0.3])
    with pytest.raises(CriticalValidationError):
        ParameterValidator.validate_probability_sum([0.5, float("nan")])
    grid = geo_bsd.SugarboxGrid(4, 4, 2)
    prop = geo_bsd.IndProperty(np.zeros((4, 4, 2), np.uint8, order="F"), np.zeros((4, 4, 2), np.uint8, order="F"), 2)
    cm = geo_bsd.CovarianceModel(type=0, ranges=(4.0, 4.0, 4.0), sill=1.0)
    data = [{"cov_model": cm, "radiuses": (3, 3, 3), "max_neighbours": 8} for _ in range(2)]
    with pytest.raises(CriticalValidationError):
        geo_bsd.sis_simulation(prop, grid, data, 1, [0.2, 0.2])
    with pytest.raises(CriticalValidationError):
        geo_bsd.sis_simulation(prop, grid, data, 1, [1.2, -0.2])
    cont = geo_bsd.ContProperty(np.zeros((4, 4, 2), np.float32, order="F"), np.zeros((4, 4, 2), np.uint8, order="F"))
    with pytest.raises(TypeError):
        geo_bsd.sis_simulation(cont, grid, data, 1, [0.5, 0.5])


def test_sim_levels_argument_checks():
    """Ranks outside [-1, n_sim) and bad sizes are EINVAL before any device work; no ranks is OK."""
    fn = W._hpgl_so.hpgl_b200_sim_levels
    out = np.zeros(4, np.int32)
    bad = np.array([[-1], [0], [4], [1]], np.int32)
    assert fn(4, 1, bad.ctypes.data, out.ctypes.data) == W.EINVAL
    assert "range" in W.last_error()
    low = np.array([[-1], [-2], [0], [1]], np.int32)
    assert fn(4, 1, low.ctypes.data, out.ctypes.data) == W.EINVAL
    assert fn(4, 0, low.ctypes.data, out.ctypes.data) == W.EINVAL
    assert fn(4, 1, None, out.ctypes.data) == W.EINVAL
    assert fn(0, 1, None, None) == W.OK
