"""geo_bsd's kriging API on the B200 engine.

Signatures, argument validation and output conventions follow HPGL's
src/geo_bsd/geo.py: ordinary_kriging (:573-607), simple_kriging (:610-649),
lvm_kriging (:651-696), median_ik (:699-738), simple_cokriging_markI (:804-841),
simple_cokriging_markII (:843-895), indicator_kriging (:759-801, two categories dispatch to
median IK with data[0]'s model, :785-793), simple_kriging_weights (:897-935),
the property/grid/model classes (:215-299) and the handler setters (:947-966).
The output property is a clone of the input that the library fills in place.

Additions (keyword-only, defaults keep the reference's behaviour):
  precision="fp64" | "fp32_refined"   FP64 solve, or FP32 factorisation with
                                      FP64-residual refinement
  refine_steps=2                      refinement steps for fp32_refined
  return_variance=False               also return the kriging variance (float64)
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy

from . import hpgl_wrap as W
from .validation import (CriticalValidationError, GridValidator, ParameterValidator, PathValidator, ValidationError,
                         ValidationWarning)

_hpgl_so = W._hpgl_so

_PRECISIONS = {"fp64": W.FP64_PLAIN, "fp64_plain": W.FP64_PLAIN, "fp32_refined": W.FP32_REFINED,
               "fp32": W.FP32_REFINED}
_default_precision = "fp64"


def set_precision(name: str) -> None:
    """Default precision mode for calls that do not pass `precision=`."""
    global _default_precision
    if name not in _PRECISIONS:
        raise ValueError(f"unknown precision {name!r}; one of {sorted(_PRECISIONS)}")
    _default_precision = name


def checkFWA(a):
    assert a.flags["F"] and a.flags["W"] and a.flags["A"]


class ContProperty:
    def __init__(self, data, mask):
        self.data = numpy.require(data, "float32", "F")
        self.mask = numpy.require(mask, "uint8", "F")

    def validate(self):
        checkFWA(self.data)
        checkFWA(self.mask)
        assert self.data.shape == self.mask.shape

    def fix_shape(self, grid):
        if self.data.ndim != 3 and self.data.size == grid.x * grid.y * grid.z:
            self.data = self.data.reshape((grid.x, grid.y, grid.z), order="F")
        if self.mask.ndim != 3 and self.mask.size == grid.x * grid.y * grid.z:
            self.mask = self.mask.reshape((grid.x, grid.y, grid.z), order="F")

    def __getitem__(self, idx):
        if idx == 0:
            return self.data
        if idx == 1:
            return self.mask
        raise RuntimeError("Index out of range.")


class IndProperty:
    def __init__(self, data, mask, indicator_count):
        self.data = numpy.require(data, "uint8", "F")
        self.mask = numpy.require(mask, "uint8", "F")
        self.indicator_count = indicator_count
        if numpy.sum(numpy.bitwise_and(numpy.asarray(mask) > 0, numpy.asarray(data) >= indicator_count)) > 0:
            raise RuntimeError("Property contains some indicators outside of [0..%s] range." % (indicator_count - 1))
        assert numpy.shape(data) == numpy.shape(mask)

    def validate(self):
        checkFWA(self.data)
        checkFWA(self.mask)
        assert self.data.shape == self.mask.shape

    def __getitem__(self, idx):
        if idx == 0:
            return self.data
        if idx == 1:
            return self.mask
        if idx == 2:
            return self.indicator_count
        raise RuntimeError("Index out of range.")


class covariance:
    spherical = 0
    exponential = 1
    gaussian = 2


class SugarboxGrid:
    def __init__(self, x, y, z):
        GridValidator.validate_grid_dimensions(x, y, z)
        self.x = x
        self.y = y
        self.z = z


class CovarianceModel:
    def __init__(self, type=0, ranges=(0, 0, 0), angles=(0.0, 0.0, 0.0), sill=1.0, nugget=0.0):
        self.type = type
        self.ranges = ranges
        self.angles = angles
        self.sill = sill
        self.nugget = nugget
        ParameterValidator.validate_covariance_parameters(sill, nugget, ranges, angles)


def _to_prop(t):
    if isinstance(t, tuple):
        if len(t) == 3:
            return IndProperty(*t)
        if len(t) == 2:
            return ContProperty(*t)
        raise AssertionError("property tuple must have 2 or 3 items")
    assert isinstance(t, (ContProperty, IndProperty))
    return t


def _clone_prop(prop):
    data2 = prop.data.copy("F")
    mask2 = prop.mask.copy("F")
    if isinstance(prop, IndProperty):
        return IndProperty(data2, mask2, prop.indicator_count)
    return ContProperty(data2, mask2)


def _output_like(prop):
    """Output arrays for an engine call that writes every cell of its outputs
    (values and mask, the informed cells copied on the device): the input's
    shapes and types, not initialised on the host."""
    data2 = numpy.empty_like(prop.data, order="F")
    mask2 = numpy.empty_like(prop.mask, order="F")
    if isinstance(prop, IndProperty):
        return IndProperty(data2, mask2, prop.indicator_count)
    return ContProperty(data2, mask2)


def _empty_clone(prop):
    """A property of the same shape with every value 0 and every cell uninformed."""
    data2 = prop.data.copy("F")
    data2.fill(0)
    mask2 = prop.mask.copy("F")
    mask2.fill(0)
    if isinstance(prop, IndProperty):
        return IndProperty(data2, mask2, prop.indicator_count)
    return ContProperty(data2, mask2)


def _dims(grid, prop):
    n = grid.x * grid.y * grid.z
    if prop.data.size != n:
        raise RuntimeError("Invalid data size. Size of data = %s. Size of grid = %s" % (prop.data.size, n))
    return (C.c_int * 3)(grid.x, grid.y, grid.z)


def _flat(a):
    # Fortran-order flattening is the node order x + nx*y + nx*ny*z
    return a.reshape(-1, order="F")


def _int_radiuses(r):
    return tuple(int(round(v)) for v in r)


def _options(precision, refine_steps, estimate64=None, variance=None, status=None, probs=None):
    o = W._HPGL_B200_OPTIONS()
    o.precision = _PRECISIONS[precision or _default_precision]
    o.refine_steps = int(refine_steps)
    o.flags = W.FLAG_OUT_IS_CLONE
    o.estimate64 = estimate64.ctypes.data if estimate64 is not None else None
    o.variance = variance.ctypes.data if variance is not None else None
    o.status = status.ctypes.data if status is not None else None
    o.ik_probs = probs.ctypes.data if probs is not None else None
    return o


def _cont_kriging(kind, prop, grid, radiuses, max_neighbours, cov_model, mean, precision, refine_steps,
                  return_variance):
    prop = _to_prop(prop)
    GridValidator.validate_grid_dimensions(grid.x, grid.y, grid.z)
    valid_radiuses = ParameterValidator.validate_radius(radiuses, "radiuses")
    ParameterValidator.validate_max_neighbors(max_neighbours)
    ParameterValidator.validate_covariance_parameters(cov_model.sill, cov_model.nugget, cov_model.ranges,
                                                      cov_model.angles)
    out_prop = _output_like(prop)
    dims = _dims(grid, prop)
    p = W._HPGL_SK_PARAMS(covariance_type=cov_model.type, ranges=tuple(cov_model.ranges),
                          angles=tuple(cov_model.angles), sill=cov_model.sill, nugget=cov_model.nugget,
                          radiuses=_int_radiuses(valid_radiuses), max_neighbours=max_neighbours,
                          automatic_mean=(mean is None), mean=(mean if mean is not None else 0))
    var = numpy.empty(prop.data.size, numpy.float64) if return_variance else None
    opt = _options(precision, refine_steps, variance=var)
    d_in = _flat(prop.data)
    m_in = _flat(prop.mask)
    d_out = _flat(out_prop.data)
    m_out = _flat(out_prop.mask)
    rc = _hpgl_so.hpgl_b200_cont_kriging_ex(kind, dims, d_in.ctypes.data, m_in.ctypes.data, C.byref(p),
                                            d_out.ctypes.data, m_out.ctypes.data, C.byref(opt))
    W.check(rc, "ordinary_kriging" if kind == 0 else "simple_kriging")
    if return_variance:
        return out_prop, var.reshape(prop.data.shape, order="F")
    return out_prop


def ordinary_kriging(prop, grid, radiuses, max_neighbours, cov_model, *, precision: Optional[str] = None,
                     refine_steps: int = 2, return_variance: bool = False):
    return _cont_kriging(0, prop, grid, radiuses, max_neighbours, cov_model, None, precision, refine_steps,
                         return_variance)


def simple_kriging(prop, grid, radiuses, max_neighbours, cov_model, mean=None, *, precision: Optional[str] = None,
                   refine_steps: int = 2, return_variance: bool = False):
    return _cont_kriging(1, prop, grid, radiuses, max_neighbours, cov_model, mean, precision, refine_steps,
                         return_variance)


def lvm_kriging(prop, grid, mean_data, radiuses, max_neighbours, cov_model, *, precision: Optional[str] = None,
                refine_steps: int = 2, return_variance: bool = False):
    """Kriging with a locally varying mean: SK weights, each neighbour centred
    on its own cell's mean and the cell's mean added back; failed cells take
    their mean. mean_data holds one value per grid cell (Fortran order, as
    the reference's ndpointer(flags='F') argument requires)."""
    prop = _to_prop(prop)
    GridValidator.validate_grid_dimensions(grid.x, grid.y, grid.z)
    valid_radiuses = ParameterValidator.validate_radius(radiuses, "radiuses")
    ParameterValidator.validate_max_neighbors(max_neighbours)
    ParameterValidator.validate_covariance_parameters(cov_model.sill, cov_model.nugget, cov_model.ranges,
                                                      cov_model.angles)
    if not isinstance(mean_data, numpy.ndarray):
        raise ValueError("lvm_kriging: mean_data must be a numpy array")
    if mean_data.dtype != numpy.float32:
        mean_data = numpy.require(mean_data, dtype="float32")
    out_prop = _output_like(prop)
    dims = _dims(grid, prop)
    if mean_data.size != prop.data.size:
        raise RuntimeError("lvm_kriging: mean_data has %d values, the grid %d" % (mean_data.size, prop.data.size))
    flags = mean_data.flags
    if not (flags.f_contiguous and flags.writeable and flags.aligned):
        # the reference binds mean_data as ndpointer(float32, flags=['F', 'W', 'A'])
        raise C.ArgumentError("argument 4: TypeError: array must have flags ['F_CONTIGUOUS', 'WRITEABLE', "
                              "'ALIGNED']")
    p = W._HPGL_OK_PARAMS(covariance_type=cov_model.type, ranges=tuple(cov_model.ranges),
                          angles=tuple(cov_model.angles), sill=cov_model.sill, nugget=cov_model.nugget,
                          radiuses=_int_radiuses(valid_radiuses), max_neighbours=max_neighbours)
    var = numpy.empty(prop.data.size, numpy.float64) if return_variance else None
    opt = _options(precision, refine_steps, variance=var)
    rc = _hpgl_so.hpgl_b200_lvm_kriging_ex(dims, _flat(prop.data).ctypes.data, _flat(prop.mask).ctypes.data,
                                           mean_data.ctypes.data, C.byref(p), _flat(out_prop.data).ctypes.data,
                                           _flat(out_prop.mask).ctypes.data, C.byref(opt))
    W.check(rc, "lvm_kriging")
    if return_variance:
        return out_prop, var.reshape(prop.data.shape, order="F")
    return out_prop


def _cokriging_props(prop, secondary):
    prop = _to_prop(prop)
    secondary = _to_prop(secondary)
    if secondary.data.size != prop.data.size:
        raise RuntimeError("Size of secondary data (%d) is different from size of primary data (%d)"
                           % (secondary.data.size, prop.data.size))
    return prop, secondary, _clone_prop(prop)


def _cokriging_call(mark, grid, prop, secondary, out_prop, m1, m2):
    dims = _dims(grid, prop)
    opt = _options(None, 0)
    rc = _hpgl_so.hpgl_b200_cokriging_ex(mark, dims, _flat(prop.data).ctypes.data, _flat(prop.mask).ctypes.data,
                                         _flat(secondary.data).ctypes.data, _flat(secondary.mask).ctypes.data,
                                         C.byref(m1) if m1 is not None else None,
                                         C.byref(m2) if m2 is not None else None,
                                         _flat(out_prop.data).ctypes.data, _flat(out_prop.mask).ctypes.data,
                                         C.byref(opt))
    W.check(rc, "simple_cokriging_mark%d" % mark)
    return out_prop


def simple_cokriging_markI(prop, grid, secondary_data, primary_mean, secondary_mean, secondary_variance,
                           correlation_coef, radiuses, max_neighbours, cov_model):
    """Simple collocated cokriging, Markov model I: the cross covariance is
    correlation_coef * sqrt(secondary_variance / C(0)) * C (the primary model)."""
    GridValidator.validate_grid_dimensions(grid.x, grid.y, grid.z)
    valid_radiuses = ParameterValidator.validate_radius(radiuses, "radiuses")
    ParameterValidator.validate_max_neighbors(max_neighbours)
    ParameterValidator.validate_covariance_parameters(cov_model.sill, cov_model.nugget, cov_model.ranges,
                                                      cov_model.angles)
    ParameterValidator.validate_correlation_coef(correlation_coef)
    ParameterValidator.validate_variance(secondary_variance, "secondary_variance")
    prop, secondary, out_prop = _cokriging_props(prop, secondary_data)
    m1 = W._HPGL_COK_M1_PARAMS(covariance_type=cov_model.type, ranges=tuple(cov_model.ranges),
                               angles=tuple(cov_model.angles), sill=cov_model.sill, nugget=cov_model.nugget,
                               radiuses=_int_radiuses(valid_radiuses), max_neighbours=max_neighbours,
                               primary_mean=primary_mean, secondary_mean=secondary_mean,
                               secondary_variance=secondary_variance, correlation_coef=correlation_coef)
    return _cokriging_call(1, grid, prop, secondary, out_prop, m1, None)


def simple_cokriging_markII(grid, primary_data, secondary_data, correlation_coef, radiuses, max_neighbours):
    """Simple collocated cokriging, Markov model II: primary_data and
    secondary_data are dicts with "data" (a property), "mean" and "cov_model";
    the cross covariance is correlation_coef * sqrt(C1(0) / C2(0)) * C2."""
    GridValidator.validate_grid_dimensions(grid.x, grid.y, grid.z)
    valid_radiuses = ParameterValidator.validate_radius(radiuses, "radiuses")
    ParameterValidator.validate_max_neighbors(max_neighbours)
    ParameterValidator.validate_correlation_coef(correlation_coef)
    for d in (primary_data, secondary_data):
        cm = d["cov_model"]
        ParameterValidator.validate_covariance_parameters(cm.sill, cm.nugget, cm.ranges, cm.angles)
    prop, secondary, out_prop = _cokriging_props(primary_data["data"], secondary_data["data"])
    pcp, scp = primary_data["cov_model"], secondary_data["cov_model"]
    m2 = W._HPGL_COK_M2_PARAMS(
        primary_cov_params=W._HPGL_COV_PARAMS(covariance_type=pcp.type, ranges=tuple(pcp.ranges),
                                              angles=tuple(pcp.angles), sill=pcp.sill, nugget=pcp.nugget),
        secondary_cov_params=W._HPGL_COV_PARAMS(covariance_type=scp.type, ranges=tuple(scp.ranges),
                                                angles=tuple(scp.angles), sill=scp.sill, nugget=scp.nugget),
        radiuses=_int_radiuses(valid_radiuses), max_neighbours=max_neighbours, primary_mean=primary_data["mean"],
        secondary_mean=secondary_data["mean"], correlation_coef=correlation_coef)
    return _cokriging_call(2, grid, prop, secondary, out_prop, None, m2)


def median_ik(prop, grid, marginal_probs, radiuses, max_neighbours, cov_model, *, precision: Optional[str] = None,
              refine_steps: int = 2):
    prop = _to_prop(prop)
    GridValidator.validate_grid_dimensions(grid.x, grid.y, grid.z)
    valid_radiuses = ParameterValidator.validate_radius(radiuses, "radiuses")
    ParameterValidator.validate_max_neighbors(max_neighbours)
    ParameterValidator.validate_covariance_parameters(cov_model.sill, cov_model.nugget, cov_model.ranges,
                                                      cov_model.angles)
    if len(marginal_probs) != 2:
        raise ValueError("median_ik: marginal_probs must have exactly 2 elements")
    for i, pr in enumerate(marginal_probs):
        ParameterValidator.validate_probability(pr, f"marginal_probs[{i}]")
    out_prop = _clone_prop(prop)
    dims = _dims(grid, prop)
    p = W._HPGL_MEDIAN_IK_PARAMS(covariance_type=cov_model.type, ranges=tuple(cov_model.ranges),
                                 angles=tuple(cov_model.angles), sill=cov_model.sill, nugget=cov_model.nugget,
                                 radiuses=_int_radiuses(valid_radiuses), max_neighbours=max_neighbours,
                                 marginal_probs=tuple(marginal_probs))
    opt = _options(precision, refine_steps)
    rc = _hpgl_so.hpgl_b200_median_ik_ex(dims, _flat(prop.data).ctypes.data, _flat(prop.mask).ctypes.data,
                                         C.byref(p), _flat(out_prop.data).ctypes.data,
                                         _flat(out_prop.mask).ctypes.data, C.byref(opt))
    W.check(rc, "median_ik")
    return out_prop


def indicator_kriging(prop, grid, data, marginal_probs, *, precision: Optional[str] = None, refine_steps: int = 2,
                      return_probabilities: bool = False):
    prop = _to_prop(prop)
    GridValidator.validate_grid_dimensions(grid.x, grid.y, grid.z)
    ParameterValidator.validate_indicator_count(len(data))
    if len(marginal_probs) != len(data):
        raise ValueError(f"indicator_kriging: marginal_probs length ({len(marginal_probs)}) must match data length "
                         f"({len(data)})")
    for i, pr in enumerate(marginal_probs):
        ParameterValidator.validate_probability(pr, f"marginal_probs[{i}]")
    for i, ikd in enumerate(data):
        ParameterValidator.validate_radius(ikd["radiuses"], f"data[{i}].radiuses")
        ParameterValidator.validate_max_neighbors(ikd["max_neighbours"])
        cm = ikd["cov_model"]
        ParameterValidator.validate_covariance_parameters(cm.sill, cm.nugget, cm.ranges, cm.angles)
    for i in range(len(data)):
        data[i]["marginal_prob"] = marginal_probs[i]
    if len(data) == 2:
        return median_ik(prop, grid, (data[0]["marginal_prob"], 1 - data[0]["marginal_prob"]),
                         data[0]["radiuses"], data[0]["max_neighbours"], data[0]["cov_model"], precision=precision,
                         refine_steps=refine_steps)
    out_prop = _clone_prop(prop)
    dims = _dims(grid, prop)
    m = len(data)
    params = (W._HPGL_IK_PARAMS * m)()
    for i, ikd in enumerate(data):
        cm = ikd["cov_model"]
        params[i] = W._HPGL_IK_PARAMS(covariance_type=cm.type, ranges=tuple(cm.ranges), angles=tuple(cm.angles),
                                      sill=cm.sill, nugget=cm.nugget, radiuses=_int_radiuses(ikd["radiuses"]),
                                      max_neighbours=ikd["max_neighbours"], marginal_prob=marginal_probs[i])
    probs = numpy.empty((prop.data.size, m), numpy.float32) if return_probabilities else None
    opt = _options(precision, refine_steps, probs=probs)
    rc = _hpgl_so.hpgl_b200_indicator_kriging_ex(dims, _flat(prop.data).ctypes.data, _flat(prop.mask).ctypes.data,
                                                 params, m, _flat(out_prop.data).ctypes.data,
                                                 _flat(out_prop.mask).ctypes.data, C.byref(opt))
    W.check(rc, "indicator_kriging")
    if return_probabilities:
        return out_prop, probs
    return out_prop


def simple_kriging_weights(center_point, n_x, n_y, n_z, ranges=(100000, 100000, 100000), sill=1,
                           cov_type=covariance.exponential, nugget=None, angles=None):
    if angles is None:
        angles = (0, 0, 0)
    if nugget is None:
        nugget = 0
    ParameterValidator.validate_covariance_parameters(sill, nugget, ranges, angles)
    if len(n_x) != len(n_y) or len(n_x) != len(n_z):
        raise RuntimeError("Invalid pointset. %s,%s,%s." % (len(n_x), len(n_y), len(n_z)))
    for name, arr in (("n_x", n_x), ("n_y", n_y), ("n_z", n_z)):
        a = numpy.asarray(arr, dtype="float32")
        if numpy.any(numpy.isnan(a)) or numpy.any(numpy.isinf(a)):
            raise ValueError(f"simple_kriging_weights: {name} contains NaN or infinite values")
    covp = W._HPGL_COV_PARAMS(covariance_type=cov_type, ranges=tuple(ranges), angles=tuple(angles), sill=sill,
                              nugget=nugget)
    weights = numpy.zeros(len(n_x), dtype="float32")
    centre = (C.c_float * 3)(*center_point)
    _hpgl_so.hpgl_simple_kriging_weights(centre, numpy.array(n_x, dtype="float32"),
                                         numpy.array(n_y, dtype="float32"), numpy.array(n_z, dtype="float32"),
                                         len(n_x), C.byref(covp), weights)
    return weights


# ------------------------------------------------------------------ property files
# write_property / write_gslib_property / load_cont_property / read_inc_file_float /
# read_inc_file_byte / load_ind_property: geo.py:418-570 of the reference.
def _shape_of(prop):
    if prop.data.ndim == 3:
        return W._HPGL_SHAPE(data=prop.data.shape, strides=(1, prop.data.shape[0],
                                                           prop.data.shape[0] * prop.data.shape[1]))
    return W._HPGL_SHAPE(data=(prop.data.size, 1, 1), strides=(1, prop.data.size, prop.data.size))


def _io_check(rc, what):
    if rc != 0:
        raise RuntimeError(what + " failed: " + W.last_error())


def write_property(prop, filename, prop_name, undefined_value, indicator_values=None):
    safe_path = PathValidator.validate_filepath(filename)
    prop = _to_prop(prop)
    if indicator_values is None:
        indicator_values = []
    sh = _shape_of(prop)
    if isinstance(prop, ContProperty):
        marr = W._HPGL_CONT_MASKED_ARRAY(data=prop.data.ctypes.data_as(C.POINTER(C.c_float)),
                                         mask=prop.mask.ctypes.data_as(C.POINTER(C.c_ubyte)), shape=sh)
        rc = _hpgl_so.hpgl_write_inc_file_float(safe_path.encode("utf-8"), C.byref(marr), undefined_value,
                                                prop_name.encode("utf-8"))
    else:
        ind_arr = numpy.array(indicator_values, dtype="uint8")
        marr = W._HPGL_IND_MASKED_ARRAY(data=prop.data.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                        mask=prop.mask.ctypes.data_as(C.POINTER(C.c_ubyte)), shape=sh,
                                        indicator_count=prop.indicator_count)
        rc = _hpgl_so.hpgl_write_inc_file_byte(safe_path.encode("utf-8"), C.byref(marr), int(undefined_value),
                                               prop_name.encode("utf-8"),
                                               ind_arr.ctypes.data_as(C.POINTER(C.c_ubyte)), len(indicator_values))
    _io_check(rc, "write_property")


def write_gslib_property(prop, filename, prop_name, undefined_value, indicator_values=None):
    safe_path = PathValidator.validate_filepath(filename)
    prop = _to_prop(prop)
    if indicator_values is None:
        indicator_values = []
    sh = _shape_of(prop)
    if isinstance(prop, ContProperty):
        marr = W._HPGL_CONT_MASKED_ARRAY(data=prop.data.ctypes.data_as(C.POINTER(C.c_float)),
                                         mask=prop.mask.ctypes.data_as(C.POINTER(C.c_ubyte)), shape=sh)
        rc = _hpgl_so.hpgl_write_gslib_cont_property(C.byref(marr), safe_path.encode("utf-8"),
                                                     prop_name.encode("utf-8"), undefined_value)
    else:
        ind_arr = (C.c_ubyte * max(len(indicator_values), 1))(*indicator_values)
        marr = W._HPGL_IND_MASKED_ARRAY(data=prop.data.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                        mask=prop.mask.ctypes.data_as(C.POINTER(C.c_ubyte)), shape=sh,
                                        indicator_count=prop.indicator_count)
        rc = _hpgl_so.hpgl_write_gslib_byte_property(C.byref(marr), safe_path.encode("utf-8"),
                                                     prop_name.encode("utf-8"), undefined_value, ind_arr,
                                                     len(indicator_values))
    _io_check(rc, "write_gslib_property")


def _load_prop_cont_slow(filename, undefined_value):
    values, mask = [], []
    with open(PathValidator.validate_filepath(filename), "r", encoding="utf-8") as f:
        for line in f:
            if line.strip().startswith("--"):
                continue
            for part in line.split():
                try:
                    val = float(part.strip())
                except (ValueError, TypeError):
                    continue
                values.append(val)
                mask.append(0 if val == undefined_value else 1)
    return ContProperty(numpy.array(values, dtype="float32"), numpy.array(mask, dtype="uint8"))


def _load_prop_ind_slow(filename, undefined_value, ind_values):
    dict_map = {v: i for i, v in enumerate(ind_values)}
    values, mask = [], []
    with open(PathValidator.validate_filepath(filename), "r", encoding="utf-8") as f:
        for line in f:
            if line.strip().startswith("--"):
                continue
            for part in line.split():
                try:
                    val = int(part.strip())
                except (ValueError, TypeError):
                    continue
                if val == undefined_value:
                    values.append(255)
                    mask.append(0)
                else:
                    values.append(dict_map[val])
                    mask.append(1)
    return IndProperty(numpy.array(values, dtype="uint8"), numpy.array(mask, dtype="uint8"), len(ind_values))


def _total(size):
    if isinstance(size, tuple) and len(size) == 3:
        GridValidator.validate_grid_dimensions(size[0], size[1], size[2])
        return size[0] * size[1] * size[2]
    return size


def read_inc_file_float(filename, undefined_value, size):
    safe_path = PathValidator.validate_filepath(filename, must_exist=True)
    total = _total(size)
    data = numpy.zeros(total, dtype="float32", order="F")
    mask = numpy.zeros(total, dtype="uint8", order="F")
    _io_check(_hpgl_so.hpgl_read_inc_file_float(safe_path.encode("utf-8"), undefined_value, total, data, mask),
              "read_inc_file_float")
    return ContProperty(data, mask)


def read_inc_file_byte(filename, undefined_value, size, indicator_values):
    safe_path = PathValidator.validate_filepath(filename, must_exist=True)
    total = _total(size)
    data = numpy.zeros(total, dtype="uint8", order="F")
    mask = numpy.zeros(total, dtype="uint8", order="F")
    vals = numpy.array(indicator_values, dtype="uint8")
    _io_check(_hpgl_so.hpgl_read_inc_file_byte(safe_path.encode("utf-8"), int(undefined_value), total, data, mask,
                                               vals, len(indicator_values)), "read_inc_file_byte")
    return IndProperty(data, mask, len(indicator_values))


def load_cont_property(filename, undefined_value, size=None):
    safe_path = PathValidator.validate_filepath(filename, must_exist=True)
    if size is None:
        print("[WARNING]. load_cont_property: Size is not specified. Using slow and ineficcient method.")
        return _load_prop_cont_slow(safe_path, undefined_value)
    return read_inc_file_float(safe_path, undefined_value, size)


def load_ind_property(filename, undefined_value, indicator_values, size=None):
    if size is None:
        print("[WARNING]. load_ind_property: Size is not specified. Using slow and ineficcient method.")
        return _load_prop_ind_slow(filename, undefined_value, indicator_values)
    return read_inc_file_byte(filename, undefined_value, size, indicator_values)


def calc_mean(prop):
    prop = _to_prop(prop)
    sel = prop.mask.reshape(-1) == 1
    if not numpy.any(sel):
        raise ValueError("calc_mean: no informed values (all masked)")
    return float(numpy.sum(prop.data.reshape(-1)[sel].astype(numpy.float64)) / numpy.count_nonzero(sel))


def set_thread_num(num):
    _hpgl_so.hpgl_set_thread_num(num)


def get_thread_num():
    return _hpgl_so.hpgl_get_thread_num()


_handlers = {}


def set_output_handler(handler, param):
    if handler is None:
        _hpgl_so.hpgl_set_output_handler(C.cast(None, W.hpgl_output_handler), None)
        _handlers.pop("out", None)
    else:
        h = W.hpgl_output_handler(handler)
        _handlers["out"] = h
        _hpgl_so.hpgl_set_output_handler(h, param)


def set_progress_handler(handler, param):
    if handler is None:
        _hpgl_so.hpgl_set_progress_handler(C.cast(None, W.hpgl_progress_handler), None)
        _handlers.pop("progress", None)
    else:
        h = W.hpgl_progress_handler(handler)
        _handlers["progress"] = h
        _hpgl_so.hpgl_set_progress_handler(h, param)


def find_neighbours(prop, grid, radiuses, max_neighbours, cov_model, nodes, kind=0):
    """Neighbour node indices per node, as the reference's lookup returns them.

    kind 0 = OK (analytic covariance), 1 = SK / IK (box-truncated). Returns
    (idx[n, k] -1-padded, count[n], template_path[n])."""
    prop = _to_prop(prop)
    dims = _dims(grid, prop)
    nodes = numpy.ascontiguousarray(nodes, dtype=numpy.int32)
    k = int(max_neighbours)
    idx = numpy.full((len(nodes), k), -1, numpy.int32)
    cnt = numpy.zeros(len(nodes), numpy.int32)
    path = numpy.zeros(len(nodes), numpy.uint8)
    p = W._HPGL_SK_PARAMS(covariance_type=cov_model.type, ranges=tuple(cov_model.ranges),
                          angles=tuple(cov_model.angles), sill=cov_model.sill, nugget=cov_model.nugget,
                          radiuses=_int_radiuses(radiuses), max_neighbours=k, automatic_mean=1, mean=0)
    rc = _hpgl_so.hpgl_b200_find_neighbours(kind, dims, _flat(prop.mask).ctypes.data, C.byref(p),
                                            nodes.ctypes.data, len(nodes), idx.ctypes.data, cnt.ctypes.data,
                                            path.ctypes.data)
    W.check(rc, "find_neighbours")
    return idx, cnt, path


__all__ = ["ContProperty", "IndProperty", "SugarboxGrid", "CovarianceModel", "covariance", "ordinary_kriging",
           "simple_kriging", "lvm_kriging", "simple_cokriging_markI",
           "simple_cokriging_markII", "median_ik", "indicator_kriging", "simple_kriging_weights", "calc_mean",
           "set_thread_num", "get_thread_num", "write_property",
           "write_gslib_property", "load_cont_property", "load_ind_property", "read_inc_file_float",
           "read_inc_file_byte", "set_output_handler", "set_progress_handler", "set_precision",
           "find_neighbours", "ValidationError", "CriticalValidationError", "ValidationWarning"]
