"""Sequential Gaussian simulation on the B200 engine (HPGL's src/geo_bsd/sgs.py).

sgs_simulation keeps the reference's signature and argument handling
(sgs.py:52-151): the covariance model is normalised by its sill, the output is
a clone of the input (or an empty one when use_harddata is False), a scalar or
missing mean selects hpgl_sgs_simulation and an array mean the LVM variant,
cdf_data (a CdfData) maps the values to the Gaussian space and back. The
simulation runs through hpgl_b200_sgs_ex so that failures raise.
"""
from __future__ import annotations

import ctypes as C

import numpy

from . import hpgl_wrap as W
from .cdf import CdfData
from .geo import CovarianceModel, _clone_prop, _empty_clone, _to_prop
from .validation import GridValidator, ParameterValidator

__all__ = ["sgs_simulation"]


def normed_cov_model(cov_model):
    coef = cov_model.sill
    return CovarianceModel(cov_model.type, cov_model.ranges, cov_model.angles, cov_model.sill / coef,
                           cov_model.nugget / coef)


def _checkFWA(a):
    assert a.flags["F"] and a.flags["W"] and a.flags["A"]


def sgs_simulation(prop, grid, cdf_data, radiuses, max_neighbours, cov_model, seed, kriging_type="sk", mean=None,
                   use_harddata=True, use_regions=False, region_size=None, mask=None, force_single_thread=False,
                   force_parallel=False, min_neighbours=0, **params):
    """Sequential Gaussian simulation. See HPGL's sgs_simulation for the
    arguments; use_regions, region_size, force_single_thread, force_parallel
    and min_neighbours are accepted and unused, as there."""
    prop = _to_prop(prop)
    GridValidator.validate_grid_dimensions(grid.x, grid.y, grid.z)
    valid_radiuses = tuple(int(r) for r in ParameterValidator.validate_radius(radiuses, "radiuses"))
    ParameterValidator.validate_max_neighbors(max_neighbours)
    ParameterValidator.validate_covariance_parameters(cov_model.sill, cov_model.nugget, cov_model.ranges,
                                                      cov_model.angles)
    ParameterValidator.validate_seed(seed)
    ParameterValidator.validate_min_neighbors(min_neighbours, max_neighbours)
    prop.fix_shape(grid)
    cov_model = normed_cov_model(cov_model)
    out_prop = _clone_prop(prop) if use_harddata else _empty_clone(prop)
    if mean is not None and not numpy.isscalar(mean):
        mean = numpy.require(mean, dtype="float32", requirements="F")
    if mask is not None:
        mask = numpy.require(mask, dtype="uint8", requirements="F")
    p = W._HPGL_SGS_PARAMS(covariance_type=cov_model.type, ranges=tuple(cov_model.ranges),
                           angles=tuple(cov_model.angles), sill=cov_model.sill, nugget=cov_model.nugget,
                           radiuses=valid_radiuses, max_neighbours=max_neighbours,
                           kriging_kind={"sk": W._HPGL_KRIGING_KIND.simple,
                                         "ok": W._HPGL_KRIGING_KIND.ordinary}[kriging_type],
                           seed=seed, min_neighbours=min_neighbours)
    cdf = None
    if cdf_data is not None:
        assert isinstance(cdf_data, CdfData)
        cdf = W._HPGL_NON_PARAMETRIC_CDF(values=cdf_data.values.ctypes.data_as(C.POINTER(C.c_float)),
                                         probs=cdf_data.probs.ctypes.data_as(C.POINTER(C.c_float)),
                                         size=cdf_data.values.size)
    n = grid.x * grid.y * grid.z
    if out_prop.data.size != n:
        raise RuntimeError("Invalid data size. Size of data = %s. Size of grid = %s" % (out_prop.data.size, n))
    means = None
    if mean is not None and not numpy.isscalar(mean):
        _checkFWA(mean)
        if mean.size != n:
            raise RuntimeError("sgs_simulation: mean has %d values, the grid %d" % (mean.size, n))
        means = mean
    if mask is not None:
        _checkFWA(mask)
        if mask.size != n:
            raise RuntimeError("sgs_simulation: mask has %d values, the grid %d" % (mask.size, n))
    dims = (C.c_int * 3)(grid.x, grid.y, grid.z)
    opt = W._HPGL_B200_OPTIONS(precision=0, refine_steps=0, flags=0, stream=None, estimate64=None, variance=None,
                               status=None, ik_probs=None)
    rc = W._hpgl_so.hpgl_b200_sgs_ex(dims, out_prop.data.ctypes.data, out_prop.mask.ctypes.data,
                                     mask.ctypes.data if mask is not None else None,
                                     C.byref(cdf) if cdf is not None else None,
                                     means.ctypes.data if means is not None else None, C.byref(p), C.byref(opt))
    W.check(rc, "sgs_simulation")
    return out_prop
