"""Sequential indicator simulation on the B200 engine (HPGL's src/geo_bsd/sis.py).

sis_simulation keeps the reference's signature and argument handling
(sis.py:52-135): a list of scalar marginal probabilities (which must sum to 1)
selects hpgl_sis_simulation, a list of per-cell mean arrays the LVM variant
with use_correlogram passed through; the output is a clone of the input (an
empty one when use_harddata is False) whose indicator_count becomes the
number of categories; each data[i]["marginal_prob"] is set as there (0 under
LVM). The simulation runs through hpgl_b200_sis_ex so that failures raise.
force_single_thread, force_parallel, use_regions, region_size and
min_neighbours are accepted and unused, as in the reference.
"""
from __future__ import annotations

import ctypes as C

import numpy

from . import hpgl_wrap as W
from .geo import IndProperty, _clone_prop, _empty_clone, _flat, _int_radiuses, _to_prop
from .validation import GridValidator, ParameterValidator

__all__ = ["sis_simulation"]


def sis_simulation(prop, grid, data, seed, marginal_probs, use_correlogram=True, mask=None,
                   force_single_thread=False, force_parallel=False, use_harddata=True, use_regions=False,
                   region_size=(), min_neighbours=0):
    """Sequential indicator simulation of the uninformed cells of `prop` (an
    IndProperty or a (data, mask, indicator_count) tuple); `data` holds one
    dict per category with "cov_model", "radiuses" and "max_neighbours"."""
    prop = _to_prop(prop)
    if not isinstance(prop, IndProperty):
        raise TypeError("sis_simulation: prop must be an indicator property")
    GridValidator.validate_grid_dimensions(grid.x, grid.y, grid.z)
    ParameterValidator.validate_indicator_count(len(data))
    ParameterValidator.validate_seed(seed)
    is_lvm = not numpy.isscalar(marginal_probs[0])
    if not is_lvm:
        ParameterValidator.validate_probability_sum(marginal_probs)
    for i, ikd in enumerate(data):
        cm = ikd["cov_model"]
        ParameterValidator.validate_covariance_parameters(cm.sill, cm.nugget, cm.ranges, cm.angles)
        ParameterValidator.validate_radius(ikd["radiuses"], f"ik_data[{i}].radiuses")
        ParameterValidator.validate_max_neighbors(ikd["max_neighbours"])
        if not is_lvm:
            ParameterValidator.validate_probability(marginal_probs[i], f"marginal_probs[{i}]")
    n = grid.x * grid.y * grid.z
    out_prop = _clone_prop(prop) if use_harddata else _empty_clone(prop)
    if out_prop.data.size != n:
        raise RuntimeError("Invalid data size. Size of data = %s. Size of grid = %s" % (out_prop.data.size, n))
    m = len(data)
    out_prop.indicator_count = m
    keep = []
    means = None
    if is_lvm:
        if len(marginal_probs) != m:
            raise ValueError(f"sis_simulation: {len(marginal_probs)} mean arrays for {m} categories")
        ptrs = (C.c_void_p * m)()
        for i, mp in enumerate(marginal_probs):
            mv = numpy.require(mp.data if hasattr(mp, "mask") and hasattr(mp, "data") else mp, "float32", "F")
            if mv.size != n:
                raise RuntimeError("sis_simulation: mean %d has %d values, the grid %d" % (i, mv.size, n))
            keep.append(mv)
            ptrs[i] = _flat(mv).ctypes.data
        means = ptrs
    for i in range(m):
        data[i]["marginal_prob"] = 0 if is_lvm else marginal_probs[i]
    params = (W._HPGL_IK_PARAMS * m)()
    for i, ikd in enumerate(data):
        cm = ikd["cov_model"]
        params[i] = W._HPGL_IK_PARAMS(covariance_type=cm.type, ranges=tuple(cm.ranges), angles=tuple(cm.angles),
                                      sill=cm.sill, nugget=cm.nugget, radiuses=_int_radiuses(ikd["radiuses"]),
                                      max_neighbours=ikd["max_neighbours"],
                                      marginal_prob=0 if is_lvm else marginal_probs[i])
    sim = None
    if mask is not None:
        sim = numpy.require(mask.data if hasattr(mask, "mask") and hasattr(mask, "data") else mask, "uint8", "F")
        if sim.size != n:
            raise RuntimeError("sis_simulation: mask has %d values, the grid %d" % (sim.size, n))
    dims = (C.c_int * 3)(grid.x, grid.y, grid.z)
    opt = W._HPGL_B200_OPTIONS(precision=0, refine_steps=0, flags=0, stream=None, estimate64=None, variance=None,
                               status=None, ik_probs=None)
    rc = W._hpgl_so.hpgl_b200_sis_ex(dims, _flat(out_prop.data).ctypes.data, _flat(out_prop.mask).ctypes.data,
                                     _flat(sim).ctypes.data if sim is not None else None, params, m,
                                     C.cast(means, C.c_void_p) if means is not None else None, int(seed),
                                     1 if use_correlogram else 0, C.byref(opt))
    W.check(rc, "sis_simulation")
    return out_prop
