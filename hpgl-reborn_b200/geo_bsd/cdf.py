"""Non-parametric CDFs for the simulations (HPGL's src/geo_bsd/cdf.py)."""
from __future__ import annotations

import numpy

__all__ = ["CdfData", "calc_cdf"]


class CdfData:
    """Ascending values and their cumulative probabilities (float32)."""

    def __init__(self, values, probs):
        self.values = numpy.require(values, "float32")
        self.probs = numpy.require(probs, "float32")


def calc_cdf(prop):
    """The empirical CDF of a property's informed values (cdf.py:8-40): the
    distinct values in ascending order without the largest, each with the
    running sum of the value frequencies."""
    informed = numpy.asarray(prop.data)[numpy.asarray(prop.mask) != 0]
    if informed.size == 0:
        raise ValueError("calc_cdf: no informed values (all cells are masked)")
    values, counts = numpy.unique(informed, return_counts=True)
    size = values.size - 1 if values.size > 1 else values.size
    values = values[:size]
    probs = numpy.cumsum(counts[:size] / float(informed.size))
    return CdfData(values=values, probs=probs)
