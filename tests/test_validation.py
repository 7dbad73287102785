"""Argument validation keeps HPGL's behaviour (src/geo_bsd/validation.py)."""
import pytest

from geo_bsd import validation as V
import geo_bsd


def test_grid_limits():
    V.GridValidator.validate_grid_dimensions(1, 1, 1)
    with pytest.raises(V.CriticalValidationError):
        V.GridValidator.validate_grid_dimensions(0, 5, 5)
    with pytest.raises(V.CriticalValidationError):
        V.GridValidator.validate_grid_dimensions(10000001, 1, 1)
    with pytest.raises(V.CriticalValidationError):
        V.GridValidator.validate_grid_dimensions(100000, 100000, 1)


def test_radius_rules():
    assert V.ParameterValidator.validate_radius((3, 4, 5)) == (3, 4, 5)
    assert V.ParameterValidator.validate_radius(2.5) == (2.5, 2.5, 2.5)
    with pytest.raises(V.CriticalValidationError):
        V.ParameterValidator.validate_radius((1, 2))
    with pytest.raises(V.CriticalValidationError):
        V.ParameterValidator.validate_radius((1, -2, 3))
    with pytest.raises(V.CriticalValidationError):
        V.ParameterValidator.validate_radius((1, float("nan"), 3))


def test_neighbour_and_covariance_rules():
    with pytest.raises(V.CriticalValidationError):
        V.ParameterValidator.validate_max_neighbors(0)
    with pytest.raises(V.ValidationWarning):
        V.ParameterValidator.validate_max_neighbors(1001)
    with pytest.raises(V.CriticalValidationError):
        V.ParameterValidator.validate_covariance_parameters(1.0, 2.0)  # nugget > sill
    with pytest.raises(V.CriticalValidationError):
        V.ParameterValidator.validate_covariance_parameters(-1.0, 0.0)
    with pytest.raises(V.CriticalValidationError):
        V.ParameterValidator.validate_covariance_parameters(1.0, 0.0, (1, 2), (0, 0, 0))
    V.ParameterValidator.validate_covariance_parameters(1.0, 0.0, (1, 2, 3), (0, 400, 0))  # warns only


def test_probabilities_and_indicators():
    with pytest.raises(V.CriticalValidationError):
        V.ParameterValidator.validate_probability(1.5)
    with pytest.raises(V.CriticalValidationError):
        V.ParameterValidator.validate_indicator_count(0)
    with pytest.raises(V.CriticalValidationError):
        V.ParameterValidator.validate_indicator_count(257)


def test_api_validates_before_calling_the_library():
    g = geo_bsd.SugarboxGrid(4, 4, 4)
    import numpy as np
    prop = geo_bsd.ContProperty(np.zeros((4, 4, 4), np.float32), np.zeros((4, 4, 4), np.uint8))
    with pytest.raises(V.CriticalValidationError):
        geo_bsd.CovarianceModel(type=0, ranges=(1, 1, 1), sill=1.0, nugget=2.0)
    cm = geo_bsd.CovarianceModel(type=0, ranges=(2, 2, 2), sill=1.0, nugget=0.0)
    with pytest.raises(V.CriticalValidationError):
        geo_bsd.ordinary_kriging(prop, g, (1, 1, 1), 0, cm)
    with pytest.raises(ValueError):
        geo_bsd.indicator_kriging(geo_bsd.IndProperty(np.zeros(64, np.uint8), np.zeros(64, np.uint8), 3), g,
                                  [{"cov_model": cm, "radiuses": (1, 1, 1), "max_neighbours": 4}] * 3, [0.5, 0.5])
