"""Argument validation with the behaviour of HPGL's geo_bsd/validation.py.

Limits and messages follow the reference (src/geo_bsd/validation.py:23-61,
:195-230 grid, :284-345 radius, :344-380 max neighbours, :397-500 covariance,
:560-580 indicator count, probability checks): the same exception classes,
the same accepted ranges, warnings (not errors) for angles outside [0, 360].
"""
from __future__ import annotations

import logging
import math
from typing import Tuple

validation_logger = logging.getLogger("hpgl.validation")


class ValidationConstants:
    MIN_GRID_DIMENSION = 1
    MAX_GRID_DIMENSION = 10000000
    MAX_GRID_SIZE = 1000000000
    MIN_NEIGHBORS = 1
    MAX_NEIGHBORS = 1000
    DEFAULT_MAX_NEIGHBORS = 12
    MIN_RADIUS = 0.0
    MAX_RADIUS = 1000000.0
    MIN_SILL = 0.0
    MAX_SILL = 1e10
    MIN_NUGGET = 0.0
    MAX_NUGGET = 1e10
    MIN_RANGE = 0.0
    MAX_RANGE = 1e10
    MIN_ANGLE = 0.0
    MAX_ANGLE = 360.0
    MIN_PROBABILITY = 0.0
    MAX_PROBABILITY = 1.0
    MAX_INDICATORS = 256
    MIN_SEED = 0
    PROBABILITY_SUM_TOLERANCE = 0.01


class ValidationError(Exception):
    def __init__(self, message: str, parameter_name: str = "", severity: str = "error"):
        self.message = message
        self.parameter_name = parameter_name
        self.severity = severity
        super().__init__(f"{parameter_name}: {message}" if parameter_name else message)


class CriticalValidationError(ValidationError):
    def __init__(self, message: str, parameter_name: str = ""):
        super().__init__(message, parameter_name, "critical")


class ValidationWarning(ValidationError):
    def __init__(self, message: str, parameter_name: str = ""):
        super().__init__(message, parameter_name, "warning")


def _bad(x) -> bool:
    return math.isnan(x) or math.isinf(x)


class PathValidator:
    """File-path checks of the property readers and writers (validation.py:96-170)."""

    @staticmethod
    def validate_filepath(filename, must_exist: bool = False) -> str:
        import os
        import pathlib
        if not filename:
            raise CriticalValidationError("Filename cannot be empty", "filename")
        path_str = os.path.normpath(str(filename))
        if ".." in path_str.split(os.sep) or "../" in str(filename) or "..\\" in str(filename):
            raise CriticalValidationError(f"Path traversal detected in filename: {filename}", "filename")
        path = pathlib.Path(filename)
        try:
            resolved = path.resolve(strict=must_exist)
        except (OSError, RuntimeError) as e:
            raise CriticalValidationError(f"File does not exist: {filename}", "filename") from e
        if must_exist and not resolved.is_file():
            raise CriticalValidationError(f"Not a file: {filename}", "filename")
        return str(resolved)


class GridValidator:
    @staticmethod
    def validate_grid_dimensions(x: int, y: int, z: int) -> None:
        for v, axis in ((x, "x"), (y, "y"), (z, "z")):
            if v < ValidationConstants.MIN_GRID_DIMENSION or v > ValidationConstants.MAX_GRID_DIMENSION:
                raise CriticalValidationError(
                    f"Grid {axis.upper()} dimension {v} outside valid range "
                    f"[{ValidationConstants.MIN_GRID_DIMENSION}, {ValidationConstants.MAX_GRID_DIMENSION}]",
                    f"grid_{axis}")
        total = x * y * z
        if total > ValidationConstants.MAX_GRID_SIZE:
            raise CriticalValidationError(
                f"Total grid size {total} exceeds maximum of {ValidationConstants.MAX_GRID_SIZE}", "grid_size")


class ParameterValidator:
    @staticmethod
    def validate_radius(radius, name: str = "radius") -> Tuple:
        is_int = isinstance(radius, int) or (
            isinstance(radius, (tuple, list)) and len(radius) == 3 and all(isinstance(r, int) for r in radius))
        if isinstance(radius, (int, float)):
            rx = ry = rz = float(radius)
        elif isinstance(radius, (tuple, list)) and len(radius) == 3:
            rx, ry, rz = map(float, radius)
        else:
            raise CriticalValidationError(f"Radius must be a number or tuple of 3 numbers, got {type(radius)}", name)
        for i, r in enumerate((rx, ry, rz)):
            if _bad(r):
                raise CriticalValidationError(f"{name}[{i}] is NaN or infinite", name)
        if is_int:
            rx = int(rx) if rx.is_integer() else rx
            ry = int(ry) if ry.is_integer() else ry
            rz = int(rz) if rz.is_integer() else rz
        for i, r in enumerate((rx, ry, rz)):
            if float(r) < ValidationConstants.MIN_RADIUS:
                raise CriticalValidationError(
                    f"{name}[{i}] = {r} is less than minimum {ValidationConstants.MIN_RADIUS}", name)
            if float(r) > ValidationConstants.MAX_RADIUS:
                raise CriticalValidationError(
                    f"{name}[{i}] = {r} exceeds maximum {ValidationConstants.MAX_RADIUS}", name)
        return (rx, ry, rz)

    @staticmethod
    def validate_max_neighbors(max_neighbors: int) -> None:
        if max_neighbors < ValidationConstants.MIN_NEIGHBORS:
            raise CriticalValidationError(
                f"Max neighbors {max_neighbors} is less than minimum {ValidationConstants.MIN_NEIGHBORS}",
                "max_neighbors")
        if max_neighbors > ValidationConstants.MAX_NEIGHBORS:
            raise ValidationWarning(
                f"Max neighbors {max_neighbors} exceeds recommended maximum {ValidationConstants.MAX_NEIGHBORS}. "
                "Performance may be degraded.", "max_neighbors")

    @staticmethod
    def validate_covariance_parameters(sill, nugget, ranges=None, angles=None) -> None:
        if _bad(sill):
            raise CriticalValidationError("Sill is NaN or infinite", "sill")
        if sill < ValidationConstants.MIN_SILL:
            raise CriticalValidationError(f"Sill {sill} is less than minimum {ValidationConstants.MIN_SILL}", "sill")
        if sill > ValidationConstants.MAX_SILL:
            raise CriticalValidationError(f"Sill {sill} exceeds maximum {ValidationConstants.MAX_SILL}", "sill")
        if _bad(nugget):
            raise CriticalValidationError("Nugget is NaN or infinite", "nugget")
        if nugget < ValidationConstants.MIN_NUGGET:
            raise CriticalValidationError(
                f"Nugget {nugget} is less than minimum {ValidationConstants.MIN_NUGGET}", "nugget")
        if nugget > ValidationConstants.MAX_NUGGET:
            raise CriticalValidationError(f"Nugget {nugget} exceeds maximum {ValidationConstants.MAX_NUGGET}", "nugget")
        if nugget > sill:
            raise CriticalValidationError(f"Nugget {nugget} exceeds sill {sill} (nugget must be <= sill)", "nugget")
        if ranges is not None:
            if len(ranges) != 3:
                raise CriticalValidationError(f"Ranges must have 3 values, got {len(ranges)}", "ranges")
            for i, r in enumerate(ranges):
                if _bad(r):
                    raise CriticalValidationError(f"Range[{i}] is NaN or infinite", "ranges")
                if r < ValidationConstants.MIN_RANGE:
                    raise CriticalValidationError(
                        f"Range[{i}] = {r} is less than minimum {ValidationConstants.MIN_RANGE}", "ranges")
                if r > ValidationConstants.MAX_RANGE:
                    raise CriticalValidationError(
                        f"Range[{i}] = {r} exceeds maximum {ValidationConstants.MAX_RANGE}", "ranges")
        if angles is not None:
            if len(angles) != 3:
                raise CriticalValidationError(f"Angles must have 3 values, got {len(angles)}", "angles")
            for i, a in enumerate(angles):
                if _bad(a):
                    raise CriticalValidationError(f"Angle[{i}] is NaN or infinite", "angles")
                if a < ValidationConstants.MIN_ANGLE or a > ValidationConstants.MAX_ANGLE:
                    validation_logger.warning(
                        f"Angle[{i}] = {a} is outside typical range "
                        f"[{ValidationConstants.MIN_ANGLE}, {ValidationConstants.MAX_ANGLE}]")

    @staticmethod
    def validate_min_neighbors(min_neighbors: int, max_neighbors: int) -> None:
        if min_neighbors > max_neighbors:
            raise CriticalValidationError(
                f"Min neighbors {min_neighbors} exceeds max neighbors {max_neighbors}", "min_neighbors")
        if min_neighbors < 0:
            raise CriticalValidationError(f"Min neighbors {min_neighbors} is negative", "min_neighbors")

    @staticmethod
    def validate_correlation_coef(coef, name: str = "correlation_coef") -> None:
        if not isinstance(coef, (int, float)):
            raise CriticalValidationError(f"{name} must be a number, got {type(coef).__name__}", name)
        if math.isnan(coef) or math.isinf(coef):
            raise CriticalValidationError(f"{name} must be finite, got {coef}", name)
        if coef < -1.0 or coef > 1.0:
            raise CriticalValidationError(f"{name} must be in [-1, 1] range, got {coef}", name)

    @staticmethod
    def validate_variance(variance, name: str = "variance") -> None:
        if not isinstance(variance, (int, float)):
            raise CriticalValidationError(f"{name} must be a number, got {type(variance).__name__}", name)
        if math.isnan(variance) or math.isinf(variance):
            raise CriticalValidationError(f"{name} must be finite, got {variance}", name)
        if variance < 0:
            raise CriticalValidationError(f"{name} must be non-negative, got {variance}", name)

    @staticmethod
    def validate_seed(seed: int) -> None:
        if seed < ValidationConstants.MIN_SEED:
            validation_logger.warning(f"Seed value {seed} is negative")

    @staticmethod
    def validate_probability(prob: float, name: str = "probability") -> None:
        if _bad(prob):
            raise CriticalValidationError(f"{name} is NaN or infinite", name)
        if prob < ValidationConstants.MIN_PROBABILITY or prob > ValidationConstants.MAX_PROBABILITY:
            raise CriticalValidationError(
                f"{name} = {prob} outside valid range "
                f"[{ValidationConstants.MIN_PROBABILITY}, {ValidationConstants.MAX_PROBABILITY}]", name)

    @staticmethod
    def validate_probability_sum(probs) -> None:
        """The probabilities must sum to 1 within PROBABILITY_SUM_TOLERANCE (validation.py:522-543)."""
        prob_sum = sum(probs)
        if _bad(prob_sum):
            raise CriticalValidationError("Probability sum is NaN or infinite", "probabilities")
        diff = abs(prob_sum - 1.0)
        if diff > ValidationConstants.PROBABILITY_SUM_TOLERANCE:
            raise CriticalValidationError(
                f"Probabilities sum to {prob_sum}, expected 1.0 (difference: {diff})", "probabilities")

    @staticmethod
    def validate_indicator_count(count: int) -> None:
        if count <= 0:
            raise CriticalValidationError(f"Indicator count must be positive, got {count}", "indicator_count")
        if count > ValidationConstants.MAX_INDICATORS:
            raise CriticalValidationError(
                f"Indicator count {count} exceeds maximum {ValidationConstants.MAX_INDICATORS}", "indicator_count")
