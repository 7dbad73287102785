"""geo_bsd — HPGL's kriging API on a B200-native engine (libhpgl_b200.so)."""
from .geo import *  # noqa: F401,F403
from .geo import __all__  # noqa: F401
from .hpgl_wrap import last_stats  # noqa: F401
from .cdf import CdfData, calc_cdf  # noqa: F401
from .sgs import sgs_simulation  # noqa: F401
from .sis import sis_simulation  # noqa: F401
from . import tune as _tune

_tune._load_default()  # the solve-kernel tuning cache (geo_bsd/tune_cache.json)
