"""geo_bsd — HPGL's kriging API on a B200-native engine (libhpgl_b200.so)."""
from .geo import *  # noqa: F401,F403
from .geo import __all__  # noqa: F401
from .hpgl_wrap import last_stats  # noqa: F401
