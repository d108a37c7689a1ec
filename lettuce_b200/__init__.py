"""lettuce_b200: B200-native pure-gauge SU(3) hot path of timo-eichhorn/Lettuce.

The compute lives in liblettuce_b200.so (hand-written sm_100a CUDA behind the C ABI declared
in include/lettuce_b200.h); this package is the Python mirror of the reference's call surface.
"""
from ._lib import LIB_PATH, LettuceError, declared_symbols, lib  # noqa: F401
from .api import *  # noqa: F401,F403
from .api import __all__ as _api_all

__all__ = ["LIB_PATH", "LettuceError", "declared_symbols", "lib", *_api_all]
