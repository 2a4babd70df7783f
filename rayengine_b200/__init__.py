"""B200-native RayEngine ray-query path: rope kd-tree traversal, fBm/Perlin
noise and exact-SDF sphere tracing behind a C ABI (include/rayengine_b200.h).
"""
from ._lib import LIB_PATH, RayEngineError  # noqa: F401
from .api import *  # noqa: F401,F403
from . import configs  # noqa: F401

__version__ = "0.1.0"
