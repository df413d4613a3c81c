"""B200-native UPBP renderer (unified points, beams and paths).

The render path runs in libupbp_b200.so (hand-written sm_100a CUDA behind the
C ABI in include/upbp.h); `upbp.Renderer` drives it from Python.
"""
from . import scenes  # noqa: F401
