"""umagnus_b200 -- B200-native (sm_100a) effective-field + LLG hot path of uMagNUS.

The device work lives in libumagnus_b200.so (C-ABI in include/umagnus_b200.h).
`opencl` mirrors the reference's device-op package, `engine` its simulation
loop.  There is no CPU fallback.
"""
from ._lib import UmagError, load  # noqa: F401

__version__ = "1.0"
