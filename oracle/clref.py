"""ctypes binding of oracle/_ref/libclref.so -- the reference's own OpenCL C
kernels compiled as C++ for the host (see build_ref.py).

TEST INFRASTRUCTURE ONLY: used to pin the oracle restatement against the
reference kernel code, and as the CPU baseline of bench.py --impl reference.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libclref.so")
_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def set_threads(n):
    """Spread every later kernel call over n host threads (1 = in order)."""
    lib().clref_set_threads(ctypes.c_int(int(n)))


def _sfx(dt):
    return "f32" if np.dtype(dt) == np.float32 else "f64"


def _S(dt):
    return ctypes.c_float if np.dtype(dt) == np.float32 else ctypes.c_double


def P(a):
    """pointer argument (None -> NULL)"""
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def call(name, dtype, *args):
    """Call clref_<name>_<sfx>; python floats become REAL, ints stay int."""
    fn = getattr(lib(), f"clref_{name}_{_sfx(dtype)}")
    S = _S(dtype)
    cargs = []
    for a in args:
        if isinstance(a, np.ndarray):
            cargs.append(P(a))
        elif a is None:
            cargs.append(None)
        elif isinstance(a, float):
            cargs.append(S(a))
        elif isinstance(a, (int, np.integer)):
            cargs.append(ctypes.c_int(int(a)))
        else:
            raise TypeError(type(a))
    fn(*cargs)
