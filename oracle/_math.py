"""Transcendental functions of the oracle -- TEST INFRASTRUCTURE ONLY.

By default ``exp``, ``log`` and ``power`` are numpy's, so the oracle repeats
the reference's numpy-backend arithmetic bit for bit (pinned by the golden
fixtures).  Inside ``device_math()`` they are the host build of the kernels'
own exp/log/pow (``fv3core_b200/csrc/fmath.h`` through
``oracle/portable_math.cpp``), so that the CUDA path can be checked to the
last bit: the acoustic substep amplifies last-place differences of these
functions (cancellation in the Riemann solvers and the pressure gradient),
and numpy's exp and power are not correctly rounded, so no other
implementation can reproduce them exactly.  The functions themselves are
checked against correctly rounded values in ``tests/test_fmath.py``.
``host_sin``/``host_log`` serve per-level constants that the library
computes on the host with the C library.
"""
import contextlib
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "portable_math.cpp")
HEADER = os.path.join(os.path.dirname(HERE), "fv3core_b200", "csrc", "fmath.h")
LIB = os.path.join(HERE, "_build", "libportable_math.so")

_lib = None
_device = False


def build():
    """Compile the host helper (g++, no implicit FMA contraction; the header's
    explicit fma() calls are exactly rounded in libm) if stale."""
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    newest = max(os.path.getmtime(SRC), os.path.getmtime(HEADER))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        subprocess.check_call(["g++", "-O2", "-ffp-contract=off", "-fno-fast-math", "-std=c++17", "-shared", "-fPIC",
                               "-o", LIB, SRC])
    return LIB


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        for name in ("pm_exp", "pm_log"):
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long]
        L.pm_pow.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long]
        _lib = L
    return _lib


def _unary(name, x):
    xa = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
    out = np.empty_like(xa)
    getattr(_load(), name)(xa.ctypes.data, out.ctypes.data, xa.size)
    return out if np.ndim(x) else float(out.reshape(-1)[0])


def exp(x):
    return _unary("pm_exp", x) if _device else np.exp(x)


def log(x):
    return _unary("pm_log", x) if _device else np.log(x)


def power(x, p):
    if not _device:
        return np.power(x, p)
    xa, pa = np.broadcast_arrays(np.asarray(x, dtype=np.float64), np.asarray(p, dtype=np.float64))
    xa, pa = np.ascontiguousarray(xa), np.ascontiguousarray(pa)
    out = np.empty_like(xa)
    _load().pm_pow(xa.ctypes.data, pa.ctypes.data, out.ctypes.data, xa.size)
    return out if out.ndim else float(out.reshape(-1)[0])


def host_sin(x):
    """Per-level constants: numpy's sin, or in device-math mode the C
    library's (what the library's host setup code calls)."""
    if not _device:
        return np.sin(x)
    import math

    return np.array([math.sin(v) for v in np.ravel(x)]).reshape(np.shape(x))


def host_log(x):
    if not _device:
        return np.log(x)
    import math

    return np.array([math.log(v) for v in np.ravel(x)]).reshape(np.shape(x))


@contextlib.contextmanager
def device_math():
    """Use the kernels' exp/log/pow inside the block."""
    global _device
    old = _device
    _device = True
    try:
        yield
    finally:
        _device = old
