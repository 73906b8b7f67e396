"""ctypes binding of ``libfv3core_b200.so`` (the C ABI in include/fv3core_b200.h).

The library is the only compute path: if it is missing or cannot be loaded,
importing an operator raises instead of falling back to anything else.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfv3core_b200.so")

_lib = None

P = ctypes.c_void_p
D = ctypes.c_double
I32 = ctypes.c_int32

ERRORS = {
    1: ValueError,
    2: RuntimeError,
    3: NotImplementedError,
    4: TimeoutError,
}


class GridDims(ctypes.Structure):
    _fields_ = [("npx", I32), ("n_halo", I32), ("npz", I32), ("reserved", I32)]


# name -> argument types after the leading dims pointer
SIGNATURES = {
    "fv3b_riem_solver_c": [D, D, D, P, P, P, P, P, P, P, P, P, P],
}

# entry points whose first argument is the context (fv3b_ctx*)
CTX_SIGNATURES = {
    "fv3b_c_sw": [P, P, P, P, P, P, P, P, P, P, P, P, P, D, ctypes.c_int, P, P, P],
    "fv3b_d_sw_setup": [P],
    "fv3b_d_sw": [P] * 24 + [D, P],
}


class DswConfig(ctypes.Structure):
    _fields_ = [(n, D) for n in ("dddmp", "d2_bg", "d2_bg_k1", "d2_bg_k2", "d4_bg", "ke_bg", "d_con", "vtdm4", "d_ext")] + [
        (n, I32)
        for n in (
            "nord", "n_sponge", "grid_type", "hord_dp", "hord_tm", "hord_mt", "hord_vt",
            "do_vort_damp", "hydrostatic", "do_f3d", "do_skeb", "inline_q", "convert_ke",
        )
    ]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m fv3core_b200.build` "
                "(there is no CPU fallback)"
            )
        L = ctypes.CDLL(LIB_PATH)
        L.fv3b_last_error.restype = ctypes.c_char_p
        L.fv3b_version.restype = ctypes.c_char_p
        for name, args in SIGNATURES.items():
            if args is None:
                continue
            fn = getattr(L, name)
            fn.argtypes = [ctypes.POINTER(GridDims)] + args
            fn.restype = ctypes.c_int
        for name, args in CTX_SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = [ctypes.c_void_p] + args
            fn.restype = ctypes.c_int
        _lib = L
    return _lib


def call(name, dims, *args):
    rc = getattr(lib(), name)(ctypes.byref(dims), *args)
    if rc != 0:
        msg = lib().fv3b_last_error().decode()
        raise ERRORS.get(rc, RuntimeError)(f"{name} failed ({rc}): {msg}")


def call_ctx(name, ctx, *args):
    rc = getattr(lib(), name)(ctx, *args)
    if rc != 0:
        msg = lib().fv3b_last_error().decode()
        raise ERRORS.get(rc, RuntimeError)(f"{name} failed ({rc}): {msg}")


def exported_symbols():
    return ["fv3b_last_error", "fv3b_version", "fv3b_ctx_create", "fv3b_ctx_destroy"] + [
        k for k, v in SIGNATURES.items() if v is not None
    ] + list(CTX_SIGNATURES)
