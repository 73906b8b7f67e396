"""ctypes binding of ``libfv3core_b200.so`` (the C ABI in include/fv3core_b200.h).

The library is the only compute path: if it is missing or cannot be loaded,
importing an operator raises instead of falling back to anything else.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfv3core_b200.so")
# the FP64 build and the mixed-precision build (FP32 fields, FP64 column solves)
LIB_PATHS = {"f64": LIB_PATH, "f32": os.path.join(_HERE, "libfv3core_b200_f32.so")}

_libs = {}
# precision of each context, by its address (a context belongs to one build)
_ctx_precision = {}

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
    "fv3b_riem_solver3": [ctypes.c_int, D, D, D] + [P] * 14 + [P],
    "fv3b_riem_solver3_adjoint": [D, D, D] + [P] * 14 + [P],
    "fv3b_riem_solver_c_adjoint": [D, D, D] + [P] * 14 + [P],
    "fv3b_del2cubed_noalloc": [P, P, D, ctypes.c_int, P],
}

# entry points whose first argument is the context (fv3b_ctx*)
CTX_SIGNATURES = {
    "fv3b_c_sw": [P, P, P, P, P, P, P, P, P, P, P, P, P, D, ctypes.c_int, P, P, P],
    "fv3b_d_sw_setup": [P],
    "fv3b_d_sw": [P] * 24 + [D, P],
    "fv3b_update_dz_c": [P] * 6 + [D, P],
    "fv3b_update_dz_c_adjoint": [P] * 9 + [D, P],
    "fv3b_update_dz_d_setup": [P, ctypes.c_int],
    "fv3b_update_dz_d": [P] * 7 + [D, P],
    "fv3b_p_grad_c": [P] * 5 + [D, P],
    "fv3b_p_grad_c_adjoint": [P] * 8 + [D, P],
    "fv3b_nh_p_grad": [P] * 6 + [D, D, D, P],
    "fv3b_nh_p_grad_adjoint": [P] * 15 + [D, D, D, P],
    "fv3b_edge_pe": [P, P, D, P],
    "fv3b_pk3_halo": [P, P, D, D, P],
    "fv3b_edge_pe_adjoint": [P, P, P],
    "fv3b_pk3_halo_adjoint": [P, P, P, D, D, P],
    "fv3b_ray_fast": [P] * 5 + [D, D, D, D, ctypes.c_int, P],
    "fv3b_ray_fast_adjoint": [P] * 5 + [D, D, D, D, ctypes.c_int, P],
    "fv3b_del2cubed": [P, D, ctypes.c_int, P],
    "fv3b_del2cubed_adjoint": [P, D, ctypes.c_int, P],
    "fv3b_pkz_tempadjust": [P] * 6 + [D, ctypes.c_int, P],
    "fv3b_pkz_tempadjust_adjoint": [P] * 10 + [D, ctypes.c_int, P],
    "fv3b_halo_update_scalar": [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P],
    "fv3b_halo_update_vector": [P, P, ctypes.c_int, ctypes.c_int, P],
    "fv3b_synchronize_vector_interfaces": [P, P, ctypes.c_int, P],
    "fv3b_halo_update_scalar_adjoint": [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P],
    "fv3b_halo_update_vector_adjoint": [P, P, ctypes.c_int, ctypes.c_int, P],
    "fv3b_synchronize_vector_interfaces_adjoint": [P, P, ctypes.c_int, P],
    "fv3b_acoustics_setup": [P] * 6,
    "fv3b_acoustics": [P, P],
    "fv3b_ppm_flux": [ctypes.c_int, ctypes.c_int, P, P, P] + [ctypes.c_int] * 6 + [P],
    "fv3b_compute_preamble": [P] * 14 + [P],
    "fv3b_post_remap": [P] * 4 + [ctypes.c_int, P],
    "fv3b_adjust_negative_tracers": [P] * 11 + [ctypes.c_int, P],
    "fv3b_cubed_to_latlon": [P] * 8 + [ctypes.c_int, P],
    "fv3b_transport_create": [ctypes.c_int, P, P, ctypes.c_int, P],
    "fv3b_remap_setup": [P, P],
    "fv3b_lagrangian_to_eulerian": [P, P, P, D, D, D, D, ctypes.c_int, ctypes.c_int, P],
}

# entry points whose first argument is a transport object (fv3b_transport*),
# which belongs to the context it was created on
TRANSPORT_SIGNATURES = {
    "fv3b_transport_destroy": [],
    "fv3b_fvtp2d": [P] * 10 + [P],
    "fv3b_tracer_advection": [ctypes.c_int, P, P, P, P, P, P, D, P],
}

# entry points that return a pointer rather than a status
PTR_SIGNATURES = {
    "fv3b_acoustics_temporary": [ctypes.c_void_p, ctypes.c_char_p],
}


class DswConfig(ctypes.Structure):
    _fields_ = [(n, D) for n in ("dddmp", "d2_bg", "d2_bg_k1", "d2_bg_k2", "d4_bg", "ke_bg", "d_con", "vtdm4", "d_ext")] + [
        (n, I32)
        for n in (
            "nord", "n_sponge", "grid_type", "hord_dp", "hord_tm", "hord_mt", "hord_vt",
            "do_vort_damp", "hydrostatic", "do_f3d", "do_skeb", "inline_q", "convert_ke",
        )
    ]


class AcousticConfig(ctypes.Structure):
    _fields_ = [(n, D) for n in ("tau", "delt_max", "rf_cutoff", "p_fac")] + [
        (n, I32) for n in ("k_split", "n_split", "rf_fast", "breed_vortex_inline", "use_old_omega", "reserved")
    ]


DYCORE_FIELDS = ("u", "v", "w", "delz", "delp", "pt", "pe", "pk", "phis", "wsd", "omga", "ua", "va", "uc", "vc",
                 "mfxd", "mfyd", "cxd", "cyd", "pkz", "peln", "q_con", "diss_estd", "cappa")


class DycoreState(ctypes.Structure):
    _fields_ = [(n, P) for n in DYCORE_FIELDS] + [("mdt", D), ("akap", D), ("ptop", D), ("n_map", I32),
                                                  ("ks", I32)]


REMAP_TRACERS = ("qvapor", "qliquid", "qrain", "qice", "qsnow", "qgraupel", "qo3mr", "qsgs_tke")
REMAP_FIELDS = ("pt", "delp", "delz", "peln", "u", "v", "w", "ua", "va", "cappa", "q_con", "pkz", "pk", "pe", "ps")


class RemapConfig(ctypes.Structure):
    _fields_ = [(n, I32) for n in ("kord_tm", "kord_tr", "kord_wz", "kord_mt", "fill", "reserved")]


class RemapFields(ctypes.Structure):
    _fields_ = [("tracers", P * 8)] + [(n, P) for n in REMAP_FIELDS] + [("wsd", P), ("qcld", P), ("dp1", P),
                                                                          ("hs", P)]


SAT_ADJUST_DOUBLES = ("sat_adj0", "ql_gen", "qs_mlt", "ql0_max", "t_sub", "qi_gen", "qi_lim", "qi0_max", "dw_ocean",
                      "dw_land", "cld_min", "tau_i2s", "tau_v2l", "tau_r2g", "tau_l2r", "tau_l2v", "tau_imlt",
                      "tau_smlt")
SAT_ADJUST_INTS = ("icloud_f", "rad_snow", "rad_rain", "rad_graupel", "tintqs", "hydrostatic")


class SatAdjustConfig(ctypes.Structure):
    _fields_ = [(n, D) for n in SAT_ADJUST_DOUBLES] + [(n, I32) for n in SAT_ADJUST_INTS]


def lib(precision="f64"):
    if precision not in LIB_PATHS:
        raise ValueError(f"precision must be one of {sorted(LIB_PATHS)}, got {precision!r}")
    if precision not in _libs:
        path = LIB_PATHS[precision]
        if not os.path.exists(path):
            raise ImportError(
                f"{path} is missing: build it with `python -m fv3core_b200.build` "
                "(there is no CPU fallback)"
            )
        L = ctypes.CDLL(path)
        L.fv3b_last_error.restype = ctypes.c_char_p
        L.fv3b_version.restype = ctypes.c_char_p
        L.fv3b_launch_count.restype = ctypes.c_longlong
        L.fv3b_launch_count.argtypes = []
        L.fv3b_set_launch_shape.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.fv3b_set_launch_shape.restype = ctypes.c_int
        L.fv3b_get_launch_shape.argtypes = [ctypes.POINTER(ctypes.c_int)] * 3
        L.fv3b_get_launch_shape.restype = None
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
        for name, args in TRANSPORT_SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = [ctypes.c_void_p] + args
            fn.restype = ctypes.c_int
        for name, args in PTR_SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_void_p
        _libs[precision] = L
    return _libs[precision]


def register_context(ctx, precision):
    _ctx_precision[ctx.value] = precision


def context_precision(ctx):
    value = ctx.value if isinstance(ctx, ctypes.c_void_p) else ctx
    return _ctx_precision.get(value, "f64")


def call(name, dims, *args, precision="f64"):
    L = lib(precision)
    rc = getattr(L, name)(ctypes.byref(dims), *args)
    if rc != 0:
        msg = L.fv3b_last_error().decode()
        raise ERRORS.get(rc, RuntimeError)(f"{name} failed ({rc}): {msg}")


def call_ctx(name, ctx, *args):
    L = lib(context_precision(ctx))
    rc = getattr(L, name)(ctx, *args)
    if rc != 0:
        msg = L.fv3b_last_error().decode()
        raise ERRORS.get(rc, RuntimeError)(f"{name} failed ({rc}): {msg}")


def call_precision(name, precision, *args):
    """Call entry point ``name`` of the ``precision`` build with its own
    argument list; raise the reference's exception type on failure."""
    L = lib(precision)
    rc = getattr(L, name)(*args)
    if rc != 0:
        msg = L.fv3b_last_error().decode()
        raise ERRORS.get(rc, RuntimeError)(f"{name} failed ({rc}): {msg}")


def exported_symbols():
    return ["fv3b_last_error", "fv3b_version", "fv3b_launch_count", "fv3b_set_launch_shape", "fv3b_get_launch_shape",
            "fv3b_ctx_create", "fv3b_ctx_create_batched", "fv3b_ctx_destroy", "fv3b_generate_grid"] + [
        k for k, v in SIGNATURES.items() if v is not None
    ] + list(CTX_SIGNATURES) + list(PTR_SIGNATURES) + list(TRANSPORT_SIGNATURES)


def launch_count(precision="f64"):
    """Kernel launches issued by the library so far."""
    return int(lib(precision).fv3b_launch_count())


def set_launch_shape(box_x, box_y, col, precision="f64"):
    rc = lib(precision).fv3b_set_launch_shape(int(box_x), int(box_y), int(col))
    if rc != 0:
        raise ValueError(lib(precision).fv3b_last_error().decode())


def get_launch_shape(precision="f64"):
    v = [ctypes.c_int(), ctypes.c_int(), ctypes.c_int()]
    lib(precision).fv3b_get_launch_shape(*[ctypes.byref(x) for x in v])
    return tuple(x.value for x in v)
