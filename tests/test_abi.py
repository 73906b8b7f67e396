"""The C ABI: the library loads without a GPU, exports every function that
include/fv3core_b200.h declares, and the ctypes mirrors of its structs have
the C layout (checked against a host-compiled probe of the header)."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fv3core_b200.h")


def _declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fv3b_\w+)\s*\(", text)))


def test_header_declares_the_entry_points():
    names = _declared_functions()
    assert "fv3b_acoustics" in names and "fv3b_c_sw" in names and len(names) >= 25


def test_library_exports_every_declared_function():
    from fv3core_b200 import _lib

    L = _lib.lib()
    missing = [n for n in _declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_every_declared_function():
    from fv3core_b200 import _lib

    bound = set(_lib.exported_symbols())
    assert set(_declared_functions()) <= bound, set(_declared_functions()) - bound


def test_version_and_error_reporting_without_gpu():
    from fv3core_b200 import _lib

    L = _lib.lib()
    assert L.fv3b_version().startswith(b"fv3core_b200")
    # a null context is rejected on the host, before any CUDA call
    rc = L.fv3b_edge_pe(None, None, None, 0.0, None)
    assert rc == 1 and b"null argument" in L.fv3b_last_error()


def test_adjoint_entry_points_reject_bad_arguments_without_gpu():
    import ctypes

    from fv3core_b200 import _lib

    L = _lib.lib()
    # null context or field: rejected on the host before any CUDA call
    for name, n_ptr in (("fv3b_p_grad_c_adjoint", 8), ("fv3b_update_dz_c_adjoint", 9)):
        rc = getattr(L, name)(None, *([None] * n_ptr), 1.0, None)
        assert rc == 1 and b"null argument" in L.fv3b_last_error(), name
    null_calls = {
        "fv3b_nh_p_grad_adjoint": [None] * 15 + [1.0, 1.0, 0.28, None],
        "fv3b_halo_update_scalar_adjoint": [None, 1, 3, 1, None],
        "fv3b_halo_update_vector_adjoint": [None, None, 0, 1, None],
        "fv3b_synchronize_vector_interfaces_adjoint": [None, None, 1, None],
        "fv3b_edge_pe_adjoint": [None, None, None],
        "fv3b_pk3_halo_adjoint": [None, None, None, 1.0, 0.28, None],
        "fv3b_ray_fast_adjoint": [None] * 5 + [1.0, 1.0, 1.0, 1.0, 0, None],
        "fv3b_del2cubed_adjoint": [None, 1.0, 3, None],
        "fv3b_pkz_tempadjust_adjoint": [None] * 10 + [1.0, 1, None],
    }
    for name, args in null_calls.items():
        rc = getattr(L, name)(None, *args)
        assert rc == 1 and b"null argument" in L.fv3b_last_error(), name
    # the column adjoints: nulls, then too few levels, then too many
    buf = ctypes.create_string_buffer(8)
    ptrs = [ctypes.addressof(buf)] * 14
    for name in ("fv3b_riem_solver3_adjoint", "fv3b_riem_solver_c_adjoint"):
        dims = _lib.GridDims(12, 3, 8, 0)
        rc = getattr(L, name)(ctypes.byref(dims), 1.0, 1.0, 0.05, *([None] * 14), None)
        assert rc == 1 and b"null argument" in L.fv3b_last_error(), name
        for npz in (2, 128):
            dims = _lib.GridDims(12, 3, npz, 0)
            rc = getattr(L, name)(ctypes.byref(dims), 1.0, 1.0, 0.05, *ptrs, None)
            assert rc == 1 and b"npz must be in 3..127" in L.fv3b_last_error(), (name, npz)


def test_oversized_grid_is_rejected_before_any_cuda_call():
    import ctypes

    from fv3core_b200 import _lib

    L = _lib.lib()
    L.fv3b_ctx_create.argtypes = [ctypes.POINTER(_lib.GridDims), ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    L.fv3b_ctx_create.restype = ctypes.c_int
    # a 3-D field of 6 x 126 x 4103^2 elements does not fit 32-bit offsets
    dims = _lib.GridDims(4096, 3, 125, 0)
    metrics = ctypes.create_string_buffer(4096)
    out = ctypes.c_void_p()
    rc = L.fv3b_ctx_create(ctypes.byref(dims), metrics, ctypes.byref(out))
    assert rc == 1 and b"2^31" in L.fv3b_last_error()


def test_launch_shape_setting_without_gpu():
    from fv3core_b200 import _lib

    for precision in ("f64", "f32"):
        default = _lib.get_launch_shape(precision)
        assert default == (32, 4, 128)
        _lib.set_launch_shape(64, 2, 256, precision=precision)
        assert _lib.get_launch_shape(precision) == (64, 2, 256)
        for bad in [(48, 4, 128), (32, 64, 128), (32, 4, 100), (32, 0, 128)]:
            with pytest.raises(ValueError):
                _lib.set_launch_shape(*bad, precision=precision)
        assert _lib.get_launch_shape(precision) == (64, 2, 256)
        _lib.set_launch_shape(*default, precision=precision)


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("no host compiler")
    src = tmp_path_factory.mktemp("abi") / "probe.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "fv3core_b200.h"\n'
        "int main(void) {\n"
        '  printf("fv3b_grid_dims %zu\\n", sizeof(fv3b_grid_dims));\n'
        '  printf("fv3b_metrics %zu %zu\\n", sizeof(fv3b_metrics), offsetof(fv3b_metrics, da_min));\n'
        '  printf("fv3b_dsw_config %zu\\n", sizeof(fv3b_dsw_config));\n'
        '  printf("fv3b_acoustic_config %zu\\n", sizeof(fv3b_acoustic_config));\n'
        '  printf("fv3b_dycore_state %zu %zu\\n", sizeof(fv3b_dycore_state), offsetof(fv3b_dycore_state, n_map));\n'
        "  return 0;\n}\n"
    )
    exe = str(src.with_suffix(""))
    subprocess.check_call(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), "-o", exe, str(src)])
    out = subprocess.check_output([exe], text=True)
    return {line.split()[0]: [int(x) for x in line.split()[1:]] for line in out.splitlines()}


def test_struct_layouts_match_ctypes(c_layout):
    from fv3core_b200 import _lib
    from fv3core_b200.grid_data import Metrics

    assert c_layout["fv3b_grid_dims"] == [ctypes.sizeof(_lib.GridDims)]
    assert c_layout["fv3b_metrics"] == [ctypes.sizeof(Metrics), Metrics.da_min.offset]
    assert c_layout["fv3b_dsw_config"] == [ctypes.sizeof(_lib.DswConfig)]
    assert c_layout["fv3b_acoustic_config"] == [ctypes.sizeof(_lib.AcousticConfig)]
    assert c_layout["fv3b_dycore_state"] == [ctypes.sizeof(_lib.DycoreState), _lib.DycoreState.n_map.offset]
