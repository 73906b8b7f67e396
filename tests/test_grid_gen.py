"""Device-side grid generation (fv3b_generate_grid, csrc/grid_gen.h): the
point functions compiled for the host against the numpy generator
(fv3core_b200/grid.py) on the CPU, and the device build against the numpy
generator on the GPU."""
import ctypes
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from fv3core_b200 import constants
from fv3core_b200.grid import LATTICES, CubedSphereGrid
from fv3core_b200.grid_device import EDGE_NAMES, GRID_FIELD_NAMES

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host compiler")
    so = str(tmp_path_factory.mktemp("grid_gen") / "grid_gen_host.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", so,
                           os.path.join(ROOT, "tests", "native", "grid_gen_host.cpp")])
    return ctypes.CDLL(so)


def _host_fields(lib, n, h=3, lattice=0):
    m = n + 2 * h + 1
    F = np.zeros((len(GRID_FIELD_NAMES), 6, m, m))
    E = np.zeros((4, 6, n + 1))
    A = np.zeros(72)
    S = np.zeros(4)
    lib.grid_gen_host(n, h, lattice, ctypes.c_double(constants.RADIUS), ctypes.c_double(constants.OMEGA), _ptr(F),
                      _ptr(E), _ptr(A), _ptr(S))
    return F, E, A.reshape(6, 4, 3), S


def _field_err(x, ref, skip=None):
    """Largest difference relative to the field's largest magnitude; NaN
    positions must agree.  Points where ``skip`` is set are left out."""
    if skip is not None:
        x, ref = np.where(skip, 0.0, x), np.where(skip, 0.0, ref)
    assert np.array_equal(np.isnan(x), np.isnan(ref))
    scale = max(float(np.nanmax(np.abs(ref))), 1e-300)
    return float(np.nanmax(np.abs(np.where(np.isnan(ref), 0.0, x - ref)))) / scale


def _degenerate(g):
    """[6, m, m] mask of the points next to the cube's vertices where the
    halo lattice folds onto itself: a corner point with an edge to a point
    it coincides with up to rounding (dx or dy below 1 m; the rest are
    40+ km at C384), or a cell of such points (area below 1 m^2).  The
    values there (lengths of 1e-9 m and their reciprocals near 1e9, angles
    between tangents towards a coinciding point, the ratios built on them)
    are rounding noise, which differs between the device's and the host's
    trigonometric functions; the stencils never use them (the cube-corner
    rules fill those points).  Checked to lie within the corner blocks
    widened by the vertex's own row and column (i <= h or i >= h + n, the
    same for j)."""
    h, n, m = g.halo, g.n, g.n + 2 * g.halo + 1
    dx, dy, area = (np.asarray(getattr(g, k)) for k in ("dx", "dy", "area"))
    ii, jj = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    bx = (dx < 1.0) & (ii < m - 1)
    by = (dy < 1.0) & (jj < m - 1)
    mask = bx | by | ((area < 1.0) & (ii < m - 1) & (jj < m - 1))
    mask[:, 1:, :] |= bx[:, :-1, :]
    mask[:, :, 1:] |= by[:, :, :-1]
    _, i, j = np.nonzero(mask)
    assert np.all(((i <= h) | (i >= h + n)) & ((j <= h) | (j >= h + n)))
    return mask


def test_field_order_matches_the_header():
    """GRID_FIELD_NAMES, the enum of csrc/grid_gen.h and the list in
    include/fv3core_b200.h name the same fields in the same order."""
    src = open(os.path.join(ROOT, "fv3core_b200", "csrc", "grid_gen.h")).read()
    enum = src.split("enum GridField")[1].split("};")[0]
    names = [x.lower() for x in re.findall(r"\bGF_(\w+)", enum) if x != "COUNT"]
    assert [{"fc": "fC"}.get(x, x) for x in names] == GRID_FIELD_NAMES
    hdr = open(os.path.join(ROOT, "include", "fv3core_b200.h")).read()
    block = hdr.split("fv3b_generate_grid:")[1].split("edge[e]")[0].split("in this order:")[1]
    listed = block.replace("*", " ").replace(";", " ").split()
    expanded = []
    for w in listed:
        m = re.fullmatch(r"(\w+?)(\d)\.\.(\d)", w)
        expanded += [f"{m.group(1)}{k}" for k in range(int(m.group(2)), int(m.group(3)) + 1)] if m else [w]
    assert expanded == GRID_FIELD_NAMES
    assert f"#define FV3B_GRID_NFIELDS {len(GRID_FIELD_NAMES)}" in hdr


@pytest.mark.parametrize("lattice", ["equiangular", "equidistant"])
@pytest.mark.parametrize("n", [7, 12, 48])
def test_host_build_matches_numpy_generator(host_lib, n, lattice):
    """Every field of the point functions, compiled for the host, equals the
    numpy generator's to rounding, on both lattices: 1e-13 of the field's
    largest magnitude (measured 4e-16), the A->B edge weights and the area
    extremes to 1e-13 relative, a2b_ord4's corner ratios (a difference
    quotient of two close distances) to 1e-12 relative."""
    F, E, A, S = _host_fields(host_lib, n, lattice=LATTICES.index(lattice))
    g = CubedSphereGrid(n, 3, lattice=lattice)
    for k, name in enumerate(GRID_FIELD_NAMES):
        assert _field_err(F[k], np.asarray(getattr(g, name))) <= 1e-13, name
    for e, name in enumerate(EDGE_NAMES):
        ref = np.asarray(getattr(g, name))
        assert np.max(np.abs(E[e] - ref) / np.abs(ref)) <= 1e-13, name
    assert np.max(np.abs(A - g.a2b_extrap) / np.abs(g.a2b_extrap)) <= 1e-12
    ref = np.array([g.da_min, g.da_max, g.da_min_c, g.da_max_c])
    assert np.max(np.abs(S - ref) / ref) <= 1e-13


@pytest.mark.parametrize("n", [12, 48])
def test_equidistant_lattice_is_the_reference_grid_type_0(n):
    """The equidistant lattice is the reference's grid_type 0 (gnomonic_ed):
    tile 0's compute-domain corners, their lengths, the cell areas and the
    cell-centre latitudes against the reference's own face and metric
    functions (tests/golden/gnomonic_ed_c*.npz, made by make_golden.py):
    corners to 1e-14, lengths to 1e-13 relative, areas to 1e-11 relative
    (the reference's area sums four spherical angles, good to 1e-12 by its
    own account: 2e-12 here at C48), centre latitudes to 1e-14, and the
    angles at the edge midpoints (cos_sg1..4) and the interior corners
    (cosa) to 1e-12 (measured 8e-14; the reference goes through lon/lat).
    The equiangular lattice differs from it by up to 20 % in lengths."""
    d = np.load(os.path.join(ROOT, "tests", "golden", f"gnomonic_ed_c{n}.npz"))
    h = 3
    lon, lat = d["lon"], d["lat"]
    ref_corners = np.stack([np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)], axis=-1)
    for lattice, agrees in (("equidistant", True), ("equiangular", False)):
        g = CubedSphereGrid(n, h, lattice=lattice)
        dx = np.asarray(g.dx)[0, h:h + n, h:h + n + 1]
        rel = np.max(np.abs(dx / d["dx"] - 1.0))
        if not agrees:
            assert rel > 0.1
            continue
        assert np.max(np.abs(g.corners[0, h:h + n + 1, h:h + n + 1] - ref_corners)) <= 1e-14
        assert rel <= 1e-13
        assert np.max(np.abs(np.asarray(g.dy)[0, h:h + n + 1, h:h + n] / d["dy"] - 1.0)) <= 1e-13
        assert np.max(np.abs(np.asarray(g.area)[0, h:h + n, h:h + n] / d["area"] - 1.0)) <= 1e-11
        assert np.max(np.abs(np.asarray(g.lat_a)[0, h:h + n, h:h + n] - d["lat_a"])) <= 1e-14
        for k in range(1, 5):
            cs = np.asarray(getattr(g, f"cos_sg{k}"))[0, h:h + n, h:h + n]
            assert np.max(np.abs(cs - d[f"cos_sg{k}"])) <= 1e-12, k
        assert np.max(np.abs(np.asarray(g.cosa)[0, h + 1:h + n, h + 1:h + n] - d["cosa_interior"])) <= 1e-12


def test_entry_point_rejects_bad_arguments_without_gpu():
    """fv3b_generate_grid checks its arguments before any CUDA call, in the
    order of the Python binding: a bad halo, lattice or radius each comes
    back as FV3B_ERR_ARGUMENT naming it."""
    from fv3core_b200 import _lib
    from fv3core_b200.grid_device import GridFields, bind

    L = bind()
    out = GridFields()
    for k in range(len(GRID_FIELD_NAMES)):
        out.field[k] = 16
    for e in range(4):
        out.edge[e] = 16
    out.a2b_extrap = out.scalars = 16
    for args, word in (((12, 99, 0, 6.4e6), "halo"), ((12, 3, 5, 6.4e6), "lattice"), ((12, 3, 1, -1.0), "radius")):
        rc = L.fv3b_generate_grid(*args, 7.3e-5, ctypes.byref(out), None)
        assert rc == 1, args
        assert word in L.fv3b_last_error().decode(), args
    assert _lib.exported_symbols().count("fv3b_generate_grid") == 1


@pytest.mark.gpu
@pytest.mark.parametrize("n", [12, 48])
def test_device_grid_matches_numpy_generator(n):
    """fv3b_generate_grid on the GPU against the numpy generator, away from
    the degenerate points at the cube's vertices (``_degenerate``): 2-D
    fields to 1e-12 of the field's largest magnitude (the device's
    trigonometric functions may differ from the host's by an ulp, which the
    smallest dual cells next to the vertices amplify to 2e-13 in rarea_c),
    the edge weights, corner ratios and area extremes to 1e-12 relative."""
    import torch

    from fv3core_b200.grid_device import DeviceGrid

    d = DeviceGrid(n, 3)
    torch.cuda.synchronize()
    g = CubedSphereGrid(n, 3)
    skip = _degenerate(g)
    for name in GRID_FIELD_NAMES:
        x = getattr(d, name).cpu().numpy().transpose(0, 2, 1)  # [6, j, i] -> [6, i, j]
        assert _field_err(x, np.asarray(getattr(g, name)), skip) <= 1e-12, name
    for name in EDGE_NAMES:
        ref = np.asarray(getattr(g, name))
        assert np.max(np.abs(getattr(d, name).cpu().numpy() - ref) / np.abs(ref)) <= 1e-12, name
    assert np.max(np.abs(d.a2b_extrap.cpu().numpy() - g.a2b_extrap) / np.abs(g.a2b_extrap)) <= 1e-12
    for name in ("da_min", "da_max", "da_min_c", "da_max_c"):
        assert abs(getattr(d, name) - getattr(g, name)) <= 1e-12 * getattr(g, name), name


@pytest.mark.gpu
def test_grid_data_from_device_grid():
    """GridData built from the device-generated grid holds the same metric
    tensors as GridData built from the numpy grid (to rounding), and its
    context runs a stage: the del-2 filter of one field gives the same
    result to 1e-12."""
    import torch

    from fv3core_b200.grid_data import METRIC_FIELDS, GridData
    from fv3core_b200.grid_device import DeviceGrid

    n, nz = 24, 6
    grid = CubedSphereGrid(n, 3)
    skip = _degenerate(grid).transpose(0, 2, 1)  # the kernels' [6, j, i] layout
    a = GridData(grid, nz)
    b = GridData(DeviceGrid(n, 3), nz)
    try:
        for name in METRIC_FIELDS:
            x, y = a.tensors[name].cpu().numpy(), b.tensors[name].cpu().numpy()
            assert _field_err(y, x, skip if x.shape == skip.shape else None) <= 1e-12, name
        assert abs(a.da_min - b.da_min) <= 1e-12 * a.da_min
        from fv3core_b200.stencil import StencilConfig, StencilFactory
        from fv3core_b200.stencils.del2cubed import HyperdiffusionDamping
        from fv3core_b200.storage import to_device, to_host

        rng = np.random.default_rng(4)
        q0 = rng.standard_normal((6, n + 7, n + 7, nz + 1))
        out = []
        for gd in (a, b):
            sf = StencilFactory(StencilConfig(), gd.grid_indexing)
            q = to_device(q0)
            HyperdiffusionDamping(sf, gd, gd.rarea, 3)(q, 0.2 * a.da_min)
            torch.cuda.synchronize()
            out.append(to_host(q))
        h = 3
        sl = (slice(None), slice(h, h + n), slice(h, h + n), slice(0, nz))
        assert _field_err(out[1][sl], out[0][sl]) <= 1e-12
    finally:
        a.close()
        b.close()
