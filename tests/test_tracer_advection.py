"""TracerAdvection (tracer_2d_1l.py) with the ord-8 PPM of hord_tr = 8, and
the stand-alone FiniteVolumeTransport and X/YPiecewiseParabolic operators:
the oracle against the reference's own output (a golden run of six
TracerAdvection instances with a threaded halo exchange), the CUDA path
against the oracle."""
import os

import numpy as np
import pytest

import cases
import oracle_runs
from metrics import parity_err

HERE = os.path.dirname(os.path.abspath(__file__))
H = 3
FIELDS = ("tracers", "dp1", "mfxd", "mfyd", "cxd", "cyd")


def _golden():
    g = np.load(os.path.join(HERE, "golden", "tracer_advection.npz"))
    n, nz, seed = int(g["arg_n"]), int(g["arg_nz"]), int(g["arg_seed"])
    return g, n, nz, cases.tracer_case(n, nz, seed)


def _same(a, b):
    return np.array_equal(a, b, equal_nan=True)


def test_oracle_matches_reference_golden():
    """Every storage point of the tracers and of the in-place updated
    inputs, bit for bit."""
    g, n, nz, case = _golden()
    out = oracle_runs.run_tracer_advection(case, n, nz)
    for k in FIELDS:
        assert _same(out[k], g[k]), k


def test_tracers_stay_within_their_initial_bounds():
    """The ord-8 limiter is monotone: on the golden case every advected
    tracer stays inside [0, 1e-2), its initial range."""
    g, n, nz, _ = _golden()
    q = g["tracers"][:, :, H:H + n, H:H + n, :nz]
    assert q.min() >= 0.0 and q.max() < 1.0e-2


def test_ord8_flux_of_a_constant_is_the_constant():
    from oracle._util import Tile
    from oracle.ppm import ppm_flux

    n, nz = 12, 2
    t = Tile(n, nz)
    g = cases.grid_for(n)
    q = np.full((t.m, t.m, t.nk), 3.5)
    c = np.random.default_rng(0).uniform(-0.9, 0.9, q.shape)
    for axis, dxa in ((0, g.dxa[0]), (1, g.dya[0])):
        f = ppm_flux(t, q, c, dxa, axis, 8)
        inner = f[H:H + n + 1, H:H + n + 1]
        assert np.allclose(inner, 3.5, rtol=0, atol=1e-14), axis


def _compute(a, n, nz):
    return a[..., H:H + n, H:H + n, :nz]


@pytest.mark.gpu
def test_gpu_matches_golden():
    """The CUDA tracer advection reproduces the reference's golden run: the
    tracers on the compute domain and the scaled fluxes on every point,
    to 1e-12 (there are no transcendentals on this path)."""
    import gpu_runs

    g, n, nz, case = _golden()
    gpu = gpu_runs.run_tracer_advection(case, n, nz)
    assert parity_err(_compute(gpu["tracers"], n, nz), _compute(g["tracers"], n, nz)) <= 1e-12
    assert parity_err(_compute(gpu["dp1"], n, nz), _compute(g["dp1"], n, nz)) <= 1e-12
    for k in ("mfxd", "mfyd", "cxd", "cyd"):
        assert parity_err(gpu[k][..., :nz], g[k][..., :nz]) <= 1e-12, k


@pytest.mark.gpu
@pytest.mark.parametrize("n,nz,seed", [(24, 16, 3), (12, 79, 4), (48, 8, 5)])
def test_gpu_matches_oracle(n, nz, seed):
    import gpu_runs

    case = cases.tracer_case(n, nz, seed)
    ref = oracle_runs.run_tracer_advection(case, n, nz)
    gpu = gpu_runs.run_tracer_advection(case, n, nz)
    assert parity_err(_compute(gpu["tracers"], n, nz), _compute(ref["tracers"], n, nz)) <= 1e-12
    assert parity_err(_compute(gpu["dp1"], n, nz), _compute(ref["dp1"], n, nz)) <= 1e-12


@pytest.mark.gpu
def test_gpu_mixed_precision_tracers():
    """The mixed-precision build (FP32 fields and arithmetic) on the golden
    case: tracers within 1e-5 of their range (1e-2) of the FP64 result."""
    import gpu_runs

    g, n, nz, case = _golden()
    f32 = gpu_runs.run_tracer_advection(case, n, nz, "f32")
    d = np.abs(_compute(f32["tracers"], n, nz) - _compute(g["tracers"], n, nz))
    assert np.all(np.isfinite(d)) and d.max() <= 1e-7, d.max()


def _transport_inputs(n, nz, seed):
    """Random Courant numbers / area fluxes in the ranges of a D-grid step
    and a noisy field with halos filled by the halo exchange."""
    from oracle.halo import HaloExchange

    st = cases.base_state(n, nz, seed)
    rng = np.random.default_rng(seed + 7)
    shp = st["delp"].shape
    g = cases.grid_for(n)
    area = g.area[:, :, :, None]
    q = st["pt"] * (1.0 + 1e-2 * rng.standard_normal(shp))
    HaloExchange(n, H).scalar(q, nk=nz + 1)
    inp = {
        "q": q,
        "crx": 0.3 * rng.standard_normal(shp),
        "cry": 0.3 * rng.standard_normal(shp),
        "xfx": 0.05 * area * rng.standard_normal(shp),
        "yfx": 0.05 * area * rng.standard_normal(shp),
        "mfx": 1e3 * area * rng.standard_normal(shp),
        "mfy": 1e3 * area * rng.standard_normal(shp),
        "mass": st["delp"] * (1.0 + 1e-3 * rng.standard_normal(shp)),
    }
    return inp


def _oracle_transport(n, nz, inp, hord, mass_flux, damping):
    from oracle._util import Tile
    from oracle.fvtp2d import DelnScratch, FvTp2dScratch, copy_corners_xy, fvtp2d

    t = Tile(n, nz)
    out = {"fx": np.zeros_like(inp["q"]), "fy": np.zeros_like(inp["q"]), "q": np.array(inp["q"], copy=True)}
    for tt in range(6):
        ns = cases.metric_namespace(n, tt)
        q = out["q"][tt]
        qy = np.zeros_like(q)
        copy_corners_xy(t, q, qy, t.nk)
        kw = {}
        if mass_flux:
            kw = {"x_mass_flux": inp["mfx"][tt], "y_mass_flux": inp["mfy"][tt], "mass": inp["mass"][tt]}
        if damping is not None:
            kw.update(nord=damping[0], damp_c=damping[1], deln_scratch=DelnScratch(q.shape))
        with np.errstate(all="ignore"):
            fvtp2d(t, ns, q, q, qy, inp["crx"][tt], inp["cry"][tt], inp["xfx"][tt], inp["yfx"][tt],
                   out["fx"][tt], out["fy"][tt], hord, FvTp2dScratch(q.shape), **kw)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("hord,mass_flux,damped", [(6, False, False), (8, True, False), (6, True, True),
                                                   (5, False, True), (8, False, False)])
def test_gpu_finite_volume_transport(hord, mass_flux, damped):
    """FiniteVolumeTransport on its own, against the oracle's fvtp2d on the
    compute-domain fluxes (damping columns of the D-grid namelist:
    nord 0 on the three sponge levels, 2 below)."""
    import torch

    from fv3core_b200.grid_data import GridData
    from fv3core_b200.stencil import StencilConfig, StencilFactory
    from fv3core_b200.stencils.fvtp2d import FiniteVolumeTransport
    from fv3core_b200.storage import to_device, to_host

    n, nz = 12, 10
    inp = _transport_inputs(n, nz, 31 + hord)
    damping = None
    if damped:
        nord = np.array([0.0, 0.0, 0.0] + [2.0] * (nz - 2))
        damp = np.array([0.1, 0.05, 0.06] + [0.06] * (nz - 2))
        damping = (nord, damp)
    ref = _oracle_transport(n, nz, inp, hord, mass_flux, damping)
    gd = GridData(cases.grid_for(n), nz)
    sf = StencilFactory(StencilConfig(), gd.grid_indexing)
    try:
        tr = FiniteVolumeTransport(sf, gd, gd, 0, hord, *(damping or (None, None)))
        dev = {k: to_device(v) for k, v in inp.items()}
        fx, fy = torch.zeros_like(dev["q"]), torch.zeros_like(dev["q"])
        kw = {"x_mass_flux": dev["mfx"], "y_mass_flux": dev["mfy"], "mass": dev["mass"]} if mass_flux else {}
        tr(dev["q"], dev["crx"], dev["cry"], dev["xfx"], dev["yfx"], fx, fy, **kw)
        torch.cuda.synchronize()
        gfx, gfy = to_host(fx), to_host(fy)
        tr.close()
    finally:
        gd.close()
    s = slice(H, H + n + 1)
    c = slice(H, H + n)
    assert parity_err(gfx[:, s, c, :nz + 1], ref["fx"][:, s, c, :nz + 1]) <= 1e-12
    assert parity_err(gfy[:, c, s, :nz + 1], ref["fy"][:, c, s, :nz + 1]) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("iord", [6, 8])
@pytest.mark.parametrize("axis", [0, 1])
def test_gpu_piecewise_parabolic(iord, axis):
    """X/YPiecewiseParabolic over the inner box fvtp2d gives them (three
    halo rows across the axis), against the oracle's ppm_flux."""
    import torch

    from oracle._util import Tile
    from oracle.ppm import ppm_flux

    from fv3core_b200.grid_data import GridData
    from fv3core_b200.stencil import StencilConfig, StencilFactory
    from fv3core_b200.stencils.xppm import XPiecewiseParabolic
    from fv3core_b200.stencils.yppm import YPiecewiseParabolic
    from fv3core_b200.storage import to_device, to_host

    n, nz = 12, 6
    inp = _transport_inputs(n, nz, 40 + iord)
    t = Tile(n, nz)
    g = cases.grid_for(n)
    if axis == 0:
        origin, domain = (H, 0, 0), (n + 1, n + 2 * H, nz + 1)
    else:
        origin, domain = (0, H, 0), (n + 2 * H, n + 1, nz + 1)
    c = inp["crx"] if axis == 0 else inp["cry"]
    ref = np.stack([ppm_flux(t, inp["q"][tt], c[tt], (g.dxa if axis == 0 else g.dya)[tt], axis, iord)
                    for tt in range(6)])
    gd = GridData(g, nz)
    sf = StencilFactory(StencilConfig(), gd.grid_indexing)
    try:
        cls = XPiecewiseParabolic if axis == 0 else YPiecewiseParabolic
        op = cls(sf, gd.dxa if axis == 0 else gd.dya, 0, iord, origin, domain)
        out = torch.zeros_like(to_device(inp["q"]))
        op(to_device(inp["q"]), to_device(c), out)
        torch.cuda.synchronize()
        got = to_host(out)
    finally:
        gd.close()
    box = tuple(slice(o, o + d) for o, d in zip(origin, domain))
    assert parity_err(got[(slice(None),) + box], ref[(slice(None),) + box]) <= 1e-12
