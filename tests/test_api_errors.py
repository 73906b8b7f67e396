"""The stage classes reject what the reference rejects, with the
reference's exception types (dyn_core.py:322-324, riem_solver3.py:123,
d_sw.py:624-626), and the options not implemented here (RiemannSolver3's
use_logp and beta), before touching the device, so these run on the CPU;
the field checks name the offending argument."""
import dataclasses

import numpy as np
import pytest
import torch

from fv3core_b200.config import RiemannConfig, baroclinic_acoustic_config
from fv3core_b200.stencil import StencilConfig, StencilFactory
from fv3core_b200.storage import GridIndexing, check_field


@pytest.fixture
def factory():
    return StencilFactory(StencilConfig(), GridIndexing((12, 12, 8), 3))


def _acoustic(config, nested=False, stretched=False):
    from fv3core_b200.stencils.dyn_core import AcousticDynamics

    return AcousticDynamics(None, None, None, None, 0, nested, stretched, config, None, None, None, None)


def test_acoustic_dynamics_rejections():
    cfg = baroclinic_acoustic_config()
    with pytest.raises(NotImplementedError):
        _acoustic(cfg, nested=True)
    with pytest.raises(NotImplementedError):
        _acoustic(cfg, stretched=True)
    # d_ext lives in the D-grid namelist, beta and use_logp in the Riemann one
    with pytest.raises(AssertionError):
        _acoustic(dataclasses.replace(cfg, d_grid_shallow_water=dataclasses.replace(cfg.d_grid_shallow_water,
                                                                                    d_ext=0.1)))
    for field, value in (("beta", 0.5), ("use_logp", True)):
        with pytest.raises(AssertionError):
            _acoustic(dataclasses.replace(cfg, riemann=dataclasses.replace(cfg.riemann, **{field: value})))
    with pytest.raises(NotImplementedError):
        _acoustic(dataclasses.replace(cfg, riemann=dataclasses.replace(cfg.riemann, a_imp=0.5)))


def test_riemann_solver3_rejections(factory):
    from fv3core_b200.stencils.riem_solver3 import RiemannSolver3

    for kw in (dict(a_imp=0.5), dict(use_logp=True), dict(beta=0.5)):
        base = dict(p_fac=0.05, a_imp=1.0, use_logp=False, beta=0.0)
        base.update(kw)
        with pytest.raises(NotImplementedError):
            RiemannSolver3(factory, RiemannConfig(**base))


def test_c_sw_and_d_sw_rejections(factory):
    from fv3core_b200.stencils.c_sw import CGridShallowWaterDynamics
    from fv3core_b200.stencils.d_sw import DGridShallowWaterLagrangianDynamics

    with pytest.raises(NotImplementedError):
        CGridShallowWaterDynamics(factory, None, False, 3, 3)
    with pytest.raises(NotImplementedError):
        CGridShallowWaterDynamics(factory, None, True, 0, 3)
    dsw = baroclinic_acoustic_config().d_grid_shallow_water
    for field, value in (("grid_type", 3), ("inline_q", True), ("d_ext", 0.1)):
        with pytest.raises(AssertionError):
            DGridShallowWaterLagrangianDynamics(factory, None, None, None, False, False,
                                                dataclasses.replace(dsw, **{field: value}))
    with pytest.raises(NotImplementedError):
        DGridShallowWaterLagrangianDynamics(factory, None, None, None, True, False, dsw)


def test_field_checks_name_the_argument(factory):
    gi = factory.grid_indexing
    m, _, nk = gi.max_shape
    with pytest.raises(TypeError, match="delp"):
        check_field(np.zeros((6, nk, m, m)), gi, "3d", "delp")
    with pytest.raises(ValueError, match="delp"):
        check_field(torch.zeros(6, nk, m, m + 1, dtype=torch.float64), gi, "3d", "delp")
    with pytest.raises(TypeError, match="delp"):
        check_field(torch.zeros(6, nk, m, m, dtype=torch.float32), gi, "3d", "delp")
    with pytest.raises(ValueError, match="CUDA"):
        check_field(torch.zeros(6, nk, m, m, dtype=torch.float64), gi, "3d", "delp")
