"""Differentiable vertically implicit solvers: RiemannSolver3 (reference
``fv3core/stencils/riem_solver3.py:145-242``) and RiemannSolverC
(``riem_solver_c.py:106-165``), both with ``sim1_solver.py``, as
``torch.autograd.Function`` s whose backward passes are the library's
hand-written adjoints (``fv3b_riem_solver3_adjoint``,
``fv3b_riem_solver_c_adjoint``).

``p_grad_c(uc, vc, delpc, pkc, gz, stencil_factory, dt2)`` (reference
``dyn_core.py:101-145``) returns the new (uc, vc), its backward pass being
``fv3b_p_grad_c_adjoint``.
``update_dz_c(dp_ref, zs, ut, vt, gz, ws, stencil_factory, dt)`` (reference
``updatedzc.py:123-163``) returns the new (gz, ws), its backward pass being
``fv3b_update_dz_c_adjoint`` (dp_ref and zs held fixed).
``nh_p_grad(u, v, pp, gz, pk3, delp, stencil_factory, dt, ptop, akap)``
(reference ``nh_p_grad.py:147-206``) returns the new (u, v, pp, gz, pk3),
its backward pass being ``fv3b_nh_p_grad_adjoint`` (the wind update's
adjoint and the transposes of the four a2b_ord4 interpolations).
``halo_update_scalar(field, stencil_factory, stagger, n_halo, nlev)``,
``halo_update_vector(x, y, stencil_factory, grid, nlev)`` and
``synchronize_vector_interfaces(u, v, stencil_factory, nlev)`` are the halo
calls the acoustic loop makes between stages, with their transposes
(``fv3b_halo_update_*_adjoint``, ``fv3b_synchronize_vector_interfaces_adjoint``)
as backward passes.
``edge_pe(pe, delp, stencil_factory, ptop)`` and ``pk3_halo(pk3, delp,
stencil_factory, ptop, akap)`` (reference ``pe_halo.py:6-33``,
``pk3_halo.py:36-68``) are the halo-ring column sums, with
``fv3b_edge_pe_adjoint`` / ``fv3b_pk3_halo_adjoint`` as backward passes.
``ray_fast(u, v, w, dp, pfull, stencil_factory, dt, ptop, rf_cutoff, tau)``
(reference ``ray_fast.py:131-192``) returns the damped (u, v, w), with
``fv3b_ray_fast_adjoint`` as its backward pass.
``del2cubed(qdel, stencil_factory, cd, nmax)`` (reference
``del2cubed.py:152-181``) returns the filtered field, with
``fv3b_del2cubed_adjoint`` as its backward pass.
``pkz_tempadjust(delp, delz, cappa, heat_source, pt, pkz, stencil_factory,
delt_time_factor, nk_heat)`` (reference ``temperature_adjust.py:8-44``)
returns the new (pt, pkz), with ``fv3b_pkz_tempadjust_adjoint`` as its
backward pass (cappa held fixed).

These are the stages of the acoustic substep with an adjoint so far; the
others have none yet, so a whole substep cannot be differentiated.

``riem_solver3(w, zh, delp, pt, cappa, zs, wsd, q_con, grid_indexing, dt,
ptop, p_fac)`` returns the new (w, delz) of the compute-domain columns;
``riem_solver_c(w3, gz, delpc, ptc, cappa, hs, ws, q_con, grid_indexing,
dt2, ptop, p_fac)`` returns the new (pef, gz) of the columns is-1..ie+1.
Neither changes its inputs; gradients flow to the first four arguments
and to the surface w (wsd, ws); cappa, q_con and the surface heights are
held fixed.  Fields are device
tensors in the kernel layout of ``grid_indexing``.
"""
import torch

from . import _lib
from .stencils._common import context, host_column
from .storage import check_field, stream_ptr


class RiemannSolver3Function(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w, zh, delp, pt, cappa, zs, wsd, q_con, gi, dt, ptop, p_fac):
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        w_new = w.detach().clone()
        zh_new = zh.detach().clone()
        delz = torch.zeros_like(w_new)
        scratch = [torch.zeros_like(w_new) for _ in range(5)]  # pe, ppe, pk3, pk, peln
        _lib.call(
            "fv3b_riem_solver3", gi.dims(), 0, float(dt), float(ptop), float(p_fac), f3(cappa, "cappa"),
            check_field(zs, gi, "2d", "zs"), check_field(wsd, gi, "2d", "wsd"), f3(delz, "delz"),
            f3(q_con, "q_con"), f3(delp, "delp"), f3(pt, "pt"), f3(zh_new, "zh"), f3(scratch[0], "pe"),
            f3(scratch[1], "ppe"), f3(scratch[2], "pk3"), f3(scratch[3], "pk"), f3(scratch[4], "peln"),
            f3(w_new, "w"), stream_ptr(), precision=gi.precision,
        )
        ctx.save_for_backward(w.detach(), zh.detach(), delp.detach(), pt.detach(), cappa, wsd.detach(), q_con)
        ctx.params = (gi, float(dt), float(ptop), float(p_fac))
        return w_new, delz

    @staticmethod
    def backward(ctx, g_w_new, g_delz):
        w, zh, delp, pt, cappa, wsd, q_con = ctx.saved_tensors
        gi, dt, ptop, p_fac = ctx.params
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        gw_out = torch.zeros_like(w) if g_w_new is None else g_w_new.contiguous()
        gdz_out = torch.zeros_like(w) if g_delz is None else g_delz.contiguous()
        grads = [torch.zeros_like(w) for _ in range(4)]  # w, zh, delp, pt
        g_wsd = torch.zeros_like(wsd)
        _lib.call(
            "fv3b_riem_solver3_adjoint", gi.dims(), dt, ptop, p_fac, f3(cappa, "cappa"),
            check_field(wsd, gi, "2d", "wsd"), f3(q_con, "q_con"), f3(delp, "delp"), f3(pt, "pt"), f3(zh, "zh"),
            f3(w, "w"), f3(gw_out, "gw_out"), f3(gdz_out, "gdz_out"), f3(grads[0], "g_w"), f3(grads[1], "g_zh"),
            f3(grads[2], "g_delp"), f3(grads[3], "g_pt"), check_field(g_wsd, gi, "2d", "g_wsd"), stream_ptr(),
            precision=gi.precision,
        )
        # w_new is w itself outside the solved points (other columns, the
        # bottom interface level): there the gradient passes through
        h, n, nz = gi.n_halo, gi.n, gi.npz
        solved = torch.zeros_like(w, dtype=torch.bool)
        solved[:, :nz, h:h + n, h:h + n] = True
        grads[0] = torch.where(solved, grads[0], gw_out)
        return grads[0], grads[1], grads[2], grads[3], None, None, g_wsd, None, None, None, None, None


def riem_solver3(w, zh, delp, pt, cappa, zs, wsd, q_con, grid_indexing, dt, ptop, p_fac):
    """New (w, delz) of RiemannSolver3 on the compute domain, differentiable
    with respect to w, zh, delp, pt and wsd."""
    return RiemannSolver3Function.apply(w, zh, delp, pt, cappa, zs, wsd, q_con, grid_indexing, dt, ptop, p_fac)


class RiemannSolverCFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w3, gz, delpc, ptc, cappa, hs, ws, q_con, gi, dt2, ptop, p_fac):
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        gz_new = gz.detach().clone()
        pef = torch.zeros_like(gz_new)
        _lib.call(
            "fv3b_riem_solver_c", gi.dims(), float(dt2), float(ptop), float(p_fac), f3(cappa, "cappa"),
            check_field(hs, gi, "2d", "hs"), check_field(ws, gi, "2d", "ws"), f3(ptc, "ptc"), f3(q_con, "q_con"),
            f3(delpc, "delpc"), f3(gz_new, "gz"), f3(pef, "pef"), f3(w3, "w3"), stream_ptr(),
            precision=gi.precision,
        )
        ctx.save_for_backward(w3.detach(), gz.detach(), delpc.detach(), ptc.detach(), cappa, ws.detach(), q_con)
        ctx.params = (gi, float(dt2), float(ptop), float(p_fac))
        return pef, gz_new

    @staticmethod
    def backward(ctx, g_pef, g_gz):
        w3, gz, delpc, ptc, cappa, ws, q_con = ctx.saved_tensors
        gi, dt2, ptop, p_fac = ctx.params
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        gpef_out = torch.zeros_like(gz) if g_pef is None else g_pef.contiguous()
        ggz_out = torch.zeros_like(gz) if g_gz is None else g_gz.contiguous()
        grads = [torch.zeros_like(gz) for _ in range(4)]  # w3, gz, delpc, ptc
        g_ws = torch.zeros_like(ws)
        _lib.call(
            "fv3b_riem_solver_c_adjoint", gi.dims(), dt2, ptop, p_fac, f3(cappa, "cappa"),
            check_field(ws, gi, "2d", "ws"), f3(q_con, "q_con"), f3(delpc, "delpc"), f3(ptc, "ptc"),
            f3(gz, "gz"), f3(w3, "w3"), f3(gpef_out, "gpef_out"), f3(ggz_out, "ggz_out"), f3(grads[0], "g_w3"),
            f3(grads[1], "g_gz"), f3(grads[2], "g_delpc"), f3(grads[3], "g_ptc"), check_field(g_ws, gi, "2d", "g_ws"),
            stream_ptr(), precision=gi.precision,
        )
        # gz outside the solved columns is gz itself: the gradient passes through
        h, n = gi.n_halo, gi.n
        solved = torch.zeros_like(gz, dtype=torch.bool)
        solved[:, :, h - 1:h + n + 1, h - 1:h + n + 1] = True
        grads[1] = grads[1] + torch.where(solved, torch.zeros_like(ggz_out), ggz_out)
        return grads[0], grads[1], grads[2], grads[3], None, None, g_ws, None, None, None, None, None


def riem_solver_c(w3, gz, delpc, ptc, cappa, hs, ws, q_con, grid_indexing, dt2, ptop, p_fac):
    """New (pef, gz) of RiemannSolverC on the columns is-1..ie+1,
    differentiable with respect to w3, gz, delpc, ptc and ws."""
    return RiemannSolverCFunction.apply(w3, gz, delpc, ptc, cappa, hs, ws, q_con, grid_indexing, dt2, ptop, p_fac)


class PGradCFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, uc, vc, delpc, pkc, gz, stencil_factory, dt2):
        gi = stencil_factory.grid_indexing
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        uc_new, vc_new = uc.detach().clone(), vc.detach().clone()
        _lib.call_ctx("fv3b_p_grad_c", context(stencil_factory), f3(uc_new, "uc"), f3(vc_new, "vc"),
                      f3(delpc, "delpc"), f3(pkc, "pkc"), f3(gz, "gz"), float(dt2), stream_ptr())
        ctx.save_for_backward(delpc.detach(), pkc.detach(), gz.detach())
        ctx.params = (stencil_factory, float(dt2))
        return uc_new, vc_new

    @staticmethod
    def backward(ctx, g_uc, g_vc):
        delpc, pkc, gz = ctx.saved_tensors
        stencil_factory, dt2 = ctx.params
        gi = stencil_factory.grid_indexing
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        g_uc = torch.zeros_like(delpc) if g_uc is None else g_uc.contiguous()
        g_vc = torch.zeros_like(delpc) if g_vc is None else g_vc.contiguous()
        grads = [torch.zeros_like(delpc) for _ in range(3)]  # delpc, pkc, gz
        _lib.call_ctx("fv3b_p_grad_c_adjoint", context(stencil_factory), f3(delpc, "delpc"), f3(pkc, "pkc"),
                      f3(gz, "gz"), f3(g_uc, "gu"), f3(g_vc, "gv"), f3(grads[0], "g_delpc"), f3(grads[1], "g_pkc"),
                      f3(grads[2], "g_gz"), dt2, stream_ptr())
        # the winds only gain increments: their gradients pass through
        return g_uc, g_vc, grads[0], grads[1], grads[2], None, None


def p_grad_c(uc, vc, delpc, pkc, gz, stencil_factory, dt2):
    """New (uc, vc) of p_grad_c_stencil, differentiable with respect to all
    five fields."""
    return PGradCFunction.apply(uc, vc, delpc, pkc, gz, stencil_factory, dt2)


class UpdateDzCFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, ut, vt, gz, ws, dp_ref, zs, stencil_factory, dt):
        gi = stencil_factory.grid_indexing
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        gz_new, ws_new = gz.detach().clone(), ws.detach().clone()
        _lib.call_ctx("fv3b_update_dz_c", context(stencil_factory), check_field(dp_ref, gi, "1d", "dp_ref"),
                      check_field(zs, gi, "2d", "zs"), f3(ut, "ut"), f3(vt, "vt"), f3(gz_new, "gz"),
                      check_field(ws_new, gi, "2d", "ws"), float(dt), stream_ptr())
        ctx.save_for_backward(ut.detach(), vt.detach(), gz.detach(), dp_ref)
        ctx.params = (stencil_factory, float(dt))
        return gz_new, ws_new

    @staticmethod
    def backward(ctx, g_gz, g_ws):
        ut, vt, gz, dp_ref = ctx.saved_tensors
        stencil_factory, dt = ctx.params
        gi = stencil_factory.grid_indexing
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        g_gz = torch.zeros_like(gz) if g_gz is None else g_gz.contiguous()
        m = gi.max_shape[0]
        g_ws = torch.zeros((6, m, m), dtype=gz.dtype, device=gz.device) if g_ws is None else g_ws.contiguous()
        grads = [torch.empty_like(gz) for _ in range(3)]  # gz, ut, vt
        _lib.call_ctx("fv3b_update_dz_c_adjoint", context(stencil_factory), check_field(dp_ref, gi, "1d", "dp_ref"),
                      f3(ut, "ut"), f3(vt, "vt"), f3(gz, "gz"), f3(g_gz, "g_gz_out"),
                      check_field(g_ws, gi, "2d", "g_ws"), f3(grads[0], "g_gz"), f3(grads[1], "g_ut"),
                      f3(grads[2], "g_vt"), dt, stream_ptr())
        # ws keeps its value outside the updated box: there its gradient passes through
        h, n = gi.n_halo, gi.n
        g_ws_in = g_ws.clone()
        g_ws_in[:, h - 1:h + n + 1, h - 1:h + n + 1] = 0.0
        return grads[1], grads[2], grads[0], g_ws_in, None, None, None, None


def update_dz_c(dp_ref, zs, ut, vt, gz, ws, stencil_factory, dt):
    """New (gz, ws) of UpdateGeopotentialHeightOnCGrid, differentiable with
    respect to ut, vt, gz and ws."""
    return UpdateDzCFunction.apply(ut, vt, gz, ws, dp_ref, zs, stencil_factory, dt)


class NhPGradFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u, v, pp, gz, pk3, delp, stencil_factory, dt, ptop, akap):
        gi = stencil_factory.grid_indexing
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        out = [t.detach().clone() for t in (u, v, pp, gz, pk3)]
        _lib.call_ctx("fv3b_nh_p_grad", context(stencil_factory), f3(out[0], "u"), f3(out[1], "v"),
                      f3(out[2], "pp"), f3(out[3], "gz"), f3(out[4], "pk3"), f3(delp, "delp"), float(dt),
                      float(ptop), float(akap), stream_ptr())
        ctx.save_for_backward(pp.detach(), gz.detach(), pk3.detach(), delp.detach())
        ctx.params = (stencil_factory, float(dt), float(ptop), float(akap))
        return tuple(out)

    @staticmethod
    def backward(ctx, g_u, g_v, g_pp, g_gz, g_pk3):
        pp, gz, pk3, delp = ctx.saved_tensors
        stencil_factory, dt, ptop, akap = ctx.params
        gi = stencil_factory.grid_indexing
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        cot = [torch.zeros_like(pp) if g is None else g.contiguous() for g in (g_u, g_v, g_pp, g_gz, g_pk3)]
        grads = [torch.empty_like(pp) for _ in range(6)]  # u, v, pp, gz, pk3, delp
        _lib.call_ctx("fv3b_nh_p_grad_adjoint", context(stencil_factory), f3(pp, "pp"), f3(gz, "gz"),
                      f3(pk3, "pk3"), f3(delp, "delp"), *[f3(c, n) for c, n in zip(cot, ("gu", "gv", "gpp", "ggz",
                                                                                       "gpk3"))],
                      *[f3(g, n) for g, n in zip(grads, ("g_u", "g_v", "g_pp", "g_gz", "g_pk3", "g_delp"))],
                      dt, ptop, akap, stream_ptr())
        return tuple(grads) + (None, None, None, None)


def nh_p_grad(u, v, pp, gz, pk3, delp, stencil_factory, dt, ptop, akap):
    """New (u, v, pp, gz, pk3) of NonHydrostaticPressureGradient,
    differentiable with respect to u, v, pp, gz, pk3 and delp."""
    return NhPGradFunction.apply(u, v, pp, gz, pk3, delp, stencil_factory, dt, ptop, akap)


class HaloUpdateScalarFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, field, stencil_factory, stagger, n_halo, nlev):
        gi = stencil_factory.grid_indexing
        out = field.detach().clone()
        _lib.call_ctx("fv3b_halo_update_scalar", context(stencil_factory), check_field(out, gi, "3d", "field"),
                      int(stagger), int(n_halo), int(nlev), stream_ptr())
        ctx.params = (stencil_factory, int(stagger), int(n_halo), int(nlev))
        return out

    @staticmethod
    def backward(ctx, g):
        stencil_factory, stagger, n_halo, nlev = ctx.params
        g = g.clone(memory_format=torch.contiguous_format)
        _lib.call_ctx("fv3b_halo_update_scalar_adjoint", context(stencil_factory),
                      check_field(g, stencil_factory.grid_indexing, "3d", "g"), stagger, n_halo, nlev, stream_ptr())
        return g, None, None, None, None


class HaloUpdateVectorFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, y, stencil_factory, grid, nlev):
        gi = stencil_factory.grid_indexing
        ox, oy = x.detach().clone(), y.detach().clone()
        _lib.call_ctx("fv3b_halo_update_vector", context(stencil_factory), check_field(ox, gi, "3d", "x"),
                      check_field(oy, gi, "3d", "y"), int(grid), int(nlev), stream_ptr())
        ctx.params = (stencil_factory, int(grid), int(nlev))
        return ox, oy

    @staticmethod
    def backward(ctx, gx, gy):
        stencil_factory, grid, nlev = ctx.params
        gi = stencil_factory.grid_indexing
        m = gi.max_shape[0]
        zeros = lambda: torch.zeros((6, gi.max_shape[2], m, m), dtype=gi.dtype, device="cuda")  # noqa: E731
        gx = zeros() if gx is None else gx.clone(memory_format=torch.contiguous_format)
        gy = zeros() if gy is None else gy.clone(memory_format=torch.contiguous_format)
        _lib.call_ctx("fv3b_halo_update_vector_adjoint", context(stencil_factory), check_field(gx, gi, "3d", "gx"),
                      check_field(gy, gi, "3d", "gy"), grid, nlev, stream_ptr())
        return gx, gy, None, None, None


class InterfaceSyncFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u, v, stencil_factory, nlev):
        gi = stencil_factory.grid_indexing
        ou, ov = u.detach().clone(), v.detach().clone()
        _lib.call_ctx("fv3b_synchronize_vector_interfaces", context(stencil_factory),
                      check_field(ou, gi, "3d", "u"), check_field(ov, gi, "3d", "v"), int(nlev), stream_ptr())
        ctx.params = (stencil_factory, int(nlev))
        return ou, ov

    @staticmethod
    def backward(ctx, gu, gv):
        stencil_factory, nlev = ctx.params
        gi = stencil_factory.grid_indexing
        m = gi.max_shape[0]
        zeros = lambda: torch.zeros((6, gi.max_shape[2], m, m), dtype=gi.dtype, device="cuda")  # noqa: E731
        gu = zeros() if gu is None else gu.clone(memory_format=torch.contiguous_format)
        gv = zeros() if gv is None else gv.clone(memory_format=torch.contiguous_format)
        _lib.call_ctx("fv3b_synchronize_vector_interfaces_adjoint", context(stencil_factory),
                      check_field(gu, gi, "3d", "gu"), check_field(gv, gi, "3d", "gv"), nlev, stream_ptr())
        return gu, gv, None, None


def halo_update_scalar(field, stencil_factory, stagger=1, n_halo=3, nlev=None):
    """The field after a scalar halo update (stagger 1 = cell centres,
    0 = cell corners), differentiable."""
    nlev = stencil_factory.grid_indexing.max_shape[2] if nlev is None else nlev
    return HaloUpdateScalarFunction.apply(field, stencil_factory, stagger, n_halo, nlev)


def halo_update_vector(x, y, stencil_factory, grid=0, nlev=None):
    """The winds after a vector halo update (grid 0 = D, 1 = C),
    differentiable."""
    nlev = stencil_factory.grid_indexing.max_shape[2] if nlev is None else nlev
    return HaloUpdateVectorFunction.apply(x, y, stencil_factory, grid, nlev)


def synchronize_vector_interfaces(u, v, stencil_factory, nlev=None):
    """The D-grid winds after synchronize_vector_interfaces, differentiable."""
    nlev = stencil_factory.grid_indexing.max_shape[2] if nlev is None else nlev
    return InterfaceSyncFunction.apply(u, v, stencil_factory, nlev)


class EdgePeFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pe, delp, stencil_factory, ptop):
        gi = stencil_factory.grid_indexing
        out = pe.detach().clone()
        _lib.call_ctx("fv3b_edge_pe", context(stencil_factory), check_field(out, gi, "3d", "pe"),
                      check_field(delp, gi, "3d", "delp"), float(ptop), stream_ptr())
        ctx.params = stencil_factory
        return out

    @staticmethod
    def backward(ctx, g):
        stencil_factory = ctx.params
        gi = stencil_factory.grid_indexing
        g = g.clone(memory_format=torch.contiguous_format)
        g_delp = torch.empty_like(g)
        _lib.call_ctx("fv3b_edge_pe_adjoint", context(stencil_factory), check_field(g, gi, "3d", "g_pe"),
                      check_field(g_delp, gi, "3d", "g_delp"), stream_ptr())
        return g, g_delp, None, None


class Pk3HaloFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pk3, delp, stencil_factory, ptop, akap):
        gi = stencil_factory.grid_indexing
        out = pk3.detach().clone()
        _lib.call_ctx("fv3b_pk3_halo", context(stencil_factory), check_field(out, gi, "3d", "pk3"),
                      check_field(delp, gi, "3d", "delp"), float(ptop), float(akap), stream_ptr())
        ctx.save_for_backward(delp.detach())
        ctx.params = (stencil_factory, float(ptop), float(akap))
        return out

    @staticmethod
    def backward(ctx, g):
        (delp,) = ctx.saved_tensors
        stencil_factory, ptop, akap = ctx.params
        gi = stencil_factory.grid_indexing
        g = g.clone(memory_format=torch.contiguous_format)
        g_delp = torch.empty_like(g)
        _lib.call_ctx("fv3b_pk3_halo_adjoint", context(stencil_factory), check_field(delp, gi, "3d", "delp"),
                      check_field(g, gi, "3d", "g_pk3"), check_field(g_delp, gi, "3d", "g_delp"), ptop, akap,
                      stream_ptr())
        return g, g_delp, None, None, None


def edge_pe(pe, delp, stencil_factory, ptop):
    """pe after edge_pe (the one-cell ring), differentiable."""
    return EdgePeFunction.apply(pe, delp, stencil_factory, ptop)


def pk3_halo(pk3, delp, stencil_factory, ptop, akap):
    """pk3 after PK3Halo (the two-cell ring), differentiable."""
    return Pk3HaloFunction.apply(pk3, delp, stencil_factory, ptop, akap)


class RayFastFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u, v, w, dp, pfull, stencil_factory, dt, ptop, rf_cutoff, tau):
        gi = stencil_factory.grid_indexing
        dp_h, pf_h = host_column(dp, gi.npz, "dp"), host_column(pfull, gi.npz, "pfull")
        out = [t.detach().clone() for t in (u, v, w)]
        args = (dp_h.ctypes.data, pf_h.ctypes.data, float(dt), float(ptop), float(rf_cutoff), float(tau), 0)
        _lib.call_ctx("fv3b_ray_fast", context(stencil_factory), *[check_field(t, gi, "3d", n)
                                                                  for t, n in zip(out, "uvw")], *args, stream_ptr())
        ctx.params = (stencil_factory, dp_h, pf_h, args)
        return tuple(out)

    @staticmethod
    def backward(ctx, gu, gv, gw):
        stencil_factory, dp_h, pf_h, args = ctx.params
        gi = stencil_factory.grid_indexing
        m = gi.max_shape[0]
        g = [torch.zeros((6, gi.max_shape[2], m, m), dtype=gi.dtype, device="cuda") if x is None
             else x.clone(memory_format=torch.contiguous_format) for x in (gu, gv, gw)]
        _lib.call_ctx("fv3b_ray_fast_adjoint", context(stencil_factory),
                      *[check_field(t, gi, "3d", n) for t, n in zip(g, ("gu", "gv", "gw"))], *args, stream_ptr())
        return g[0], g[1], g[2], None, None, None, None, None, None, None


def ray_fast(u, v, w, dp, pfull, stencil_factory, dt, ptop, rf_cutoff, tau):
    """The winds after RayleighDamping (nonhydrostatic), differentiable with
    respect to u, v and w."""
    return RayFastFunction.apply(u, v, w, dp, pfull, stencil_factory, dt, ptop, rf_cutoff, tau)


class Del2CubedFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, qdel, stencil_factory, cd, nmax):
        gi = stencil_factory.grid_indexing
        out = qdel.detach().clone()
        _lib.call_ctx("fv3b_del2cubed", context(stencil_factory), check_field(out, gi, "3d", "qdel"), float(cd),
                      int(nmax), stream_ptr())
        ctx.params = (stencil_factory, float(cd), int(nmax))
        return out

    @staticmethod
    def backward(ctx, g):
        stencil_factory, cd, nmax = ctx.params
        g = g.clone(memory_format=torch.contiguous_format)
        _lib.call_ctx("fv3b_del2cubed_adjoint", context(stencil_factory),
                      check_field(g, stencil_factory.grid_indexing, "3d", "gq"), cd, nmax, stream_ptr())
        return g, None, None, None


def del2cubed(qdel, stencil_factory, cd, nmax):
    """The field after HyperdiffusionDamping, differentiable."""
    return Del2CubedFunction.apply(qdel, stencil_factory, cd, nmax)


class PkzTempadjustFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, delp, delz, cappa, heat_source, pt, pkz, stencil_factory, delt_time_factor, nk_heat):
        gi = stencil_factory.grid_indexing
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        new_pt, new_pkz = pt.detach().clone(), pkz.detach().clone()
        _lib.call_ctx("fv3b_pkz_tempadjust", context(stencil_factory), f3(delp, "delp"), f3(delz, "delz"),
                      f3(cappa, "cappa"), f3(heat_source, "heat_source"), f3(new_pt, "pt"), f3(new_pkz, "pkz"),
                      float(delt_time_factor), int(nk_heat), stream_ptr())
        ctx.save_for_backward(delp.detach(), delz.detach(), cappa, heat_source.detach(), pt.detach())
        ctx.params = (stencil_factory, float(delt_time_factor), int(nk_heat))
        return new_pt, new_pkz

    @staticmethod
    def backward(ctx, g_pt, g_pkz):
        delp, delz, cappa, heat_source, pt = ctx.saved_tensors
        stencil_factory, dtf, nk_heat = ctx.params
        gi = stencil_factory.grid_indexing
        f3 = lambda t, n: check_field(t, gi, "3d", n)  # noqa: E731
        g_pt = torch.zeros_like(pt) if g_pt is None else g_pt.clone(memory_format=torch.contiguous_format)
        g_pkz = torch.zeros_like(pt) if g_pkz is None else g_pkz.clone(memory_format=torch.contiguous_format)
        out = [torch.empty_like(pt) for _ in range(3)]  # delp, delz, heat_source
        _lib.call_ctx("fv3b_pkz_tempadjust_adjoint", context(stencil_factory), f3(delp, "delp"), f3(delz, "delz"),
                      f3(cappa, "cappa"), f3(heat_source, "heat_source"), f3(pt, "pt"), f3(g_pt, "g_pt"),
                      f3(g_pkz, "g_pkz"), f3(out[0], "g_delp"), f3(out[1], "g_delz"), f3(out[2], "g_heat"), dtf,
                      nk_heat, stream_ptr())
        return out[0], out[1], None, out[2], g_pt, g_pkz, None, None, None


def pkz_tempadjust(delp, delz, cappa, heat_source, pt, pkz, stencil_factory, delt_time_factor, nk_heat):
    """New (pt, pkz) of compute_pkz_tempadjust, differentiable with respect
    to delp, delz, heat_source, pt and pkz."""
    return PkzTempadjustFunction.apply(delp, delz, cappa, heat_source, pt, pkz, stencil_factory, delt_time_factor,
                                       nk_heat)
