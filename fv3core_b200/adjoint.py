"""Differentiable RiemannSolver3: the vertically implicit acoustic solve
(reference ``fv3core/stencils/riem_solver3.py:145-242`` with
``sim1_solver.py``) as a ``torch.autograd.Function`` whose backward pass is
the library's hand-written adjoint (``fv3b_riem_solver3_adjoint``).

This is the first stage of the acoustic substep with an adjoint; the other
stages have none yet, so a whole substep cannot be differentiated.

``riem_solver3(w, zh, delp, pt, cappa, zs, wsd, q_con, grid_indexing, dt,
ptop, p_fac)`` returns the new (w, delz) of the compute-domain columns
without changing its inputs; gradients flow to w, zh, delp and pt (cappa,
q_con and the surface terms are held fixed).  Fields are device tensors in
the kernel layout of ``grid_indexing``.
"""
import torch

from . import _lib
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
        ctx.save_for_backward(w.detach(), zh.detach(), delp.detach(), pt.detach(), cappa, wsd, q_con)
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
        _lib.call(
            "fv3b_riem_solver3_adjoint", gi.dims(), dt, ptop, p_fac, f3(cappa, "cappa"),
            check_field(wsd, gi, "2d", "wsd"), f3(q_con, "q_con"), f3(delp, "delp"), f3(pt, "pt"), f3(zh, "zh"),
            f3(w, "w"), f3(gw_out, "gw_out"), f3(gdz_out, "gdz_out"), f3(grads[0], "g_w"), f3(grads[1], "g_zh"),
            f3(grads[2], "g_delp"), f3(grads[3], "g_pt"), stream_ptr(), precision=gi.precision,
        )
        # w_new is w itself outside the solved points (other columns, the
        # bottom interface level): there the gradient passes through
        h, n, nz = gi.n_halo, gi.n, gi.npz
        solved = torch.zeros_like(w, dtype=torch.bool)
        solved[:, :nz, h:h + n, h:h + n] = True
        grads[0] = torch.where(solved, grads[0], gw_out)
        return grads[0], grads[1], grads[2], grads[3], None, None, None, None, None, None, None, None


def riem_solver3(w, zh, delp, pt, cappa, zs, wsd, q_con, grid_indexing, dt, ptop, p_fac):
    """New (w, delz) of RiemannSolver3 on the compute domain, differentiable
    with respect to w, zh, delp and pt."""
    return RiemannSolver3Function.apply(w, zh, delp, pt, cappa, zs, wsd, q_con, grid_indexing, dt, ptop, p_fac)
