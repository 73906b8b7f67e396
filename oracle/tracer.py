"""Tracer advection (reference ``fv3core/stencils/tracer_2d_1l.py``,
``TracerAdvection`` 120-300): the accumulated Courant numbers and mass
fluxes of the acoustic loop advect every tracer in ``n_split`` sub-steps of
finite-volume transport with the ord-8 PPM (``hord_tr``), each tracer
re-weighted by the pressure thickness before and after.

Test infrastructure: the oracle the CUDA tracer advection is checked
against.  Six-tile arrays ``[6, m, m, nk]``; the halo exchange is the
oracle's own (``halo.py``).
"""
import numpy as np

from . import corners
from ._util import Tile, c3, put, sh
from .fvtp2d import FvTp2dScratch, fvtp2d
from .halo import HaloExchange


def flux_compute(t: Tile, g, cx, cy, xfx, yfx):
    """flux_compute with flux_x / flux_y (tracer_2d_1l.py:19-60) on the
    full domain plus one interface, restricted to the regions of flux_x and
    flux_y."""
    s, e, js, je = t.isc, t.iec, t.jsc, t.jec
    dxa, dya, dx, dy = c3(g.dxa), c3(g.dya), c3(g.dx), c3(g.dy)
    sin1, sin2, sin3, sin4 = c3(g.sin_sg1), c3(g.sin_sg2), c3(g.sin_sg3), c3(g.sin_sg4)
    fx = np.where(cx > 0, cx * sh(dxa, -1, 0) * dy * sh(sin3, -1, 0), cx * dxa * dy * sin1)
    fy = np.where(cy > 0, cy * sh(dya, 0, -1) * dx * sh(sin4, 0, -1), cy * dya * dx * sin2)
    nk = cx.shape[2]
    put(xfx, fx, s, e + 2, js - 3, je + 4, 0, nk - 1)
    put(yfx, fy, s - 3, e + 4, js, je + 2, 0, nk - 1)


class TracerAdvection:
    """TracerAdvection (tracer_2d_1l.py:120-300) over all six tiles with a
    FiniteVolumeTransport of order ``hord`` and no damping."""

    def __init__(self, grid, metrics, nz, tracer_count, hord=8):
        n = grid.n
        self.t = Tile(n, nz)
        self.g = metrics
        self.halo = HaloExchange(n, grid.halo)
        self.tracer_count = tracer_count
        self.hord = hord
        shp = (6, self.t.m, self.t.m, self.t.nk)
        # instance storages of the reference (zero-initialised, tracer_2d_1l.py:140-149)
        self.xfx = np.zeros(shp)
        self.yfx = np.zeros(shp)
        self.fx = np.zeros(shp)
        self.fy = np.zeros(shp)
        self.dp = np.zeros(shp)
        self.q_y = np.zeros(shp)
        self.scratch = [FvTp2dScratch(shp[1:]) for _ in range(6)]

    def __call__(self, tracers, dp1, mfxd, mfyd, cxd, cyd, mdt):
        """tracers: list of six-tile arrays, updated in place.  dp1, mfxd,
        mfyd, cxd and cyd are updated in place as the reference's are (the
        fluxes and Courant numbers scaled by 1/n_split, dp1 used as the
        sub-steps' ping-pong buffer)."""
        if len(tracers) != self.tracer_count:
            raise ValueError(
                f"incorrect number of tracers, {self.tracer_count} was specified on init but "
                f"{len(tracers)} were passed"
            )
        t = self.t
        for tt in range(6):
            flux_compute(t, self.g[tt], cxd[tt], cyd[tt], self.xfx[tt], self.yfx[tt])
        # cmax is fixed at 2 in the reference (tracer_2d_1l.py:233), so 3 sub-steps
        cmax_max_all_ranks = 2.0
        n_split = int(np.floor(1.0 + cmax_max_all_ranks))
        full = t.m  # domain_full(add=(1, 1, 0)): every storage point of nz levels
        nz = t.nz
        if n_split > 1.0:
            frac = 1.0 / n_split
            for a in (cxd, self.xfx, mfxd, cyd, self.yfx, mfyd):
                a[:, :full, :full, :nz] = a[:, :full, :full, :nz] * frac
        # the tracers' halo spec has dims (X, Y, Z): npz levels
        self.halo.scalar(*tracers, nk=nz)
        s, e, js, je = t.isc, t.iec, t.jsc, t.jec
        dp1_buf, dp2_buf = dp1, self.dp
        for it in range(n_split):
            last_call = it == n_split - 1
            for tt in range(6):
                ra = c3(self.g[tt].rarea)
                mfx, mfy = mfxd[tt], mfyd[tt]
                dp2 = dp1_buf[tt] + (mfx - sh(mfx, 1, 0) + mfy - sh(mfy, 0, 1)) * ra
                put(dp2_buf[tt], dp2, s, e + 1, js, je + 1, 0, nz)
            for q in tracers:
                for tt in range(6):
                    qt = q[tt]
                    # CopyCornersXY on dims (X, Y, Z), corners.py:64-117: x
                    # copy in place, y copy in the factory's own temporary
                    # (zero at the extra level npz, which the transport
                    # still computes fluxes for)
                    qx = corners.copy_corners(t, qt, "x")
                    qy = corners.copy_corners(t, qt, "y")
                    put(self.q_y[tt], qy, 0, t.m - 1, 0, t.m - 1, 0, nz)
                    put(qt, qx, 0, t.m - 1, 0, t.m - 1, 0, nz)
                    fvtp2d(t, self.g[tt], qt, qt, self.q_y[tt], cxd[tt], cyd[tt], self.xfx[tt], self.yfx[tt],
                           self.fx[tt], self.fy[tt], self.hord, self.scratch[tt],
                           x_mass_flux=mfxd[tt], y_mass_flux=mfyd[tt])
                    fx, fy = self.fx[tt], self.fy[tt]
                    ra = c3(self.g[tt].rarea)
                    qn = (qt * dp1_buf[tt] + (fx - sh(fx, 1, 0) + fy - sh(fy, 0, 1)) * ra) / dp2_buf[tt]
                    put(qt, qn, s, e + 1, js, je + 1, 0, nz)
            if not last_call:
                self.halo.scalar(*tracers, nk=nz)
                dp1_buf, dp2_buf = dp2_buf, dp1_buf

