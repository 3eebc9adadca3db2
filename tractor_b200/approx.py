"""c_gauss_2d_approx3 (tractor/approx3.c:1-465) on the device: the mixture
is evaluated on the whole box with approx3's per-component floors (and, if
asked, the d/dmean planes) by tb_mog_render, then tb_approx3_region walks
approx3's rings over those values in the same plan -- starting at (xc, yc)
or, if that is outside the box, at the brightest pixel of the nearest box
edge(s) under the plain evaluation -- zeroes every pixel approx3 would not
have evaluated, and returns the region's extent, updated only by the rows
(y) and columns (x) of each ring, exactly as approx3.c does.
"""
import numpy as np

from .plan import Pending
from .patch import Patch


def plan_approx3(plan, mix, x0, x1, y0, y1, fx, fy, minval, xc, yc, minradius=3,
                 doslice=True, derivs=False):
    """Pending result of evaluate_grid_approx3 (mixture_profiles.py:333-399):
    a Patch, or (patch, dx, dy) with derivs."""
    W, H = x1 - x0, y1 - y0
    box = plan.mog.add(x0, y0, W, H, mix.amp, mix.mean, mix.var, fx=fx, fy=fy, minval=minval,
                       derivs=derivs)
    inside = x0 <= xc < x1 and y0 <= yc < y1
    edge_col = edge_row = None
    if xc < x0 or xc >= x1:
        ex = x0 if xc < x0 else x1 - 1
        edge_col = (ex - x0, plan.mog.add(ex, y0, 1, H, mix.amp, mix.mean, mix.var, fx=fx,
                                          fy=fy, floor=-100.))
    if yc < y0 or yc >= y1:
        ey = y0 if yc < y0 else y1 - 1
        edge_row = (ey - y0, plan.mog.add(x0, ey, W, 1, mix.amp, mix.mean, mix.var, fx=fx,
                                          fy=fy, floor=-100.))
    # approx3.c's default start when no edge value is positive: C's (x0 + x1) / 2
    cdiv = lambda a: int(a / 2)  # noqa: E731  (truncates toward zero, as C)
    ring = plan.mog.add_ring(box, W, H, minval, minradius,
                             start=(xc - x0, yc - y0) if inside else None,
                             default_start=(cdiv(x0 + x1) - x0, cdiv(y0 + y1) - y0),
                             edge_col=edge_col, edge_row=edge_row,
                             deriv_off=box + W * H if derivs else -1)

    def finish():
        plan.run()
        buf = plan._mog_host
        sx0, sx1, sy0, sy1 = plan.ring_extent(ring)
        planes = [buf[box:box + W * H].reshape(H, W).astype(np.float64)]
        if derivs:
            for k in (1, 2):
                planes.append(buf[box + k * W * H:box + (k + 1) * W * H].reshape(H, W)
                              .astype(np.float64))
        px0, py0 = x0, y0
        if doslice:
            planes = [p[sy0:sy1, sx0:sx1].copy() for p in planes]
            px0 += sx0
            py0 += sy0
        if derivs:
            return tuple(Patch(px0, py0, p) for p in planes)
        return Patch(px0, py0, planes[0])
    return Pending(finish)
