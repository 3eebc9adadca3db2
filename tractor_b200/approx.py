"""The ring-grown evaluation region of c_gauss_2d_approx3
(tractor/approx3.c:1-465) over GPU-evaluated pixel values.

The GPU evaluates the mixture on the whole box with approx3's per-component
floors (and, if asked, the d/dmean planes); this module decides which pixels
approx3 would have evaluated and zeroes the rest, so the result equals the
reference's.  Rules, as in approx3.c: start at (xc, yc) or, if that is outside
the box, at the brightest pixel of the nearest box edge(s) under the plain
evaluation; visit square rings R = 1, 2, ...; a ring pixel is evaluated when
a passing pixel of the previous ring marked it (passing: R <= minradius or
value >= minval); top / bottom rows own the ring corners; stop at the first
ring with nothing evaluated.  The returned extent is updated only by the
rows (y) and columns (x) of each ring, exactly as approx3.c does.
"""
import numpy as np

from . import render
from .plan import Pending
from .patch import Patch


def ring_region(vals, cx, cy, minval, minradius):
    """Boolean mask of evaluated pixels and (sx0, sx1, sy0, sy1) (exclusive
    upper bounds), for box-relative start pixel (cx, cy)."""
    H, W = vals.shape
    ev = np.zeros((H, W), bool)

    def mark(arr, i, n):
        if 0 <= i < n:
            arr[i] = True

    nT, nB = np.zeros(W, bool), np.zeros(W, bool)
    nL, nR = np.zeros(H, bool), np.zeros(H, bool)
    if cy > 0:
        for d in (-1, 0, 1):
            mark(nB, cx + d, W)
    if cy < H - 1:
        for d in (-1, 0, 1):
            mark(nT, cx + d, W)
    if cx > 0:
        mark(nL, cy, H)
    if cx < W - 1:
        mark(nR, cy, H)
    ev[cy, cx] = True
    sx0 = sx1 = cx
    sy0 = sy1 = cy

    def spread(marks, n):
        """Union of i-1, i, i+1 over marked i, clipped to [0, n)."""
        out = marks.copy()
        out[1:] |= marks[:-1]
        out[:-1] |= marks[1:]
        return out

    R = 1
    while True:
        cT, cB, cL, cR = nT, nB, nL, nR
        nT, nB = np.zeros(W, bool), np.zeros(W, bool)
        nL, nR = np.zeros(H, bool), np.zeros(H, bool)
        anyev = False
        # top (y = cy + R), bottom (y = cy - R)
        for side in (0, 1):
            y = cy + R if side == 0 else cy - R
            if not (0 <= y < H):
                continue
            cur = cT if side == 0 else cB
            idx = np.flatnonzero(cur)
            if len(idx) == 0:
                continue
            anyev = True
            ev[y, idx] = True
            if side == 0:
                sy1 = y
            else:
                sy0 = y
            ok = np.zeros(W, bool)
            ok[idx] = (R <= minradius) | (vals[y, idx] >= minval)
            inward = -1 if side == 0 else 1
            if cx - R > 0 and 0 <= cx - R < W and ok[cx - R]:
                mark(nL, y, H)
                mark(nL, y + inward, H)
            if cx + R < W - 1 and 0 <= cx + R < W and ok[cx + R]:
                mark(nR, y, H)
                mark(nR, y + inward, H)
            if (side == 0 and y < H - 1) or (side == 1 and y > 0):
                nxt = spread(ok, W)
                if side == 0:
                    nT |= nxt
                else:
                    nB |= nxt
        # left (x = cx - R), right (x = cx + R)
        for side in (0, 1):
            x = cx - R if side == 0 else cx + R
            if not (0 <= x < W):
                continue
            cur = cL if side == 0 else cR
            idx = np.flatnonzero(cur)
            if len(idx) == 0:
                continue
            anyev = True
            ev[idx, x] = True
            if side == 0:
                sx0 = x
            else:
                sx1 = x
            ok = np.zeros(H, bool)
            ok[idx] = (R <= minradius) | (vals[idx, x] >= minval)
            if (side == 0 and x > 0) or (side == 1 and x < W - 1):
                nxt = spread(ok, H)
                if side == 0:
                    nL |= nxt
                else:
                    nR |= nxt
        if not anyev:
            break
        R += 1
    return ev, (sx0, sx1 + 1, sy0, sy1 + 1)


def plan_approx3(plan, mix, x0, x1, y0, y1, fx, fy, minval, xc, yc, minradius=3,
                 doslice=True, derivs=False):
    """Pending result of evaluate_grid_approx3 (mixture_profiles.py:333-399):
    a Patch, or (patch, dx, dy) with derivs."""
    W, H = x1 - x0, y1 - y0
    box = plan.mog.add(x0, y0, W, H, mix.amp, mix.mean, mix.var, fx=fx, fy=fy, minval=minval,
                       derivs=derivs)
    edges = []
    if xc < x0 or xc >= x1:
        ex = x0 if xc < x0 else x1 - 1
        edges.append(('col', ex, plan.add_mog(ex, y0, 1, H, mix.amp, mix.mean, mix.var, fx=fx,
                                              fy=fy, floor=-100.)))
    if yc < y0 or yc >= y1:
        ey = y0 if yc < y0 else y1 - 1
        edges.append(('row', ey, plan.add_mog(x0, ey, W, 1, mix.amp, mix.mean, mix.var, fx=fx,
                                              fy=fy, floor=-100.)))

    def finish():
        plan.run()
        buf = plan._mog_host
        vals = buf[box:box + W * H].reshape(H, W).astype(np.float64)
        cx, cy = xc, yc
        if edges:
            best = 0.
            bx, by = (x0 + x1) // 2, (y0 + y1) // 2
            for kind, e, h in edges:
                v = plan.get(h).ravel()
                for i, val in enumerate(v):
                    if val > best:
                        best = val
                        if kind == 'col':
                            bx, by = e, y0 + i
                        else:
                            bx, by = x0 + i, e
            cx, cy = bx, by
        ev, (sx0, sx1, sy0, sy1) = ring_region(vals, cx - x0, cy - y0, minval, minradius)
        res = np.where(ev, vals, 0.)
        planes = [res]
        if derivs:
            for k in (1, 2):
                d = buf[box + k * W * H:box + (k + 1) * W * H].reshape(H, W).astype(np.float64)
                planes.append(np.where(ev, d, 0.))
        px0, py0 = x0, y0
        if doslice:
            planes = [p[sy0:sy1, sx0:sx1].copy() for p in planes]
            px0 += sx0
            py0 += sy0
        if derivs:
            return tuple(Patch(px0, py0, p) for p in planes)
        return Patch(px0, py0, planes[0])
    return Pending(finish)
