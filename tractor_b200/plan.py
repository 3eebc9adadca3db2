"""Deferred GPU rendering.

A RenderPlan collects the renders that one reference-level call needs --
mixture-of-Gaussians rectangles, Fourier-path galaxies and Lanczos-shifted
PSF stamps -- runs each kind in one batched launch, copies the results to
the host once, and then resolves the pending Patch objects.  Source and PSF
classes add to a plan through their _plan_* methods; the reference-facing
methods (getModelPatch, getParamDerivatives, ...) create a plan, add their
renders and resolve it, while Tractor-level calls share one plan across all
sources.
"""
import numpy as np
import torch

from . import render
from .patch import Patch


class Pending(object):
    """A value computed after the plan runs: `fn()` builds it."""

    def __init__(self, fn):
        self.fn = fn

    def result(self):
        return self.fn()


NONE = Pending(lambda: None)


def done(value):
    return Pending(lambda: value)


class RenderPlan(object):

    def __init__(self):
        self.mog = render.MogBatch()
        self.fft = render.FftBatch()
        self.lanczos = {}     # (h, w) -> list of (stamp, dx, dy, index)
        self.nlz = 0
        self._ran = False
        self._mog_host = None
        self._ring_host = None
        self._fft_host = None
        self._lz_host = {}

    # -- adding work -----------------------------------------------------
    def add_mog(self, x0, y0, w, h, amp, mean, var, fx=0., fy=0., floor=render.FLOOR_GRID,
                mask=None, diff=None):
        """Mixture on [x0, x0+w) x [y0, y0+h); returns a handle to its float32
        (h, w) result.  `diff` = (amp2, var2): the result is mixture 2 minus
        this one (same means), rendered as one difference item."""
        if w <= 0 or h <= 0:
            return ('empty', h, w)
        off = self.mog.add(x0, y0, w, h, amp, mean, var, fx=fx, fy=fy, floor=floor, mask=mask,
                           diff=diff)
        return ('mog', off, h, w)

    def add_fft(self, amp, var, sz, spec_key, spec, mw, mh, sx, sy, mux, muy, diff=None):
        if mw <= 0 or mh <= 0:
            return ('empty', mh, mw)
        off = self.fft.add(amp, var, sz, spec_key, spec, mw, mh, sx, sy, mux, muy, diff=diff)
        return ('fft', off, mh, mw)

    def add_lanczos(self, stamp, dx, dy):
        stamp = np.ascontiguousarray(stamp, np.float32)
        key = stamp.shape
        lst = self.lanczos.setdefault(key, [])
        lst.append((stamp, float(dx), float(dy)))
        return ('lz', key, len(lst) - 1)

    # -- running -----------------------------------------------------------
    def run(self):
        if self._ran:
            return
        self._ran = True
        outs = []
        if len(self.mog):
            if self.mog.rings or render.device().type != 'cuda':
                outs.append(('mog', self.mog.run(check=False)))
            else:
                # staging, launch and read-back in one library call
                self._mog_host = self.mog.run_host()
        if len(self.fft):
            outs.append(('fft', self.fft.run(check=False)))
        lz = {}
        for key, lst in self.lanczos.items():
            imgs = torch.from_numpy(np.stack([s for s, _, _ in lst])).to(render.device())
            shifts = np.array([[dx, dy] for _, dx, dy in lst])
            lz[key] = render.lanczos_shift(imgs, shifts)
        stream = None
        for kind, t in outs:
            # the status word rides at the end
            if t.device.type == 'cuda':
                if stream is None:
                    stream = torch.cuda.current_stream()
                host = render.to_host(t, np.float32, stream)
            else:
                host = t.numpy().copy()
            st = host[-4:]
            if kind == 'mog':
                render.check_status_host(st, 'tb_mog_render')
                if self.mog.extents is not None:
                    render.check_status(self.mog.ring_status, 'tb_approx3_region')
                    self._ring_host = self.mog.extents.cpu().numpy().reshape(-1, 4)
                self._mog_host = host
            else:
                render.check_status_host(st, 'tb_fourier_render')
                self._fft_host = host
        for key, t in lz.items():
            self._lz_host[key] = t.cpu().numpy()

    def get(self, handle):
        """float32 host array of a finished render (a view into the batch
        buffer; copy before modifying in place)."""
        self.run()
        kind = handle[0]
        if kind == 'empty':
            return np.zeros((handle[1], handle[2]), np.float32)
        if kind == 'mog':
            _, off, h, w = handle
            return self._mog_host[off:off + h * w].reshape(h, w)
        if kind == 'fft':
            _, off, h, w = handle
            return self._fft_host[off:off + h * w].reshape(h, w)
        if kind == 'lz':
            _, key, i = handle
            return self._lz_host[key][i]
        raise KeyError(kind)

    def ring_extent(self, i):
        """(sx0, sx1, sy0, sy1) of approx3 region walk i (MogBatch.add_ring)."""
        self.run()
        return tuple(int(v) for v in self._ring_host[i])

    def patch(self, x0, y0, handle, dtype=np.float32):
        return Patch(x0, y0, np.array(self.get(handle), dtype=dtype))


def resolve(pending_list):
    return [p.result() if p is not None else None for p in pending_list]
