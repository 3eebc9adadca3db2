"""Analytic parameter derivatives of the pixelized-PSF (Fourier) path and of
the mixture-of-Gaussians PSF path (blobs of galaxies and point sources), each
behind a torch.autograd.Function.

For each galaxy, tb_galaxy_fft_jac_prep makes seven derivative items on the
geometry of its value item -- position (x, y) through the derivative of the
Lanczos-3 taps, counts (the unit-flux render), the three shape parameters and
the Sersic index through the derivative of the Gaussian-mixture spectrum,
d/dtheta sum_k a_k exp(-2 pi^2 f^T C_k f) = sum_k (da_k - 2 pi^2 a_k
f^T dC_k f) exp(...) -- and tb_fourier_render_deriv renders them through the
same FFT / Lanczos / crop pipeline as the model.  In TB_FFT_DOT mode the
kernel contracts each derivative item with an upstream gradient instead of
writing it (the vector-Jacobian product), so backward never materialises
the Jacobian.

These replace the finite-difference derivatives of Galaxy.getParamDerivatives
and SersicGalaxy.getParamDerivatives (tractor/galaxy.py:137-223,
tractor/sersic.py:402-445) where exact derivatives are wanted.  The seven
parameters are the first seven fields of a GALAXY_SRC record: px, py,
counts, s0, s1, s2 (shape, per shape_type) and sersic_n.
"""
import ctypes

import numpy as np
import torch

from . import _lib, batch, render

NPARAM = 7
PARAM_NAMES = ('x', 'y', 'counts', 's0', 's1', 's2', 'sersic_n')


class FourierJacobian(object):
    """Derivative items for the galaxies of a FourierGalaxyRenderer (same PSF
    spectra, WCS and profile tables)."""

    def __init__(self, renderer):
        self.r = renderer
        self._scratch = {}

    def _work(self, n):
        if n not in self._scratch:
            dev = render.device()
            S = batch.COMP_STRIDE
            items = torch.empty(7 * n * _lib.FFT_ITEM.itemsize, dtype=torch.uint8, device=dev)
            camp = torch.empty(n * S, dtype=torch.float64, device=dev)
            cvar = torch.empty(n * S * 4, dtype=torch.float64, device=dev)
            dcoef = torch.zeros(4 * n * S * 4, dtype=torch.float64, device=dev)
            flags = torch.empty(n, dtype=torch.int32, device=dev)
            misc = torch.zeros(8, dtype=torch.int32, device=dev)
            self._scratch[n] = (items, camp, cvar, dcoef, flags, misc)
        return self._scratch[n]

    def _run(self, srcs, n, out, mode, col_stride, dots=None, stream=None):
        lib = _lib.load()
        items, camp, cvar, dcoef, flags, misc = self._work(n)
        s = _lib.stream_ptr(stream)
        rc = lib.tb_galaxy_fft_jac_prep(srcs.data_ptr(), n, ctypes.addressof(self.r.image),
                                        ctypes.addressof(self.r.tables.struct), items.data_ptr(),
                                        camp.data_ptr(), cvar.data_ptr(), dcoef.data_ptr(),
                                        batch.COMP_STRIDE, mode, col_stride, flags.data_ptr(), s)
        _lib.check(rc, 'tb_galaxy_fft_jac_prep')
        render.fourier_render(items.data_ptr(), 7 * n, camp.data_ptr(), cvar.data_ptr(),
                              self.r.spec.data_ptr(), out.data_ptr(), misc.data_ptr() + 16,
                              dcoef_ptr=dcoef.data_ptr(),
                              dots_ptr=None if dots is None else dots.data_ptr(), stream=stream)
        return flags, misc[4:8]

    def jacobian(self, srcs, n, npix, stream=None):
        """float32 (7, npix) device tensor: row j holds d(model)/d(param j)
        of every galaxy, each at its record's out_off (the layout of the
        value patches).  Also returns the prep flags."""
        out = torch.empty(7 * npix, dtype=torch.float32, device=render.device())
        flags, st = self._run(srcs, n, out, _lib.MOG_STORE, npix, stream=stream)
        return out.view(7, npix), flags, st

    def vjp(self, srcs, n, grad, stream=None):
        """float64 (n, 7): sum over each galaxy's patch of grad * d(model)/
        d(param), grad laid out like the value patches (one kernel: the
        derivative renders are contracted as they are produced)."""
        dots = torch.zeros(7 * n, dtype=torch.float64, device=render.device())
        flags, st = self._run(srcs, n, grad.contiguous(), _lib.FFT_DOT, 0, dots=dots,
                              stream=stream)
        return dots.view(n, 7), flags, st


def records_with_params(template, theta):
    """Device GALAXY_SRC records: `template` (uint8 device tensor of records)
    with its first seven fields replaced by theta (n, 7) float64."""
    n = theta.shape[0]
    rec = template.clone()
    rec.view(torch.float64).view(n, _lib.GALAXY_SRC.itemsize // 8)[:, :NPARAM] = theta
    return rec


class RenderGalaxies(torch.autograd.Function):
    """model = RenderGalaxies.apply(theta, renderer, template, npix):
    the galaxies' model patches (float32, the template records' layout) as
    a differentiable function of theta (n, 7) float64 = (x, y, counts, s0,
    s1, s2, n).  Backward is the analytic vector-Jacobian product of
    FourierJacobian.vjp."""

    @staticmethod
    def forward(ctx, theta, renderer, template, npix):
        n = theta.shape[0]
        rec = records_with_params(template, theta.detach())
        out = torch.empty(npix, dtype=torch.float32, device=theta.device)
        flags = renderer.render_device(rec, n, out)
        ctx.renderer = renderer
        ctx.rec = rec
        ctx.n = n
        ctx.mark_non_differentiable(flags)
        return out, flags

    @staticmethod
    def backward(ctx, grad_out, grad_flags):
        jac = getattr(ctx.renderer, '_jacobian', None)
        if jac is None:
            jac = ctx.renderer._jacobian = FourierJacobian(ctx.renderer)
        g, _, _ = jac.vjp(ctx.rec, ctx.n, grad_out.float())
        return g, None, None, None


# ---------------------------------------------------------------------------
# Mixture-of-Gaussians PSF path: blobs of point sources and galaxies
# ---------------------------------------------------------------------------

class BlobModel(object):
    """The model images of a BlobFitter's blobs as a function of their
    parameters (n_src, 9: x, y, flux per band, log r_e, ee1, ee2, Sersic n),
    and the analytic vector-Jacobian product, both from tb_fit_model_vjp
    (FP64 evaluation: the sources' PSF-convolved mixtures over their masks,
    the derivative columns of Galaxy.getParamDerivatives /
    PointSource.getParamDerivatives, tractor/galaxy.py:137-223,
    tractor/pointsource.py:130-241, taken analytically).  The images are laid
    out as the fitter's data (fit.pix_offsets)."""

    def __init__(self, fitter):
        self.f = fitter
        f = fitter
        P = f.blobs_np['P'].astype(np.int64)
        ns = f.blobs_np['n_slices'].astype(np.int64)
        maxs = int(ns.max())
        blob_of = np.repeat(np.arange(f.n_blobs), np.diff(np.concatenate(
            [[0], np.cumsum(f.blobs_np['n_src'])])))
        first = np.concatenate([[0], np.cumsum(f.blobs_np['n_src'])[:-1]])
        idx = np.full((f.n_src * NPAR_FIT, maxs), int(f.gbuf.numel()), np.int64)
        for q in range(f.n_src * NPAR_FIT):
            s = q // NPAR_FIT
            b = blob_of[s]
            local = (s - first[b]) * NPAR_FIT + q % NPAR_FIT
            for k in range(int(ns[b])):
                idx[q, k] = int(f.blobs_np['g_off'][b]) + k * int(P[b]) + local
        # slot gbuf.numel() reads a zero appended to the slices
        self._idx = torch.from_numpy(idx).to(f.dev)

    def _prep(self, theta):
        f = self.f
        f.trial.copy_(theta.reshape(-1).to(torch.float64))
        f._prep(all_blobs=True)

    def _launch(self, mode, grad=None, model=None):
        f = self.f
        lib = _lib.load()
        _lib.check(lib.tb_fit_model_vjp(f.d_pass_units.data_ptr(), f.d_order.data_ptr(),
                                        len(f.pass_units_np), f.d_blobs.data_ptr(),
                                        f.d_sources.data_ptr(), f.n_src, f.workspace.data_ptr(),
                                        None if grad is None else grad.data_ptr(),
                                        None if model is None else model.data_ptr(),
                                        f.d_tiles.data_ptr(), f.gbuf.data_ptr(), f.n_bands, mode,
                                        f.misc.data_ptr(), f.misc.data_ptr() + 16,
                                        _lib.stream_ptr()), 'tb_fit_model_vjp')
        render.check_status(f.misc[4:8].clone(), 'tb_fit_model_vjp')

    def model(self, theta):
        """float32 (npix,) device tensor of the blobs' model images."""
        self._prep(theta)
        out = torch.zeros(int(self.f.pix_offsets[-1]), dtype=torch.float32, device=self.f.dev)
        self._launch(_lib.FIT_MODEL, model=out)
        return out

    def vjp(self, theta, grad):
        """float64 (n_src, 9): sum over the images of grad * d(model)/d(theta)."""
        self._prep(theta)
        g = grad.contiguous().to(torch.float32)
        self._launch(_lib.FIT_VJP, grad=g)
        ext = torch.cat([self.f.gbuf, torch.zeros(1, dtype=torch.float64, device=self.f.dev)])
        return ext[self._idx].sum(dim=1).view(self.f.n_src, NPAR_FIT)


NPAR_FIT = _lib.FIT_NPAR


class RenderBlobs(torch.autograd.Function):
    """model = RenderBlobs.apply(theta, blob_model): the blobs' model images
    (float32, the fitter's data layout) as a differentiable function of theta
    (n_src, 9) float64; backward is BlobModel.vjp, the analytic
    vector-Jacobian product (no finite differences, no Jacobian in memory)."""

    @staticmethod
    def forward(ctx, theta, blob_model):
        ctx.blob_model = blob_model
        ctx.save_for_backward(theta)
        return blob_model.model(theta.detach())

    @staticmethod
    def backward(ctx, grad_out):
        theta, = ctx.saved_tensors
        return ctx.blob_model.vjp(theta.detach(), grad_out), None
