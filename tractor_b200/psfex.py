"""Spatially varying pixelized PSFs from PsfEx models (tractor/psfex.py).

A PsfEx model is a set of eigen-PSF images combined with polynomial weights
in the image position.  PixelizedPsfEx renders point sources by Lanczos-3
shifting the model's image at the source's position, and gives galaxies the
Fourier path with the spectrum of that image (tb_psf_spectrum); the
reference sums the bases' spectra with the same weights, which is the same
linear combination.  Reading PsfEx FITS files is not provided: models are
built from their arrays.
"""
import numpy as np

from . import render
from .psf import PixelizedPSF


class PsfExModel(object):
    """Eigen-PSF bases and their polynomial weights (tractor/psfex.py:155-345).

    bases: (nb, H, W) float32 images, nb = (degree + 1)(degree + 2) / 2;
    the weight of basis ii at (x, y) is dx^j dy^k with dx = (x - x0) / xscale,
    dy = (y - y0) / yscale, ii = j + (degree + 1) k - k (k - 1) / 2 (the
    PSFEx term order: total degree d = j + k outer, j inner)."""

    def __init__(self, bases=None, degree=0, x0=0., y0=0., xscale=1., yscale=1., sampling=1.,
                 fwhm=None):
        if bases is None:
            return
        bases = np.asarray(bases, np.float32)
        assert bases.ndim == 3 and bases.shape[0] == (degree + 1) * (degree + 2) // 2
        self.psfbases = bases
        self.degree = int(degree)
        self.x0, self.y0 = float(x0), float(y0)
        self.xscale, self.yscale = float(xscale), float(yscale)
        self.sampling = sampling
        bh, bw = bases[0].shape
        self.radius = (bh + 1) / 2.
        self.fwhm = fwhm

    @property
    def shape(self):
        return self.psfbases[0].shape

    @property
    def nbases(self):
        return self.psfbases.shape[0]

    def copy(self):
        return self.shifted(0., 0.)

    def shifted(self, dx, dy):
        c = self.__class__()
        for key in ['sampling', 'psfbases', 'xscale', 'yscale', 'degree', 'radius', 'x0', 'y0',
                    'fwhm']:
            setattr(c, key, getattr(self, key))
        c.shift(dx, dy)
        return c

    def shift(self, dx, dy):
        """The model applies to the subimage starting at (dx, dy)."""
        self.x0 -= dx
        self.y0 -= dy

    def bases(self):
        return self.psfbases

    def polynomials(self, x, y, powers=False):
        dx = (x - self.x0) / self.xscale
        dy = (y - self.y0) / self.yscale
        nb = self.nbases
        terms = np.zeros(nb)
        xp = np.zeros(nb, int)
        yp = np.zeros(nb, int)
        for d in range(self.degree + 1):
            for j in range(d + 1):
                k = d - j
                ii = j + (self.degree + 1) * k - (k * (k - 1)) // 2
                terms[ii] = dx ** j * dy ** k
                xp[ii], yp[ii] = j, k
        if powers:
            return terms, xp, yp
        return terms

    def at(self, x, y):
        """The PSF image at pixel (x, y) (float32, accumulated term by term)."""
        psf = np.zeros_like(self.psfbases[0])
        for term, base in zip(self.polynomials(x, y), self.psfbases):
            psf += term * base
        return psf


class PixelizedPsfEx(PixelizedPSF):
    """PixelizedPSF whose image varies over the image as a PsfEx model
    (tractor/psfex.py:428-521).  `fn` (a PsfEx FITS file) is not supported:
    pass the model as `psfex`."""

    def __init__(self, fn=None, ext=1, psfex=None):
        if fn is not None:
            raise NotImplementedError('reading PsfEx files is not provided; pass psfex=PsfExModel')
        super(PixelizedPsfEx, self).__init__(psfex.bases()[0], sampling=psfex.sampling)
        self.psfex = psfex
        self.fwhm = psfex.fwhm
        self.fn, self.ext = fn, ext

    def __str__(self):
        return 'PixelizedPsfEx'

    def hashkey(self):
        return ('PixelizedPsfEx', id(self.psfex))

    def copy(self):
        return self.__class__(None, psfex=self.psfex.copy())

    def getShifted(self, dx, dy):
        return self.__class__(None, psfex=self.psfex.shifted(dx, dy))

    def shift(self, dx, dy):
        self.psfex.shift(dx, dy)

    def constantPsfAt(self, x, y):
        return PixelizedPSF(self.psfex.at(x, y), sampling=self.sampling)

    def getImage(self, px, py):
        return self.psfex.at(px, py)

    def fourier_spectrum(self, px, py, sz):
        """The spectrum of the model's image at (px, py) (not cached: it
        depends on the position)."""
        spec, cx, cy = render.psf_spectra().compute(self.getImage(px, py), sz)
        key = ('PixelizedPsfEx', id(self), float(px), float(py), self.psfex.x0, self.psfex.y0)
        return key, spec, cx, cy
