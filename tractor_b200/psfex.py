"""Spatially varying pixelized PSFs from PsfEx models (tractor/psfex.py).

A PsfEx model is a set of eigen-PSF images combined with polynomial weights
in the image position.  PixelizedPsfEx renders point sources by Lanczos-3
shifting the model's image at the source's position, and gives galaxies the
Fourier path with the spectrum of that image (tb_psf_spectrum); the
reference sums the bases' spectra with the same weights, which is the same
linear combination.  Models are read from PsfEx FITS files (a numpy FITS
reader, `fitsbin`), from rows of merged tables, or built from their arrays.
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

    def __init__(self, fn=None, ext=1, Ti=None, bases=None, degree=0, x0=0., y0=0., xscale=1.,
                 yscale=1., sampling=1., fwhm=None):
        """From a PsfEx FITS file `fn` (extension `ext`), from one row `Ti`
        of a merged PsfEx table (tractor/psfex.py:160-232), or from the bases
        and polynomial given as arrays."""
        if fn is not None:
            self._from_file(fn, ext)
            return
        if Ti is not None:
            self._from_row(Ti)
            return
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

    def _set_bases(self, ims, degree):
        ne = (degree + 1) * (degree + 2) // 2
        ims = np.asarray(ims).astype(np.float32)
        assert ims.ndim == 3 and ims.shape[0] == ne
        self.psfbases = ims
        self.degree = degree
        bh, bw = self.psfbases[0].shape
        self.radius = (bh + 1) / 2.

    def _from_file(self, fn, ext):
        # psfex.py:166-206: the PSF_MASK column's first row holds the bases
        from .fitsbin import read_table
        hdr, cols = read_table(fn, ext)
        ims = cols['psf_mask'][0]
        ngrp = hdr['POLNGRP']
        assert ngrp in [0, 1]
        if ngrp == 0:
            degree, x0, y0, xscale, yscale = 0, 0., 0., 1., 1.
        else:
            assert str(hdr['POLNAME1']).strip() in ['X_IMAGE', 'XWIN_IMAGE']
            assert str(hdr['POLNAME2']).strip() in ['Y_IMAGE', 'YWIN_IMAGE']
            assert hdr['POLGRP1'] == 1
            assert hdr['POLGRP2'] == 1
            x0, xscale = hdr.get('POLZERO1'), hdr.get('POLSCAL1')
            y0, yscale = hdr.get('POLZERO2'), hdr.get('POLSCAL2')
            degree = hdr.get('POLDEG1')
        self.sampling = hdr.get('PSF_SAMP')
        ne = (degree + 1) * (degree + 2) // 2
        assert hdr['PSFAXIS3'] == ne
        self._set_bases(ims, degree)
        self.xscale, self.yscale = xscale, yscale
        self.x0, self.y0 = x0, y0
        self.fwhm = hdr.get('PSF_FWHM')

    def _from_row(self, Ti):
        # psfex.py:208-232
        self.sampling = Ti.psf_samp
        degree = Ti.poldeg1
        if degree > 0:
            assert Ti.polname1.strip() == 'X_IMAGE'
            assert Ti.polname2.strip() == 'Y_IMAGE'
            assert Ti.polgrp1 == 1
            assert Ti.polgrp2 == 1
            assert Ti.polngrp == 1
        self.x0, self.y0 = Ti.polzero1, Ti.polzero2
        self.xscale, self.yscale = Ti.polscal1, Ti.polscal2
        assert Ti.psfaxis3 == (degree + 1) * (degree + 2) // 2
        self._set_bases(Ti.psf_mask, degree)
        self.fwhm = Ti.psf_fwhm

    def writeto(self, fn):
        """PsfExModel.writeto (psfex.py:234-257): one PSF_MASK row and the
        polynomial's header keywords."""
        from .fitsbin import write_table
        ne = (self.degree + 1) * (self.degree + 2) // 2
        hdr = dict(POLNAME1='X_IMAGE', POLNAME2='Y_IMAGE', POLGRP1=1, POLGRP2=1, POLNGRP=1,
                   PSFAXIS3=ne, POLZERO1=self.x0, POLZERO2=self.y0, POLSCAL1=self.xscale,
                   POLSCAL2=self.yscale, POLDEG1=self.degree, PSF_SAMP=self.sampling,
                   PSF_FWHM=self.fwhm)
        write_table(fn, {'psf_mask': np.array([self.psfbases])}, header=hdr)

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
    (tractor/psfex.py:428-521), read from the PsfEx FITS file `fn` or given
    as `psfex`.  Oversampled models (PSF_SAMP != 1) are not provided."""

    def __init__(self, fn=None, ext=1, psfexmodel=PsfExModel, psfex=None):
        if psfex is None:
            psfex = psfexmodel(fn, ext=ext)
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
