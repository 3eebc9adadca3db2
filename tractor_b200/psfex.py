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
from .params import MultiParams
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


class VaryingGaussianPSF(MultiParams):
    """A mixture-of-Gaussians PSF varying over the image: the mixture is fit
    at an nx x ny grid of positions and each of its parameters interpolated
    by a bicubic spline (tractor/psfex.py:8-150).  Subclasses provide
    `instantiateAt(x, y)`, the PSF image at a position.

    The grid fits: for the default psfClass (GaussianMixturePSF, fitted by
    EM) all grid points are fitted in one batched launch, each from
    fromStamp's default start (the reference starts each fit from the
    previous one's flat parameter list, which GaussianMixturePSF.fromStamp
    cannot unpack); for other classes (GaussianMixtureEllipsePSF, or a given
    `fitfunc`) the fits run one after another, each started from the
    previous one as the reference does."""

    def __init__(self, W, H, nx=11, ny=11, K=3, psfClass=None):
        super(VaryingGaussianPSF, self).__init__()
        from .psf import GaussianMixturePSF
        self.psfclass = GaussianMixturePSF if psfClass is None else psfClass
        self.splines = None
        self.W, self.H = W, H
        self.K = K
        self.nx, self.ny = nx, ny
        self.savesplinedata = False

    def __str__(self):
        return '%s: %s, %i x %i' % (type(self).__name__, self.psfclass.__name__, self.nx,
                                    self.ny)

    def getShifted(self, x0, y0):
        return _ShiftedMogPsf(self, x0, y0)

    def getRadius(self):
        return getattr(self, 'radius', 25.)

    def fitSavedData(self, pp, XX, YY):
        import scipy.interpolate
        self.splines = [scipy.interpolate.RectBivariateSpline(XX, YY, pp[:, :, i].T)
                        for i in range(len(pp[0][0]))]

    def ensureSplines(self):
        if self.splines is None:
            self.fitSavedData(*self.splinedata)

    def ensureFit(self):
        if self.splines is None:
            self._fitParamGrid()

    def psfParamsAt(self, x, y):
        """The mixture parameters at pixel (x, y) (psfex.py:85-101)."""
        self.ensureFit()
        return np.array([float(spl(x, y, grid=False)) for spl in self.splines])

    def psfAt(self, x, y):
        return self.psfclass(*self.psfParamsAt(x, y))

    mogAt = psfAt

    def getMixtureOfGaussians(self, px=None, py=None):
        return self.psfAt(0. if px is None else px, 0. if py is None else py) \
            .getMixtureOfGaussians()

    def getPointSourcePatch(self, px, py, **kwargs):
        return self.psfAt(px, py).getPointSourcePatch(px, py, **kwargs)

    def _plan_point_source(self, plan, px, py, **kwargs):
        return self.psfAt(px, py)._plan_point_source(plan, px, py, **kwargs)

    def _fitParamGrid(self, fitfunc=None, trim=0, **kwargs):
        """Fits the mixture at the grid points (psfex.py:118-150)."""
        from .psf import GaussianMixturePSF
        YY = np.linspace(0, self.H, self.ny)
        XX = np.linspace(0, self.W, self.nx)
        stamps = []
        for y in YY:
            for x in XX:
                im = self.instantiateAt(x, y)
                if trim > 0:
                    im = im[trim:-trim, trim:-trim]
                stamps.append(im)
        if fitfunc is None and self.psfclass is GaussianMixturePSF:
            psfs = GaussianMixturePSF.fromStamps(stamps, N=self.K, **kwargs)
            if any(p is None for p in psfs):
                raise RuntimeError('VaryingGaussianPSF: an EM fit failed (non-positive '
                                   'covariance determinant)')
            flat = [np.array(p.getAllParams()) for p in psfs]
        else:
            f = fitfunc if fitfunc is not None else self.psfclass.fromStamp
            flat, p0, px0 = [], None, None
            for iy in range(self.ny):
                p0 = px0
                for ix in range(self.nx):
                    psf = f(stamps[iy * self.nx + ix], N=self.K, P0=p0, **kwargs)
                    p0 = psf.getParams()
                    if ix == 0:
                        px0 = p0
                    flat.append(np.array(psf.getAllParams()))
        pp = np.array(flat).reshape(self.ny, self.nx, -1)
        self.fitSavedData(pp, XX, YY)
        if self.savesplinedata:
            self.splinedata = (pp, XX, YY)


class _ShiftedMogPsf(object):
    """A position-dependent PSF seen from a subimage starting at (x0, y0)
    (tractor/shifted.py:63-110): positions are shifted into the parent's
    frame and patches shifted back."""

    def __init__(self, psf, x0, y0):
        self.psf, self.x0, self.y0 = psf, x0, y0

    def __str__(self):
        return ('ShiftedPsf: %i,%i + ' % (self.x0, self.y0)) + str(self.psf)

    def hashkey(self):
        return ('ShiftedPsf', self.x0, self.y0) + tuple(self.psf.hashkey())

    def getRadius(self):
        return self.psf.getRadius()

    def getMixtureOfGaussians(self, px=None, py=None):
        return self.psf.getMixtureOfGaussians(px=(px or 0.) + self.x0, py=(py or 0.) + self.y0)

    def _plan_point_source(self, plan, px, py, **kwargs):
        # the mixture of the parent's position, rendered at the subimage's
        return self.psf.psfAt(px + self.x0, py + self.y0)._plan_point_source(plan, px, py,
                                                                             **kwargs)

    def getPointSourcePatch(self, px, py, **kwargs):
        return self.psf.psfAt(px + self.x0, py + self.y0).getPointSourcePatch(px, py, **kwargs)


class VaryingGaussianPsfEx(VaryingGaussianPSF):
    """VaryingGaussianPSF of a PsfEx model read from `fn`
    (tractor/psfex.py:522-553): the grid images are the model's images."""

    def __init__(self, fn, W, H, ext=1, scale=True, nx=11, ny=11, K=3, psfClass=None):
        assert scale
        self.psfex = PsfExModel(fn, ext=ext)
        self.scale = scale
        super(VaryingGaussianPsfEx, self).__init__(W, H, nx, ny, K, psfClass=psfClass)

    def instantiateAt(self, x, y):
        return self.psfex.at(x, y)


# the reference's original name for VaryingGaussianPsfEx
PsfEx = VaryingGaussianPsfEx
