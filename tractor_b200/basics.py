"""Positions, WCS, brightnesses, photometric calibration, sky and Image, with
the reference Tractor's semantics (tractor/wcs.py, tractor/brightness.py,
tractor/sky.py, tractor/image.py, tractor/ducks.py)."""
import numpy as np

from .params import BaseParams, ScalarParam, ParamList, MultiParams
from .patch import Patch


# ---------------------------------------------------------------------------
# Positions and WCS
# ---------------------------------------------------------------------------

class PixPos(ParamList):
    """Pixel position (tractor/wcs.py:373-390): step 0.1, max step 1."""

    @staticmethod
    def getNamedParams():
        return dict(x=0, y=1)

    def __init__(self, *args):
        super(PixPos, self).__init__(*args)
        self.stepsizes = [0.1, 0.1]
        self.maxstep = [1., 1.]

    def __str__(self):
        return 'pixel (%.2f, %.2f)' % (self.x, self.y)

    def getDimension(self):
        return 2


class NullWCS(BaseParams):
    """Identity WCS for pixel positions (tractor/wcs.py:8-49).

    cd_inverse is I / (pixscale / 3600), as in the reference; note that the
    reference's pixelDerivsToPositionDerivs (tractor/ducks.py:413-423) scales
    PixPos derivatives by it, which this class reproduces exactly."""

    def __init__(self, pixscale=1., dx=0., dy=0.):
        self.dx = dx
        self.dy = dy
        self.setPixscale(pixscale)

    def hashkey(self):
        return ('NullWCS', self.dx, self.dy)

    def copy(self):
        return NullWCS(self.pixscale, self.dx, self.dy)

    def setPixscale(self, pixscale):
        self.pixscale = pixscale
        self.cd = np.array([[1., 0.], [0., 1.]]) * self.pixscale / 3600.
        self.cd_inverse = np.array([[1., 0.], [0., 1.]]) / (self.pixscale / 3600.)

    def positionToPixel(self, pos, src=None):
        return pos.x + self.dx, pos.y + self.dy

    def pixelToPosition(self, x, y, src=None):
        return PixPos(x - self.dx, y - self.dy)

    def cdAtPixel(self, x, y):
        return self.cd

    def cdInverseAtPixel(self, x, y):
        return self.cd_inverse

    def cdInverseAtPosition(self, pos, src=None):
        return self.cd_inverse

    def pixscale_at(self, x, y):
        return self.pixscale

    def shifted(self, x, y):
        return self.copy()

    def pixelDerivsToPositionDerivs(self, pos, src, counts0, patch0, patchdx, patchdy):
        """tractor/ducks.py:413-423."""
        cdi = self.cdInverseAtPosition(pos, src=src)
        derivs = []
        for i, pname in pos.getThawedParamIndicesAndNames():
            d = (patchdx * cdi[0, i] + patchdy * cdi[1, i]) * counts0
            d.setName('d(ptsrc)/d(pos.%s)' % pname)
            derivs.append(d)
        return derivs


# ---------------------------------------------------------------------------
# Brightness and photometric calibration
# ---------------------------------------------------------------------------

class Flux(ScalarParam):
    """Raw counts (tractor/brightness.py:14-24)."""

    def __mul__(self, factor):
        new = self.copy()
        new.val *= factor
        return new

    __rmul__ = __mul__


class Mag(ScalarParam):
    stepsize = -0.01
    strformat = '%.3f'


class MultiBandBrightness(ParamList):
    """Per-band values in a fixed band order (tractor/brightness.py:26-71)."""

    def __init__(self, **kwargs):
        keys = kwargs.pop('order', None)
        if keys is None:
            keys = sorted(kwargs.keys())
        assert set(kwargs.keys()) == set(keys)
        super(MultiBandBrightness, self).__init__(*[kwargs[k] for k in keys])
        self.order = list(keys)
        self.addNamedParams(**dict((k, i) for i, k in enumerate(keys)))

    def copy(self):
        return self * 1.

    def getBand(self, band):
        return getattr(self, band)

    def setBand(self, band, value):
        return setattr(self, band, value)


class Mags(MultiBandBrightness):
    """Magnitudes in several bands, for MagsPhotoCal (tractor/brightness.py:72-132)."""

    def __init__(self, **kwargs):
        super(Mags, self).__init__(**kwargs)
        self.stepsizes = [-0.01] * self.numberOfParams()

    def getMag(self, bandname):
        return self.getBand(bandname)

    def setMag(self, bandname, mag):
        return self.setBand(bandname, mag)

    def __add__(self, other):
        if np.isscalar(other):
            return Mags(order=self.order, **dict((b, self.getMag(b) + other) for b in self.order))
        # the magnitude of the summed fluxes
        return Mags(order=self.order,
                    **dict((b, -2.5 * np.log10(10. ** (-self.getMag(b) / 2.5) +
                                               10. ** (-other.getMag(b) / 2.5)))
                           for b in self.order))

    def __mul__(self, factor):
        # the magnitude of the flux scaled by |factor|
        dmag = -2.5 * np.log10(np.abs(factor))
        return self.__class__(order=self.order,
                              **dict((b, self.getMag(b) + dmag) for b in self.order))


class Fluxes(MultiBandBrightness):
    """tractor/brightness.py:135-161."""

    def __add__(self, other):
        return self.__class__(order=self.order,
                              **dict((b, self.getBand(b) + other.getBand(b)) for b in self.order))

    def __mul__(self, factor):
        return self.__class__(order=self.order,
                              **dict((b, self.getFlux(b) * factor) for b in self.order))

    def getFlux(self, band):
        return self.getBand(band)

    def setFlux(self, band, value):
        return self.setBand(band, value)


class NanoMaggies(Fluxes):
    """Linear calibrated fluxes (tractor/brightness.py:163-240)."""

    def __repr__(self):
        return str(self)

    def __str__(self):
        ss = []
        for b in self.order:
            f = self.getFlux(b)
            if f <= 0:
                ss.append('%s=(flux %.3g)' % (b, f))
            else:
                ss.append('%s=%.3f' % (b, self.getMag(b)))
        return 'NanoMaggies: ' + ', '.join(ss)

    def getMag(self, band):
        return NanoMaggies.nanomaggiesToMag(self.getFlux(band))

    @staticmethod
    def nanomaggiesToMag(nm):
        return -2.5 * (np.log10(nm) - 9)

    @staticmethod
    def magToNanomaggies(mag):
        return 10. ** ((mag - 22.5) / -2.5)

    @staticmethod
    def fromMag(mag):
        """NanoMaggies of a Mags (brightness.py:192-198)."""
        return NanoMaggies(order=mag.order,
                           **dict((k, NanoMaggies.magToNanomaggies(mag.getMag(k)))
                                  for k in mag.order))

    @staticmethod
    def zeropointToScale(zp):
        """The factor from nanomaggies to counts of a magnitude zeropoint."""
        return 10. ** ((zp - 22.5) / 2.5)

    @staticmethod
    def scaleToZeropoint(zpscale):
        """The magnitude zeropoint of a nanomaggies-to-counts factor."""
        return 22.5 + 2.5 * np.log10(zpscale)

    @staticmethod
    def fluxErrorsToMagErrors(flux, flux_invvar):
        """(mag, mag error) float32 arrays; NaN where the flux or its inverse
        variance is not positive (brightness.py:228-243)."""
        flux = np.atleast_1d(flux)
        flux_invvar = np.atleast_1d(flux_invvar)
        dflux = np.zeros(len(flux))
        okiv = flux_invvar > 0
        dflux[okiv] = 1. / np.sqrt(flux_invvar[okiv])
        okflux = flux > 0
        mag = np.zeros(len(flux))
        mag[okflux] = NanoMaggies.nanomaggiesToMag(flux[okflux])
        dmag = np.zeros(len(flux))
        ok = okiv * okflux
        dmag[ok] = np.abs((-2.5 / np.log(10.)) * dflux[ok] / flux[ok])
        mag[np.logical_not(okflux)] = np.nan
        dmag[np.logical_not(ok)] = np.nan
        return mag.astype(np.float32), dmag.astype(np.float32)


class FluxesPhotoCal(BaseParams):
    """counts = the flux in the calibration's band (brightness.py:246-259)."""

    def __init__(self, band):
        self.band = band
        BaseParams.__init__(self)

    def copy(self):
        return FluxesPhotoCal(self.band)

    def brightnessToCounts(self, brightness):
        return brightness.getFlux(self.band)

    def hashkey(self):
        return ('FluxesPhotoCal', self.band)

    def __str__(self):
        return 'FluxesPhotoCal(band=%s)' % (self.band)


class MagsPhotoCal(ParamList):
    """Zeropoint calibration of Mags: counts = 10^(0.4 (zp - mag)), 0 beyond
    mag 50 or for a non-finite mag (brightness.py:262-303)."""

    def __init__(self, band, zeropoint):
        self.band = band
        self.maxmag = 50.
        ParamList.__init__(self, zeropoint)

    def copy(self):
        return MagsPhotoCal(self.band, self.zp)

    @staticmethod
    def getNamedParams():
        return dict(zp=0)

    def getStepSizes(self, *args, **kwargs):
        return [0.01]

    def brightnessToCounts(self, brightness):
        mag = brightness.getMag(self.band)
        if not np.isfinite(mag):
            return 0.
        if mag > self.maxmag:
            return 0.
        return 10. ** (0.4 * (self.zp - mag))

    def countsToMag(self, counts):
        return self.zp - 2.5 * np.log10(counts)

    def hashkey(self):
        return ('MagsPhotoCal', self.band, self.zp)

    def __str__(self):
        return 'MagsPhotoCal(band=%s, zp=%.3f)' % (self.band, self.zp)


class NullPhotoCal(BaseParams):
    """Brightness is already in counts (tractor/brightness.py:305-314)."""

    def brightnessToCounts(self, brightness):
        return brightness.getValue()

    def copy(self):
        return NullPhotoCal()

    def hashkey(self):
        return ('NullPhotoCal',)


class LinearPhotoCal(ScalarParam):
    """counts = flux * scale (tractor/brightness.py:316-348)."""

    def __init__(self, scale, band=None):
        super(LinearPhotoCal, self).__init__(scale)
        self.band = band

    def copy(self):
        return self.__class__(self.getValue(), band=self.band)

    def getScale(self):
        return self.val

    def brightnessToCounts(self, brightness):
        if self.band is None:
            return brightness.getValue() * self.val
        return brightness.getFlux(self.band) * self.val


# ---------------------------------------------------------------------------
# Sky
# ---------------------------------------------------------------------------

class NullSky(BaseParams):
    """Zero background (tractor/sky.py:6-12)."""

    def addTo(self, img, scale=1.):
        pass

    def copy(self):
        return NullSky()

    def hashkey(self):
        return ('NullSky',)

    def shifted(self, x0, y0):
        return self.copy()


class ConstantSky(ScalarParam):
    """Constant background level (tractor/sky.py:15-60)."""

    def getParamDerivatives(self, tractor, img, srcs):
        p = Patch(0, 0, np.ones_like(img.getImage()))
        p.setName('dsky')
        return [p]

    def addTo(self, img, scale=1.):
        if self.val == 0:
            return
        img += (self.val * scale)

    def getParamNames(self):
        return ['sky']

    def getConstant(self):
        return self.val

    def subtract(self, con):
        self.val -= con

    def scale(self, s):
        """Scales the sky level by s."""
        self.val *= s

    def shifted(self, x0, y0):
        return self.copy()


# ---------------------------------------------------------------------------
# Image
# ---------------------------------------------------------------------------

class Image(MultiParams):
    """An image with inverse error, PSF, WCS, photometric calibration and sky
    (tractor/image.py:6-272).  The model for an Image can be computed on the
    GPU; the pixel arrays stay numpy arrays as in the reference."""

    def __init__(self, data=None, invvar=None, inverr=None, psf=None, wcs=None, sky=None,
                 photocal=None, name=None, time=None, **kwargs):
        self.data = data
        if inverr is not None:
            self.inverr = inverr
        elif invvar is not None:
            self.setInvvar(invvar)
        self.name = name
        self.zr = kwargs.pop('zr', None)
        self.time = time
        if wcs is None:
            wcs = NullWCS()
        if sky is None:
            sky = NullSky()
        if photocal is None:
            photocal = NullPhotoCal()
        self.modelMinval = 0.
        super(Image, self).__init__(psf, wcs, photocal, sky)

    @staticmethod
    def getNamedParams():
        return dict(psf=0, wcs=1, photocal=2, sky=3)

    def __str__(self):
        return 'Image ' + str(self.name)

    def copy(self):
        return self.__class__(data=self.data.copy(), inverr=self.inverr.copy(),
                              wcs=self.wcs.copy(), psf=self.psf.copy(), sky=self.sky.copy(),
                              photocal=self.photocal.copy(), name=self.name, time=self.time)

    def subimage(self, x0, x1, y0, y1):
        """The image of pixels [x0, x1) x [y0, y1) (image.py:82-92): pixels
        copied, WCS / PSF / sky shifted to the subimage's origin."""
        slc = (slice(y0, y1), slice(x0, x1))
        subtim = Image(data=self.data[slc].copy(), inverr=self.inverr[slc].copy(),
                       wcs=self.wcs.shifted(x0, y0), psf=self.psf.getShifted(x0, y0),
                       sky=self.sky.shifted(x0, y0), photocal=self.photocal.copy())
        subtim.name = self.name
        subtim.time = self.time
        return subtim

    def getTime(self):
        return self.time

    def getParamDerivatives(self, tractor, srcs):
        derivs = []
        for s in self._getActiveSubs():
            if hasattr(s, 'getParamDerivatives'):
                sd = s.getParamDerivatives(tractor, self, srcs)
                assert len(sd) == s.numberOfParams()
                derivs.extend(sd)
            else:
                derivs.extend([False] * s.numberOfParams())
        return derivs

    @property
    def shape(self):
        return self.getShape()

    @property
    def invvar(self):
        return self.inverr ** 2

    def getShape(self):
        return self.data.shape

    def getModelShape(self):
        return self.getShape()

    def getWidth(self):
        return self.getShape()[1]

    def getHeight(self):
        return self.getShape()[0]

    def numberOfPixels(self):
        H, W = self.data.shape
        return W * H

    def hashkey(self):
        return ('Image', id(self.data), id(self.inverr), self.psf.hashkey(), self.sky.hashkey(),
                self.wcs.hashkey(), self.photocal.hashkey())

    def getInvError(self):
        return self.inverr

    def setInvError(self, inverr):
        self.inverr = inverr

    def getInvvar(self):
        return self.inverr ** 2

    def setInvvar(self, iv):
        with np.errstate(invalid='ignore'):
            self.inverr = np.sqrt(iv)

    def getImage(self):
        return self.data

    def setImage(self, img):
        self.data = img

    def getPsf(self):
        return self.psf

    def setPsf(self, psf):
        self.psf = psf

    def getWcs(self):
        return self.wcs

    def getPhotoCal(self):
        return self.photocal

    def getSky(self):
        return self.sky

    def setSky(self, sky):
        self.sky = sky

    # -- FITS (image.py:186-256) ---------------------------------------------
    def getFitsHeader(self, header=None, prefix=''):
        """image.py:224-256: the calibration classes' names under PSF, WCS,
        SKY, PHO and each one's parameters under its prefix (its own
        toFitsHeader, or ImageCalibration.toFitsHeader's P0, P1, ... cards,
        ducks.py:162-168).  `header`: a fitsbin.FITSHDR (or any object with
        add_record)."""
        from .fitsbin import FITSHDR
        hdr = FITSHDR() if header is None else header
        parts = (('PSF', self.getPsf(), 'PSF class'), ('WCS', self.getWcs(), 'WCS class'),
                 ('SKY', self.getSky(), 'Sky class'), ('PHO', self.getPhotoCal(), 'PhotoCal class'))
        for key, obj, comment in parts:
            tt = type(obj)
            hdr.add_record(dict(name=prefix + key, value='%s.%s' % (tt.__module__, tt.__name__),
                                comment=comment))
        for key, obj, _ in parts:
            calibration_to_fits_header(obj, hdr, prefix + key + '_')
        return hdr

    def toFits(self, fits, prefix='', primheader=None, imageheader=None, invvarheader=None):
        """image.py:218-222: the header in an empty primary HDU, then the
        image and the inverse variance.  `fits`: a fitsbin.FITS (or any object
        with fitsio.FITS's write(data, header=...))."""
        hdr = self.getFitsHeader(header=primheader, prefix=prefix)
        fits.write(None, header=hdr)
        fits.write(self.getImage(), header=imageheader)
        fits.write(self.getInvvar(), header=invvarheader)

    @staticmethod
    def readFromFits(fits, prefix=''):
        """image.py:186-216: pixels and inverse variance from HDUs 1 and 2,
        each calibration rebuilt by its class's fromFitsHeader."""
        hdr = fits[0].read_header()
        pix = fits[1].read()
        iv = fits[2].read()
        assert pix.shape == iv.shape

        def read_object(key):
            clazz = _class_from_name(hdr[key])
            return clazz.fromFitsHeader(hdr, prefix=key + '_')
        return Image(data=pix, invvar=iv, psf=read_object(prefix + 'PSF'),
                     wcs=read_object(prefix + 'WCS'), sky=read_object(prefix + 'SKY'),
                     photocal=read_object(prefix + 'PHO'))


def calibration_to_fits_header(obj, hdr, prefix=''):
    """An image calibration's toFitsHeader, or ducks.py:163-168's default:
    one card P<i> per parameter, the parameter's name as the comment."""
    own = getattr(obj, 'toFitsHeader', None)
    if own is not None:
        own(hdr, prefix)
        return
    for i, (name, val) in enumerate(zip(obj.getParamNames(), obj.getAllParams())):
        hdr.add_record(dict(name=prefix + 'P%i' % i, value=val, comment=name))


def _class_from_name(name):
    """The class a header names: module.Class, or the class of that name
    exported by tractor_b200 (for headers written by the reference, whose
    modules are tractor.*)."""
    import importlib
    mod, _, cls = str(name).rpartition('.')
    try:
        return getattr(importlib.import_module(mod), cls)
    except (ImportError, AttributeError, ValueError):
        import tractor_b200
        return getattr(tractor_b200, cls)
