"""PSF models with the reference's rendering rules (tractor/psf.py), rendered
on the GPU.

GaussianMixturePSF / NCircularGaussianPSF render point sources with the MoG
evaluator (exact grid, masked, or ring-grown approx3 when minval > 0);
PixelizedPSF shifts its stamp with the Lanczos-3 kernel and provides the
spectra for the Fourier galaxy path.
"""
import numpy as np

from . import render
from .params import ParamList, MultiParams
from .plan import RenderPlan, Pending, NONE
from .patch import Patch, get_overlapping_region
from .profiles import MixtureOfGaussians


class HybridPSF(object):
    """Marker class (tractor/psf.py:64-65)."""


def _mog_extent(px, py, rr, clipExtent):
    """get_extent of GaussianMixturePSF.getPointSourcePatch (psf.py:482-494)."""
    x0 = int(np.floor(px - rr))
    x1 = int(np.ceil(px + rr)) + 1
    y0 = int(np.floor(py - rr))
    y1 = int(np.ceil(py + rr)) + 1
    if clipExtent is not None:
        xl, xh, yl, yh = clipExtent
        x0, x1, y0, y1 = max(x0, xl), min(x1, xh), max(y0, yl), min(y1, yh)
    return x0, x1, y0, y1


def plan_mog_grid(plan, mix, x0, x1, y0, y1, fx, fy, diff=None):
    """MixtureOfGaussians.evaluate_grid (mixture_profiles.py:248-263) as a
    pending float64 Patch.  With `diff` (a mixture of the same size and
    means), the Patch is evaluate_grid(diff) - evaluate_grid(mix), rendered
    as one difference item."""
    d = None if diff is None else (diff.amp, diff.var)
    h = plan.add_mog(x0, y0, x1 - x0, y1 - y0, mix.amp, mix.mean, mix.var, fx=fx, fy=fy, diff=d)
    return Pending(lambda: plan.patch(x0, y0, h, np.float64))


def plan_mog_masked(plan, mix, x0, y0, mask, fx, fy, diff=None):
    """MixtureOfGaussians.evaluate_grid_masked (mixture_profiles.py:299-331),
    values only: float32, zero outside the mask, exponent floor -30.  With
    `diff`, the difference of the two mixtures' values as plan_mog_grid."""
    mh, mw = mask.shape
    f32 = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731
    d = None if diff is None else (f32(diff.amp), f32(diff.var))
    h = plan.add_mog(x0, y0, mw, mh, f32(mix.amp), f32(mix.mean), f32(mix.var), fx=fx, fy=fy,
                     floor=render.FLOOR_MASKED, mask=np.asarray(mask, bool), diff=d)
    return Pending(lambda: plan.patch(x0, y0, h, np.float32))


def plan_mog_approx3(plan, mix, x0, x1, y0, y1, fx, fy, minval, minradius=3, doslice=True,
                     maxmargin=100):
    """MixtureOfGaussians.evaluate_grid_approx3 (mixture_profiles.py:333-399).
    The ring-grown evaluated region of c_gauss_2d_approx3 (tractor/approx3.c)
    is computed from the exact grid values on the host side of the plan."""
    cx = int(mix.mean[0, 0] + fx)
    cy = int(mix.mean[0, 1] + fy)
    if cx < x0 - maxmargin or cx > x1 + maxmargin or cy < y0 - maxmargin or cy > y1 + maxmargin:
        return NONE
    from . import approx
    return approx.plan_approx3(plan, mix, x0, x1, y0, y1, fx, fy, minval, cx, cy, minradius,
                               doslice)


def mixture_to_patch(plan, mix, x0, x1, y0, y1, minval=0., exactExtent=False):
    """tractor/mixture_profiles.py:425-438."""
    if minval == 0. or minval is None:
        return plan_mog_grid(plan, mix, x0, x1, y0, y1, 0., 0.)
    return plan_mog_approx3(plan, mix, x0, x1, y0, y1, 0., 0., minval, doslice=not exactExtent)


class MogParams(ParamList):
    """A MixtureOfGaussians as parameters (tractor/utils.py:1298-1370):
    amp[K], then means (x, y) per component, then (vxx, vyy, vxy) per
    component."""

    def __init__(self, *args):
        if len(args) == 3:
            amp, mean, var = args
        else:
            assert len(args) % 6 == 0
            K = len(args) // 6
            amp = np.array(args[:K])
            mean = np.array(args[K:3 * K]).reshape((K, 2))
            rest = args[3 * K:]
            var = np.zeros((K, 2, 2))
            var[:, 0, 0] = rest[::3]
            var[:, 1, 1] = rest[1::3]
            var[:, 0, 1] = var[:, 1, 0] = rest[2::3]
        self.mog = MixtureOfGaussians(amp, mean, var)
        K = self.mog.K
        super(MogParams, self).__init__()
        self._set_param_names(K)
        self.liquid = [True] * self._numberOfThings()
        self.lowers = [None] * self._numberOfThings()
        self.uppers = [None] * self._numberOfThings()
        self.maxstep = [None] * self._numberOfThings()

    def _set_param_names(self, K):
        names = {}
        for k in range(K):
            names['amp%i' % k] = k
            names['meanx%i' % k] = K + 2 * k
            names['meany%i' % k] = K + 2 * k + 1
            names['varxx%i' % k] = 3 * K + 3 * k
            names['varyy%i' % k] = 3 * K + 3 * k + 1
            names['varxy%i' % k] = 3 * K + 3 * k + 2
        self.addNamedParams(**names)

    def _numberOfThings(self):
        return 6 * self.mog.K

    def _getThings(self):
        m = self.mog
        v = np.column_stack([m.var[:, 0, 0], m.var[:, 1, 1], m.var[:, 0, 1]]).ravel()
        return list(m.amp) + list(m.mean.ravel()) + list(v)

    def _getThing(self, i):
        return self._getThings()[i]

    def _setThings(self, vals):
        K = self.mog.K
        self.mog.amp[:] = vals[:K]
        self.mog.mean[:, :] = np.reshape(vals[K:3 * K], (K, 2))
        rest = vals[3 * K:]
        self.mog.var[:, 0, 0] = rest[::3]
        self.mog.var[:, 1, 1] = rest[1::3]
        self.mog.var[:, 0, 1] = self.mog.var[:, 1, 0] = rest[2::3]

    def _setThing(self, i, val):
        v = self._getThings()
        v[i] = val
        self._setThings(v)

    def setParams(self, p):
        v = self._getThings()
        for i, j in self._indexBoth():
            v[j] = p[i]
        self._setThings(v)

    def setAllParams(self, p):
        self._setThings(list(p))

    def getLogPrior(self):
        if np.any((self.mog.var[:, 0, 0] < 0.) | (self.mog.var[:, 1, 1] < 0.)):
            return -np.inf
        return 0.

    def copy(self):
        return self.__class__(self.mog.amp.copy(), self.mog.mean.copy(), self.mog.var.copy())


class GaussianMixturePSF(MogParams):
    """General 2-D Gaussian mixture PSF (tractor/psf.py:369-597)."""

    def __init__(self, *args):
        super(GaussianMixturePSF, self).__init__(*args)
        self.radius = 25
        K = self.mog.K
        self.stepsizes = [0.01] * K + [0.01] * (2 * K) + [0.1] * (3 * K)

    def getShifted(self, x0, y0):
        return self

    def constantPsfAt(self, x, y):
        return self

    def mogAt(self, x, y):
        return self

    def hashkey(self):
        return ('GaussianMixturePSF',) + tuple(self.getAllParams())

    def __str__(self):
        return ('GaussianMixturePSF: amps=' + str(tuple(self.mog.amp.ravel())) +
                ', means=' + str(tuple(self.mog.mean.ravel())) +
                ', var=' + str(tuple(self.mog.var.ravel())))

    def getMixtureOfGaussians(self, px=None, py=None):
        return self.mog

    def get_wmuvar(self):
        return (self.mog.amp, self.mog.mean, self.mog.var)

    @classmethod
    def fromFitsHeader(clazz, hdr, prefix=''):
        """The PSF from header cards <prefix>P0, P1, ... holding its
        parameters (psf.py:407-423)."""
        params = []
        for i in range(100):
            k = prefix + 'P%i' % i
            if k not in hdr:
                break
            params.append(hdr.get(k))
        if len(params) == 0 or (len(params) % 6 != 0):
            raise RuntimeError('Failed to create %s from FITS header: expected factor of 6 '
                               'parameters, got %i' % (str(clazz), len(params)))
        K = len(params) // 6
        psf = clazz(np.zeros(K), np.zeros((K, 2)), np.zeros((K, 2, 2)))
        psf.setParams(params)
        return psf

    def applyTo(self, image):
        raise RuntimeError('Not implemented')

    def scaleBy(self, factor):
        """A new mixture with means x factor and variances x factor^2."""
        return GaussianMixturePSF(self.mog.amp, self.mog.mean * factor,
                                  self.mog.var * factor ** 2)

    def shiftBy(self, dx, dy):
        self.mog.mean[:, 0] += dx
        self.mog.mean[:, 1] += dy

    def computeRadius(self):
        """getNSigma() x the largest component's largest standard deviation."""
        meig = max([max(abs(np.linalg.eigvalsh(v))) for v in self.mog.var])
        return self.getNSigma() * np.sqrt(meig)

    def getRadius(self):
        return self.radius

    def getNSigma(self):
        return 5.

    def _plan_point_source(self, plan, px, py, minval=0., radius=None, derivs=False,
                           minradius=None, modelMask=None, clipExtent=None, **kwargs):
        """getPointSourcePatch (tractor/psf.py:458-528)."""
        if modelMask is not None:
            if modelMask.mask is None:
                return plan_mog_grid(plan, self.mog, modelMask.x0, modelMask.x1, modelMask.y0,
                                     modelMask.y1, px, py)
            return plan_mog_masked(plan, self.mog, modelMask.x0, modelMask.y0, modelMask.mask,
                                   px, py)
        if minval is None:
            minval = 0.
        if minval > 0. or minradius is not None:
            if radius is not None:
                rr = radius
            elif self.radius is not None:
                rr = self.radius
            else:
                r = 0.
                for v in self.mog.var:
                    vv = v[0, 0] + v[1, 1]
                    norm = 2. * np.pi * np.linalg.det(v)
                    r2 = vv * -2. * np.log(minval * norm)
                    if r2 > 0:
                        r = max(r, np.sqrt(r2))
                rr = int(np.ceil(r))
            x0, x1, y0, y1 = _mog_extent(px, py, rr, clipExtent)
            if x0 >= x1 or y0 >= y1:
                return NONE
            kw = {}
            if minradius is not None:
                kw['minradius'] = minradius
            return plan_mog_approx3(plan, self.mog, x0, x1, y0, y1, px, py, minval, **kw)
        r = self.getRadius() if radius is None else radius
        x0, x1, y0, y1 = _mog_extent(px, py, r, clipExtent)
        if x0 >= x1 or y0 >= y1:
            return NONE
        return plan_mog_grid(plan, self.mog, x0, x1, y0, y1, px, py)

    def getPointSourcePatch(self, px, py, **kwargs):
        plan = RenderPlan()
        p = self._plan_point_source(plan, px, py, **kwargs)
        return p.result()

    @staticmethod
    def _stamp_for_em(stamp):
        # fromStamp's preprocessing, in the stamp's own dtype (psf.py:590-591)
        stamp = np.array(stamp, copy=True)
        stamp /= stamp.sum()
        return np.maximum(stamp, 0)

    @staticmethod
    def fromStamp(stamp, N=3, P0=None, xy0=None, alpha=0., emsteps=1000, v2=False,
                  approx=1e-30, v3=False):
        """GaussianMixturePSF.fromStamp (tractor/psf.py:536-597): an N-component
        mixture fit to a PSF stamp by EM on the GPU (em_fit_2d_reg), with v2
        by EM with a flat sky term (em_fit_2d_reg2; returns (psf, skyamp)), or
        with v3 by the Tractor optimiser with the PSF's parameters thawed."""
        from .emfit import em_init_params, em_fit_2d_reg
        if P0 is not None:
            w, mu, var = P0
        else:
            w, mu, var = em_init_params(N, None, None, None)
        stamp = stamp.copy()
        if xy0 is None:
            xm, ym = -(stamp.shape[1] // 2), -(stamp.shape[0] // 2)
        else:
            xm, ym = xy0
        if v3:
            from .basics import Image, PixPos, Flux
            from .engine import Tractor
            from .sources import PointSource
            tpsf = GaussianMixturePSF(w, mu, var)
            tim = Image(data=stamp, invvar=1e6 * np.ones_like(stamp), psf=tpsf)
            h, ww = tim.shape
            src = PointSource(PixPos(ww // 2, h // 2), Flux(1.))
            tr = Tractor([tim], [src])
            tr.freezeParam('catalog')
            tim.freezeAllBut('psf')
            tim.modelMinval = approx
            for step in range(20):
                dlnp, X, alpha = tr.optimize(shared_params=False)
                if dlnp < 1e-6:
                    break
            return tpsf
        if v2:
            # the EM fit with a flat sky term on the stamp as given: returns
            # (psf, sky level per pixel), as the reference does
            from .emfit import em_fit_2d_reg2
            w = np.array(w, np.float64)
            mu = np.array(mu, np.float64)
            var = np.array(var, np.float64)
            ok, skyamp = em_fit_2d_reg2(stamp, xm, ym, w, mu, var, alpha, emsteps, approx)
            return GaussianMixturePSF(w, mu, var), skyamp
        stamp = GaussianMixturePSF._stamp_for_em(stamp)
        w = np.array(w, np.float64)
        mu = np.array(mu, np.float64)
        var = np.array(var, np.float64)
        em_fit_2d_reg(stamp, xm, ym, w, mu, var, alpha, emsteps)
        return GaussianMixturePSF(w, mu, var)

    @staticmethod
    def fromStamps(stamps, N=3, P0=None, xy0=None, alpha=0., emsteps=1000):
        """fromStamp's EM fit for many stamps of one size at once (one launch;
        P0 and xy0 apply to every stamp).  Returns a list of
        GaussianMixturePSF, None where the fit failed (a non-positive
        covariance determinant: fromStamp's em_fit_2d_reg returns -1 there)."""
        from .emfit import em_init_params, em_fit_2d_batch
        if P0 is not None:
            w, mu, var = P0
        else:
            w, mu, var = em_init_params(N, None, None, None)
        stamps = [GaussianMixturePSF._stamp_for_em(s) for s in stamps]
        if not stamps:
            return []
        ny, nx = stamps[0].shape
        n = len(stamps)
        if xy0 is None:
            xy0 = (-(nx // 2), -(ny // 2))
        a, m, v, st = em_fit_2d_batch(np.stack(stamps),
                                      np.broadcast_to(np.asarray(w, np.float64), (n, len(w))),
                                      np.broadcast_to(np.asarray(mu, np.float64), (n,) + np.shape(mu)),
                                      np.broadcast_to(np.asarray(var, np.float64), (n,) + np.shape(var)),
                                      alpha, emsteps, xy0=xy0)
        return [None if st[i] else GaussianMixturePSF(a[i], m[i], v[i]) for i in range(n)]


class GaussianMixtureEllipsePSF(GaussianMixturePSF):
    """A GaussianMixturePSF whose covariances are EllipseESoft shapes
    (tractor/psf.py:658-789): parameters amp[K], the means (x, y) per
    component, then (logr, ee1, ee2) per component; rendered as the mixture
    of their covariances."""

    def __init__(self, *args):
        from .ellipses import EllipseESoft
        if len(args) == 3:
            amp, mean, ell = args
        else:
            assert len(args) % 6 == 0
            K = len(args) // 6
            amp = np.array(args[:K])
            mean = np.array(args[K:3 * K]).reshape((K, 2))
            rest = args[3 * K:]
            ell = [EllipseESoft(*rest[3 * k: 3 * (k + 1)]) for k in range(K)]
        K = len(amp)
        var = np.zeros((K, 2, 2))
        for k in range(K):
            var[k] = self.ellipseToVariance(ell[k])
        self.ellipses = [e.copy() for e in ell]
        super(GaussianMixtureEllipsePSF, self).__init__(amp, mean, var)
        self.stepsizes = [0.001] * K + [0.001] * (K * 2) + [0.001] * (K * 3)

    def ellipseToVariance(self, ell):
        return ell.getCovariance()

    def getShifted(self, x0, y0):
        return self

    def _set_param_names(self, K):
        names = {}
        for k in range(K):
            names['amp%i' % k] = k
            names['meanx%i' % k] = K + (k * 2)
            names['meany%i' % k] = K + (k * 2) + 1
            names['logr%i' % k] = K * 3 + (k * 3)
            names['ee1-%i' % k] = K * 3 + (k * 3) + 1
            names['ee2-%i' % k] = K * 3 + (k * 3) + 2
        self.addNamedParams(**names)

    def toMog(self):
        return GaussianMixturePSF(self.mog.amp, self.mog.mean, self.mog.var)

    def mogAt(self, x, y):
        return self.toMog()

    def constantPsfAt(self, x, y):
        return self.mogAt(x, y)

    def hashkey(self):
        return ('GaussianMixtureEllipsePSF',) + tuple(self.getAllParams())

    def copy(self):
        return GaussianMixtureEllipsePSF(self.mog.amp.copy(), self.mog.mean.copy(),
                                         [e.copy() for e in self.ellipses])

    def __str__(self):
        return ('GaussianMixtureEllipsePSF: amps=' +
                '[' + ', '.join(['%.3f' % a for a in self.mog.amp.ravel()]) + ']' +
                ', means=[' + ', '.join(['(%.3f, %.3f)' % (x, y) for x, y in self.mog.mean]) +
                ']' + ', ellipses=' + ', '.join(str(e) for e in self.ellipses) +
                ', var=' + str(tuple(self.mog.var.ravel())))

    def _getThings(self):
        p = list(self.mog.amp) + list(self.mog.mean.ravel())
        for e in self.ellipses:
            p += e.getAllParams()
        return p

    def _setThings(self, p):
        K = self.mog.K
        self.mog.amp = np.atleast_1d(np.asarray(p[:K], np.float64))
        pp = p[K:]
        self.mog.mean = np.atleast_2d(np.asarray(pp[:K * 2], np.float64)).reshape(K, 2)
        pp = pp[K * 2:]
        for i, e in enumerate(self.ellipses):
            e.setAllParams(pp[:3])
            pp = pp[3:]
            self.mog.var[i, :, :] = self.ellipseToVariance(e)

    def _setThing(self, i, p):
        things = self._getThings()
        old = things[i]
        things[i] = p
        self._setThings(things)
        return old

    @staticmethod
    def fromStamp(stamp, N=3, P0=None, approx=1e-6, damp=0.):
        """GaussianMixtureEllipsePSF.fromStamp (tractor/psf.py:757-789): the
        Tractor optimiser, the PSF's parameters thawed, fitting a point
        source at the stamp centre (model images and their forward
        differences rendered on the GPU)."""
        from .basics import Image, PixPos, Flux
        from .ellipses import EllipseESoft
        from .engine import Tractor
        from .sources import PointSource
        w = np.ones(N) / float(N)
        mu = np.zeros((N, 2))
        ell = [EllipseESoft(np.log(2 * r), 0., 0.) for r in range(1, N + 1)]
        psf = GaussianMixtureEllipsePSF(w, mu, ell)
        if P0 is not None:
            psf.setAllParams(P0)
        tim = Image(data=stamp, invvar=1e6 * np.ones_like(stamp), psf=psf)
        H, W = stamp.shape
        src = PointSource(PixPos(W // 2, H // 2), Flux(1.))
        tr = Tractor([tim], [src])
        tr.freezeParam('catalog')
        tim.freezeAllBut('psf')
        tim.modelMinval = approx
        alphas = [0.1, 0.3, 1.0]
        for step in range(50):
            dlnp, X, alpha = tr.optimize(shared_params=False, alphas=alphas, damp=damp)
            if dlnp < 1e-6:
                break
        return psf


def getCircularMog(amps, sigmas):
    """float32 tables as tractor/psf.py:931-944."""
    K = len(amps)
    amp = np.array(amps).astype(np.float32)
    mean = np.zeros((K, 2), np.float32)
    var = np.zeros((K, 2, 2), np.float32)
    for k in range(K):
        var[k, 0, 0] = var[k, 1, 1] = sigmas[k] ** 2
    return MixtureOfGaussians(amp, mean, var, quick=True)


class NCircularGaussianPSF(MultiParams):
    """N concentric circular Gaussians (tractor/psf.py:792-929)."""

    def __init__(self, sigmas, weights):
        assert len(sigmas) == len(weights)
        psig = ParamList(*sigmas)
        psig.stepsizes = [0.01] * len(sigmas)
        pw = ParamList(*weights)
        pw.stepsizes = [0.01] * len(weights)
        super(NCircularGaussianPSF, self).__init__(psig, pw)
        self.minradius = 1.

    @staticmethod
    def getNamedParams():
        return dict(sigmas=0, weights=1)

    def getShifted(self, x0, y0):
        return self

    def constantPsfAt(self, x, y):
        return self

    def scale(self, factor):
        """A new PSF factor times wider (psf.py:860-863)."""
        return NCircularGaussianPSF(np.array(self.mysigmas) * factor, self.myweights)

    @property
    def mysigmas(self):
        return self.sigmas.vals

    @property
    def myweights(self):
        return self.weights.vals

    @property
    def amp(self):
        return self.weights

    @property
    def mog(self):
        return self.getMixtureOfGaussians()

    def __str__(self):
        return ('NCircularGaussianPSF: sigmas [ ' + ', '.join('%.3f' % s for s in self.mysigmas) +
                ' ], weights [ ' + ', '.join('%.3f' % w for w in self.myweights) + ' ]')

    def hashkey(self):
        return ('NCircularGaussianPSF', tuple(self.mysigmas), tuple(self.myweights))

    def copy(self):
        return NCircularGaussianPSF(list(self.mysigmas), list(self.myweights))

    def getMixtureOfGaussians(self, px=None, py=None):
        return getCircularMog(tuple(self.myweights), tuple(self.mysigmas))

    def getNSigma(self):
        return 5.

    def getRadius(self):
        if hasattr(self, 'radius'):
            return self.radius
        return max(self.minradius, max(self.mysigmas) * self.getNSigma())

    def _plan_point_source(self, plan, px, py, minval=0., radius=None, modelMask=None,
                           clipExtent=None, **kwargs):
        """getPointSourcePatch (tractor/psf.py:898-929)."""
        if modelMask is not None:
            x0, x1, y0, y1 = modelMask.extent
        else:
            ix = int(round(px))
            iy = int(round(py))
            rad = int(np.ceil(self.getRadius())) if radius is None else radius
            x0, x1, y0, y1 = ix - rad, ix + rad + 1, iy - rad, iy + rad + 1
        if clipExtent is not None:
            xl, xh, yl, yh = clipExtent
            x0, x1, y0, y1 = max(x0, xl), min(x1, xh), max(y0, yl), min(y1, yh)
        mix = self.getMixtureOfGaussians()
        mix = MixtureOfGaussians(mix.amp, mix.mean + np.array([px, py]), mix.var, quick=True)
        return mixture_to_patch(plan, mix, x0, x1, y0, y1, minval=minval,
                                exactExtent=(modelMask is not None))

    def getPointSourcePatch(self, px, py, **kwargs):
        plan = RenderPlan()
        return self._plan_point_source(plan, px, py, **kwargs).result()


class PixelizedPSF(ParamList):
    """A PSF image shifted to sub-pixel positions with Lanczos-3; galaxies
    are rendered through its Fourier transform (tractor/psf.py:68-367).
    The PSF has no fitted parameters (as in the reference)."""

    def __init__(self, img, sampling=1., Lorder=3):
        super(PixelizedPSF, self).__init__()
        img = np.asarray(img).astype(np.float32)
        H, W = img.shape
        assert (H % 2) == 1 and (W % 2) == 1
        if sampling != 1.:
            raise NotImplementedError('PixelizedPSF sampling != 1 is not supported')
        self.img = img
        self.radius = np.hypot(H / 2., W / 2.)
        self.H, self.W = H, W
        self.Lorder = Lorder
        self.sampling = sampling
        self._key = ('PixelizedPSF', id(self), img.tobytes().__hash__())

    def __str__(self):
        return 'PixelizedPSF'

    @property
    def shape(self):
        return (self.H, self.W)

    def hashkey(self):
        return ('PixelizedPSF', tuple(self.img.ravel()))

    def copy(self):
        return self.__class__(self.img.copy())

    def getShifted(self, x0, y0):
        return self

    def constantPsfAt(self, x, y):
        return self

    def getRadius(self):
        return self.radius

    def getImage(self, px, py):
        return self.img

    _normalized = False

    def getFourierTransformSize(self, radius):
        return 2 ** int(np.ceil(np.log2(radius * 2.)))

    def spectrum(self, sz):
        """(device spectrum, cx, cy) at FFT size sz (getFourierTransform,
        tractor/psf.py:249-280, complex64, NormalizedPsf divides by |P00|)."""
        return render.psf_spectra().get(self._key, self.getImage(0., 0.), sz,
                                        normalize=self._normalized)

    def fourier_spectrum(self, px, py, sz):
        """(spectrum key, device spectrum, cx, cy) at FFT size sz for a source
        at (px, py); the same for every position of a constant PSF."""
        spec, cx, cy = self.spectrum(sz)
        return self._key, spec, cx, cy

    def getFourierTransform(self, px, py, radius):
        """Host copy of the spectrum in the reference's layout:
        (P (sz, sz/2+1) complex64, (cx, cy), (sz, sz), (v, w))."""
        sz = self.getFourierTransformSize(radius)
        _, spec, cx, cy = self.fourier_spectrum(px, py, sz)
        P = spec.cpu().numpy().view(np.complex64).reshape(sz // 2 + 1, sz).T.copy()
        return P, (cx, cy), (sz, sz), (np.fft.rfftfreq(sz), np.fft.fftfreq(sz))

    def _plan_point_source(self, plan, px, py, minval=0., modelMask=None, radius=None,
                           derivs=False, **kwargs):
        """getPointSourcePatch (tractor/psf.py:137-207)."""
        img = self.getImage(px, py)
        if radius is not None:
            R = int(np.ceil(radius))
            H, W = img.shape
            cx, cy = W // 2, H // 2
            img = img[max(cy - R, 0):min(cy + R + 1, H - 1), max(cx - R, 0):min(cx + R + 1, W - 1)]
        H, W = img.shape
        ix = round(float(px))
        iy = round(float(py))
        dx = px - ix
        dy = py - iy
        x0 = ix - W // 2
        y0 = iy - H // 2
        if modelMask is None:
            h = plan.add_lanczos(img, dx, dy)
            return Pending(lambda: plan.patch(x0, y0, h, np.float32))
        mh, mw = modelMask.shape
        mx0, my0 = modelMask.x0, modelMask.y0
        if (mx0 >= x0 + W) or (mx0 + mw <= x0) or (my0 >= y0 + H) or (my0 + mh <= y0):
            return NONE
        L = 3
        mm = np.zeros((mh + 2 * L, mw + 2 * L), np.float32)
        yi, yo = get_overlapping_region(my0 - y0 - L, my0 - y0 + mh - 1 + L, 0, H - 1)
        xi, xo = get_overlapping_region(mx0 - x0 - L, mx0 - x0 + mw - 1 + L, 0, W - 1)
        mm[yo, xo] = img[yi, xi]
        h = plan.add_lanczos(mm, dx, dy)

        def finish():
            a = np.array(plan.get(h)[L:-L, L:-L], np.float32)
            patch = Patch(mx0, my0, a)
            if not derivs:
                return patch
            ddx = np.zeros_like(a)
            ddx[1:-1, 1:-1] = -(a[1:-1, 2:] - a[1:-1, :-2]) / 2.
            ddy = np.zeros_like(a)
            ddy[1:-1, 1:-1] = -(a[2:, 1:-1] - a[:-2, 1:-1]) / 2.
            return patch, Patch(mx0, my0, ddx), Patch(mx0, my0, ddy)
        return Pending(finish)

    def getPointSourcePatch(self, px, py, **kwargs):
        plan = RenderPlan()
        return self._plan_point_source(plan, px, py, **kwargs).result()


class HybridPixelizedPSF(HybridPSF):
    """A PixelizedPSF with a Gaussian-mixture approximation
    (tractor/psf.py:600-655).  Point sources use the pixelized model;
    galaxies take the Fourier path with the pixelized spectrum, except their
    components that are wide for the FFT box, which are rendered in pixel
    space through the mixture `gauss` (with a linear ramp between the two,
    ProfileGalaxy's hybrid split).  Every other attribute is the pixelized
    model's.  Without `gauss`, an N-component GaussianMixturePSF is fit to
    the pixelized model's image at (cx, cy) by GaussianMixturePSF.fromStamp
    (the EM fit, on the GPU), as the reference does."""

    def __init__(self, pix, gauss=None, N=2, cx=0., cy=0.):
        object.__setattr__(self, 'pix', pix)
        if gauss is None:
            gauss = GaussianMixturePSF.fromStamp(pix.getImage(cx, cy), N=N)
        object.__setattr__(self, 'gauss', gauss)

    def __str__(self):
        return ('HybridPixelizedPSF: Gaussian sigma %.2f, Pix %s' %
                (np.sqrt(self.gauss.mog.var[0, 0, 0]), str(self.pix)))

    def copy(self):
        return self.__class__(self.pix.copy(), self.gauss.copy())

    def getMixtureOfGaussians(self, **kwargs):
        return self.gauss.getMixtureOfGaussians(**kwargs)

    def getShifted(self, dx, dy):
        return HybridPixelizedPSF(self.pix.getShifted(dx, dy), self.gauss)

    def constantPsfAt(self, x, y):
        return HybridPixelizedPSF(self.pix.constantPsfAt(x, y), self.gauss)

    def __getattr__(self, name):
        # only called for attributes this object does not have: the
        # pixelized model's (never 'pix' itself, which __init__ sets first)
        if name in ('pix', 'gauss'):
            raise AttributeError(name)
        return getattr(self.__dict__['pix'], name)

    def __setattr__(self, name, val):
        if name in ('gauss', 'pix'):
            return object.__setattr__(self, name, val)
        setattr(self.__dict__['pix'], name, val)

    def __getstate__(self):
        return (self.gauss, self.pix)

    def __setstate__(self, state):
        object.__setattr__(self, 'gauss', state[0])
        object.__setattr__(self, 'pix', state[1])


class NormalizedPixelizedPsf(PixelizedPSF):
    """PixelizedPSF with its image and spectrum normalised to unit sum
    (tractor/psf.py:947-971)."""
    _normalized = True

    def getImage(self, px, py):
        img = self.img.copy()
        n = np.sum(img)
        if n != 0:
            img /= n
        return img

    def __str__(self):
        return 'NormalizedPixelizedPSF'
