"""Sources: point sources and exp / deV / Gaussian / Sersic / fixed-composite
galaxies with the reference Tractor's API and rendering rules
(tractor/pointsource.py, tractor/galaxy.py, tractor/sersic.py), rendered on the
GPU through RenderPlan.

Every public method has the reference's signature and return convention
(Patch objects holding numpy arrays, None where the reference returns None).
The _plan_* methods add a source's renders to a shared plan so that
Tractor-level calls batch all sources into one launch per kernel.
"""
import numpy as np

from . import profiles, render
from .params import MultiParams, ScalarParam
from .patch import Patch, ModelMask, add_patches, get_overlapping_region
from .plan import RenderPlan, Pending, NONE, done
from .profiles import MixtureOfGaussians
from .psf import HybridPSF, plan_mog_grid, plan_mog_masked, mixture_to_patch


def _counts(img, brightness):
    return img.getPhotoCal().brightnessToCounts(brightness)


class BasicSource(object):

    def getPosition(self):
        return self.pos

    def setPosition(self, position):
        self.pos = position


class SingleProfileSource(BasicSource):
    """tractor/pointsource.py:10-60."""

    def getBrightness(self):
        return self.brightness

    def setBrightness(self, brightness):
        self.brightness = brightness

    def getBrightnesses(self):
        return [self.getBrightness()]

    def getUnitFluxModelPatches(self, *args, **kwargs):
        return [self.getUnitFluxModelPatch(*args, **kwargs)]

    def _plan_model_patch(self, plan, img, minsb=None, modelMask=None, **kwargs):
        """getModelPatch (pointsource.py:36-60): unit-flux patch times counts."""
        counts = _counts(img, self.brightness)
        if counts == 0:
            return NONE
        if not np.isfinite(np.float32(counts)):
            return NONE
        if minsb is None:
            minsb = img.modelMinval
        minval = minsb / counts
        up = self._plan_unit_patch(plan, img, minval=minval, modelMask=modelMask, **kwargs)

        def finish():
            u = up.result()
            if u is None:
                return None
            if u.patch is not None:
                assert np.all(np.isfinite(u.patch))
            return u * counts
        return Pending(finish)

    def getModelPatch(self, img, minsb=None, modelMask=None, **kwargs):
        plan = RenderPlan()
        return self._plan_model_patch(plan, img, minsb=minsb, modelMask=modelMask,
                                      **kwargs).result()

    def getUnitFluxModelPatch(self, img, **kwargs):
        plan = RenderPlan()
        return self._plan_unit_patch(plan, img, **kwargs).result()

    def getParamDerivatives(self, img, modelMask=None, **kwargs):
        plan = RenderPlan()
        return [p.result() if p is not None else None
                for p in self._plan_derivatives(plan, img, modelMask=modelMask, **kwargs)]


# ---------------------------------------------------------------------------
# Point sources
# ---------------------------------------------------------------------------

class PointSource(MultiParams, SingleProfileSource):
    """tractor/pointsource.py:63-241."""

    def __init__(self, pos, br):
        super(PointSource, self).__init__(pos, br)
        self.fixedRadius = None
        self.minRadius = None

    @staticmethod
    def getNamedParams():
        return dict(pos=0, brightness=1)

    def copy(self):
        c = super(PointSource, self).copy()
        c.fixedRadius = self.fixedRadius
        c.minRadius = self.minRadius
        return c

    def getSourceType(self):
        return 'PointSource'

    def __str__(self):
        return self.getSourceType() + ' at ' + str(self.pos) + ' with ' + str(self.brightness)

    def __repr__(self):
        return self.getSourceType() + '(' + repr(self.pos) + ', ' + repr(self.brightness) + ')'

    def _getPsf(self, img):
        return img.getPsf()

    def _plan_unit_patch(self, plan, img, minval=0., derivs=False, modelMask=None, px=None,
                         py=None, **kwargs):
        """getUnitFluxModelPatch (pointsource.py:102-125)."""
        if px is None or py is None:
            px, py = img.getWcs().positionToPixel(self.getPosition(), self)
        H, W = img.shape
        psf = self._getPsf(img)
        r = self.fixedRadius
        if r is None:
            r = psf.getRadius()
        if px + r < 0 or px - r > W or py + r < 0 or py - r > H:
            return NONE
        clipExtent = [0, W, 0, H] if modelMask is None else None
        return psf._plan_point_source(plan, px, py, minval=minval, radius=self.fixedRadius,
                                      derivs=derivs, minradius=self.minRadius,
                                      modelMask=modelMask, clipExtent=clipExtent)

    def _plan_derivatives(self, plan, img, fastPosDerivs=True, modelMask=None, **kwargs):
        """getParamDerivatives (pointsource.py:130-241): analytic position
        derivatives when the PSF path provides them, else forward finite
        differences with the position step sizes; brightness columns are the
        unit patch times d(counts)/d(brightness)."""
        pos_frozen = self.isParamFrozen('pos') or (self.pos.numberOfParams() == 0)
        bright_frozen = self.isParamFrozen('brightness')
        photo = img.getPhotoCal()
        counts0 = photo.brightnessToCounts(self.brightness)
        nparams = self.numberOfParams()
        if pos_frozen and not bright_frozen:
            bsteps = self.brightness.getStepSizes(img)
            bvals = self.brightness.getParams()
            allzero = True
            for i, bstep in enumerate(bsteps):
                old = self.brightness.setParam(i, bvals[i] + bstep)
                ci = photo.brightnessToCounts(self.brightness)
                self.brightness.setParam(i, old)
                if ci != counts0:
                    allzero = False
                    break
            if allzero:
                return [None] * nparams
        pos = self.getPosition()
        wcs = img.getWcs()
        minval = img.modelMinval / counts0 if counts0 > 0 else None
        want_d = (not pos_frozen) and fastPosDerivs
        p0 = self._plan_unit_patch(plan, img, minval=minval, derivs=want_d, modelMask=modelMask)
        steps = []
        if not pos_frozen and counts0 != 0:
            psteps = pos.getStepSizes(img)
            pvals = pos.getParams()
            for i, pstep in enumerate(psteps):
                old = pos.setParam(i, pvals[i] + pstep)
                px1 = self._plan_unit_patch(plan, img, minval=minval, modelMask=modelMask)
                pm = None
                if getattr(pos, 'symmetric_derivs', False):
                    pos.setParam(i, pvals[i] - pstep)
                    pm = self._plan_unit_patch(plan, img, minval=minval, modelMask=modelMask)
                pos.setParam(i, old)
                steps.append((pstep, px1, pm))
        cache = {}

        def all_derivs():
            if 'd' in cache:
                return cache['d']
            r = p0.result()
            patchdx = patchdy = None
            if r is None:
                cache['d'] = [None] * nparams
                return cache['d']
            if isinstance(r, tuple):
                patch0, patchdx, patchdy = r
            else:
                patch0 = r
            H, W = img.shape
            if not patch0.overlapsBbox((0, W, 0, H)):
                cache['d'] = [None] * nparams
                return cache['d']
            derivs = []
            if not pos_frozen:
                if patchdx is not None and patchdy is not None:
                    derivs.extend(wcs.pixelDerivsToPositionDerivs(pos, self, counts0, patch0,
                                                                  patchdx, patchdy))
                elif counts0 == 0:
                    derivs.extend([None] * pos.numberOfParams())
                else:
                    for i, (pstep, px1, pm) in enumerate(steps):
                        patchx = px1.result()
                        pdiff = pstep
                        pp0 = patch0
                        if pm is not None:
                            pp0 = pm.result()
                            pdiff = pstep * 2
                        if patchx is None:
                            dx = patch0 * (-1 * counts0 / pstep)
                        else:
                            dx = (patchx - pp0) * (counts0 / pdiff)
                        dx.setName('d(ptsrc)/d(pos%i)' % i)
                        derivs.append(dx)
            if not bright_frozen:
                bsteps = self.brightness.getStepSizes(img)
                bvals = self.brightness.getParams()
                for i, bstep in enumerate(bsteps):
                    old = self.brightness.setParam(i, bvals[i] + bstep)
                    ci = photo.brightnessToCounts(self.brightness)
                    self.brightness.setParam(i, old)
                    if ci == counts0:
                        df = None
                    else:
                        df = patch0 * ((ci - counts0) / bstep)
                        df.setName('d(ptsrc)/d(bright%i)' % i)
                    derivs.append(df)
            cache['d'] = derivs
            return derivs
        return [Pending(lambda k=k: all_derivs()[k]) for k in range(nparams)]


# ---------------------------------------------------------------------------
# Galaxies
# ---------------------------------------------------------------------------

class _NoDifference(Exception):
    """Raised while planning a difference render that one difference item
    cannot stand for (a hybrid PSF splitting the two mixtures' components
    differently between its Fourier and pixel-space parts), before anything
    is added to the plan; the caller renders and subtracts instead."""


class _SteppedProfiles(object):
    """The `diff_of` of a difference render: a galaxy's affine and sheared
    profiles with shape parameter i set to `value`, each computed when the
    render path first asks for it (the shape is stepped for that call and
    restored)."""

    def __init__(self, gal, i, value):
        self.gal, self.i, self.value = gal, i, value
        self.cache = {}

    def _profile(self, method, img, px, py):
        if method not in self.cache:
            old = self.gal.shape.setParam(self.i, self.value)
            try:
                self.cache[method] = getattr(self.gal, method)(img, px, py)
            finally:
                self.gal.shape.setParam(self.i, old)
        return self.cache[method]

    def _getAffineProfile(self, img, px, py):
        return self._profile('_getAffineProfile', img, px, py)

    def _getShearedProfile(self, img, px, py):
        return self._profile('_getShearedProfile', img, px, py)


class Galaxy(MultiParams, SingleProfileSource):
    """Position, brightness, shape (tractor/galaxy.py:92-223)."""

    def __init__(self, *args):
        super(Galaxy, self).__init__(*args)
        self.name = self.getName()
        self.dname = self.getDName()

    @staticmethod
    def getNamedParams():
        return dict(pos=0, brightness=1, shape=2)

    def getName(self):
        return 'Galaxy'

    def getDName(self):
        return 'gal'

    def getSourceType(self):
        return self.name

    def getShape(self):
        return self.shape

    def __str__(self):
        return (self.name + ' at ' + str(self.pos) + ' with ' + str(self.brightness) + ' and ' +
                str(self.shape))

    def __repr__(self):
        return (self.name + '(pos=' + repr(self.pos) + ', brightness=' + repr(self.brightness) +
                ', shape=' + repr(self.shape) + ')')

    def _extra_derivative_renders(self, plan, img, px0, py0, modelMask, minval, counts,
                                  **kwargs):
        return []

    def _plan_derivatives(self, plan, img, modelMask=None, get_patch0=False, **kwargs):
        """Galaxy.getParamDerivatives (galaxy.py:137-223): position from pixel
        central differences of the unit patch, brightness by scaling, shape
        by forward finite differences (one extra render per shape
        parameter, rendered on patch0's extent)."""
        pos0 = self.getPosition()
        wcs = img.getWcs()
        px0, py0 = wcs.positionToPixel(pos0, self)
        counts = _counts(img, self.brightness)
        minsb = img.modelMinval
        minval = minsb / counts if counts > 0 else None
        p0 = self._plan_unit_patch(plan, img, px=px0, py=py0, minval=minval, modelMask=modelMask,
                                   **kwargs)
        nparams = self.numberOfParams()
        # The stepped renders need patch0's extent when there is no mask; the
        # common case (a mask, or an exact grid) is known in advance.
        shape_plans = None
        mm_fixed = modelMask
        if modelMask is not None and (px0 < modelMask.x0 or px0 > modelMask.x1 - 1 or
                                      py0 < modelMask.y0 or py0 > modelMask.y1 - 1):
            # the source lies outside its mask: patch0 may be None (the
            # reference then takes no shape step), so the steps wait for it
            mm_fixed = None
        elif mm_fixed is None and self._extent_known(img, px0, py0, minval):
            ext = self._no_mask_extent(img, px0, py0, minval)
            # (no extent: the source misses the image and patch0 is None)
            if ext is not None:
                mm_fixed = ModelMask.fromExtent(*ext)
        if mm_fixed is not None:
            shape_plans = self._plan_shape_steps(plan, img, px0, py0, minval, mm_fixed, counts,
                                                 patch0_mask=modelMask,
                                                 **kwargs)
        # Extra columns (Sersic index) render with the caller's modelMask.
        extra = self._extra_derivative_renders(plan, img, px0, py0, modelMask, minval, counts,
                                               **kwargs)
        cache = {}

        def all_derivs():
            if 'd' in cache:
                return cache['d']
            patch0 = p0.result()
            derivs = []
            if get_patch0:
                derivs.append(patch0)
            if patch0 is None:
                derivs.extend([None] * nparams)
                cache['d'] = derivs
                return derivs
            mm = modelMask
            sp = shape_plans
            ex = extra
            if mm is None:
                x0, x1, y0, y1 = patch0.getExtent()
                mm = ModelMask.fromExtent(x0, x1, y0, y1)
            if sp is None:
                sub = RenderPlan()
                sp = self._plan_shape_steps(sub, img, px0, py0, minval, mm, counts,
                                            patch0_mask=modelMask, **kwargs)
            if self.isParamThawed('pos') and self.pos.numberOfParams() > 0:
                if counts == 0:
                    derivs.extend([None] * len(pos0.getParams()))
                else:
                    p = patch0.patch
                    dx = np.zeros_like(p)
                    dx[1:-1, 1:-1] = (p[1:-1, :-2] - p[1:-1, 2:]) / 2.
                    dy = np.zeros_like(p)
                    dy[1:-1, 1:-1] = (p[:-2, 1:-1] - p[2:, 1:-1]) / 2.
                    derivs.extend(wcs.pixelDerivsToPositionDerivs(
                        pos0, self, counts, patch0, Patch(patch0.x0, patch0.y0, dx),
                        Patch(patch0.x0, patch0.y0, dy)))
            if not self.isParamFrozen('brightness'):
                bsteps = self.brightness.getStepSizes()
                params = self.brightness.getParams()
                for i, bstep in enumerate(bsteps):
                    old = self.brightness.setParam(i, params[i] + bstep)
                    ci = _counts(img, self.brightness)
                    self.brightness.setParam(i, old)
                    if ci == counts:
                        df = None
                    else:
                        df = patch0 * ((ci - counts) / bstep)
                        df.setName('d(%s)/d(bright%i)' % (self.dname, i))
                    derivs.append(df)
            if not self.isParamFrozen('shape'):
                gnames = self.shape.getParamNames()
                if counts == 0:
                    derivs.extend([None] * len(self.shape.getParams()))
                else:
                    for i, (gstep, pend, is_diff) in enumerate(sp):
                        patchx = pend.result()
                        if patchx is None:
                            derivs.append(None)
                            continue
                        if is_diff:
                            d = patchx * (counts / gstep)
                        else:
                            d = (patchx - patch0) * (counts / gstep)
                        d.setName('d(%s)/d(%s)' % (self.dname, gnames[i]))
                        derivs.append(d)
            derivs.extend(self._finish_extra(ex, patch0, counts) if ex is not None else [])
            cache['d'] = derivs
            return derivs
        n_out = nparams + (1 if get_patch0 else 0)
        return [Pending(lambda k=k: all_derivs()[k]) for k in range(n_out)]

    def _finish_extra(self, extra, patch0, counts):
        return []

    def _plan_shape_steps(self, plan, img, px0, py0, minval, mm, counts, patch0_mask=None,
                          **kwargs):
        """The forward-difference shape renders (galaxy.py:196-222), on
        patch0's rectangle `mm`.  Returns (step, pending, is_difference) per
        shape parameter.  Without a minval cut or a hybrid PSF the stepped
        and the unstepped mixtures render the same rectangle with as many
        components and the same means, so the difference patchx - patch0 is
        rendered directly as difference items (as the Sersic-index column):
        its float32 error is then relative to the difference, not to the two
        patches, which matters where a shape step barely changes the model
        (a galaxy much smaller than a pixel).  Otherwise patchx is rendered
        and patch0 subtracted, as the reference does."""
        if self.isParamFrozen('shape') or counts == 0:
            return []
        gsteps = self.shape.getStepSizes()
        oldvals = self.shape.getParams()
        # One difference item stands for patchx - patch0 only when both are
        # rendered the same way: on the Fourier path a source outside `mm`
        # is rendered in pixel space (hybrid PSF, galaxy.py:354-372), so
        # unless patch0 had that same mask its render took the other path.
        psf = img.getPsf()
        pure_mog = hasattr(psf, 'getMixtureOfGaussians') and not isinstance(psf, HybridPSF)
        outside = mm is not None and (px0 < mm.x0 or px0 > mm.x1 - 1 or
                                      py0 < mm.y0 or py0 > mm.y1 - 1)
        diff_ok = (mm is not None and minval in (0., None) and
                   (pure_mog or not outside or mm is patch0_mask))
        out = []
        for i, gstep in enumerate(gsteps):
            if diff_ok:
                stepped = _SteppedProfiles(self, i, oldvals[i] + gstep)
                try:
                    p = self._plan_unit_patch(plan, img, px=px0, py=py0, minval=minval,
                                              modelMask=mm, force_sourceOut=True,
                                              diff_of=stepped, **kwargs)
                    out.append((gstep, p, True))
                    continue
                except _NoDifference:
                    pass
            old = self.shape.setParam(i, oldvals[i] + gstep)
            p = self._plan_unit_patch(plan, img, px=px0, py=py0, minval=minval,
                                      modelMask=mm, force_sourceOut=True, **kwargs)
            self.shape.setParam(i, old)
            out.append((gstep, p, False))
        return out

    def _extent_known(self, img, px, py, minval):
        return False

    def _no_mask_extent(self, img, px, py, minval):
        raise NotImplementedError


class ProfileGalaxy(object):
    """Rendering of a mixture-of-Gaussians profile (galaxy.py:226-519)."""

    def getProfile(self):
        return None

    def _getAffineProfile(self, img, px, py):
        return None

    def _getShearedProfile(self, img, px, py):
        return None

    def _getUnitFluxPatchSize(self, img, **kwargs):
        return 0

    def _extent_known(self, img, px, py, minval):
        psf = img.getPsf()
        return (minval == 0. or minval is None) and hasattr(psf, 'getMixtureOfGaussians') and \
            not isinstance(psf, HybridPSF)

    def _no_mask_extent(self, img, px, py, minval):
        halfsize = self._getUnitFluxPatchSize(img, px=px, py=py, minval=minval)
        H, W = img.shape
        outx, inx = get_overlapping_region(int(np.floor(px - halfsize)),
                                           int(np.ceil(px + halfsize + 1)), 0, W - 1)
        outy, iny = get_overlapping_region(int(np.floor(py - halfsize)),
                                           int(np.ceil(py + halfsize + 1)), 0, H - 1)
        if inx == [] or iny == []:
            return None
        return outx.start, outx.stop, outy.start, outy.stop

    def getUnitFluxModelPatch(self, img, px=None, py=None, minval=0.0, modelMask=None, **kwargs):
        plan = RenderPlan()
        return self._plan_unit_patch(plan, img, px=px, py=py, minval=minval,
                                     modelMask=modelMask, **kwargs).result()

    def _plan_unit_patch(self, plan, img, px=None, py=None, minval=0.0, modelMask=None,
                         **kwargs):
        if px is None or py is None:
            px, py = img.getWcs().positionToPixel(self.getPosition(), self)
        p = self._plan_real_unit_patch(plan, img, px, py, minval, modelMask=modelMask, **kwargs)
        if modelMask is None:
            return p

        def check():
            r = p.result()
            if r is not None:
                assert r.shape == modelMask.shape
            return r
        return Pending(check)

    def _plan_real_unit_patch(self, plan, img, px, py, minval, modelMask=None,
                              inner_real_nsigma=3., outer_real_nsigma=4., force_halfsize=None,
                              force_sourceOut=False, diff_of=None, **kwargs):
        """ProfileGalaxy._realGetUnitFluxModelPatch (galaxy.py:266-519).

        diff_of: another galaxy with a profile of as many components (and the
        same geometry): the planned Patch is then its unit-flux patch minus
        this one's, rendered as difference items (the caller checks that the
        two renders share their extent; see _difference_render_ok)."""
        if modelMask is not None:
            x0, y0 = modelMask.x0, modelMask.y0
        else:
            ext = self._no_mask_extent(img, px, py, minval)
            if ext is None:
                return NONE
            x0, x1, y0, y1 = ext
        psf = img.getPsf()
        hybrid = isinstance(psf, HybridPSF)

        def run_mog(amix=None, mm=None, damix=None):
            if amix is None:
                amix = self._getAffineProfile(img, px, py)
            if mm is None:
                mm = modelMask
            psfmix = psf.getMixtureOfGaussians(px=px, py=py)
            cmix = amix.convolve(psfmix)
            dmix = None
            if diff_of is not None:
                if damix is None:
                    damix = diff_of._getAffineProfile(img, px, py)
                dmix = damix.convolve(psfmix)
            if mm is None:
                if dmix is not None:
                    return plan_mog_grid(plan, cmix, x0, x1, y0, y1, 0., 0., diff=dmix)
                return mixture_to_patch(plan, cmix, x0, x1, y0, y1, minval)
            if mm.mask is not None:
                return plan_mog_masked(plan, cmix, mm.x0, mm.y0, mm.mask, 0., 0., diff=dmix)
            return plan_mog_grid(plan, cmix, mm.x0, mm.x1, mm.y0, mm.y1, 0., 0., diff=dmix)

        if hasattr(psf, 'getMixtureOfGaussians') and not hybrid:
            return run_mog(mm=modelMask)

        # Fourier path
        if modelMask is not None:
            mh, mw = modelMask.shape
            x1 = x0 + mw
            y1 = y0 + mh
            halfsize = max(mh / 2., mw / 2.)
            halfsize = max(halfsize, max(max(1 + px - x0, 1 + x1 - px),
                                         max(1 + py - y0, 1 + y1 - py)))
            psfh, psfw = psf.shape
            halfsize = max(halfsize, max(psfw / 2., psfh / 2.))
            if force_halfsize is not None:
                halfsize = force_halfsize
            halfsize = int(np.ceil(halfsize))
            sourceOut = (px < x0 or px > x1 - 1 or py < y0 or py > y1 - 1)
            if sourceOut:
                neardx, neardy = 0., 0.
                if px < x0:
                    neardx = x0 - px
                if px > x1:
                    neardx = px - x1
                if py < y0:
                    neardy = y0 - py
                if py > y1:
                    neardy = py - y1
                nearest = np.hypot(neardx, neardy)
                pixscale = img.wcs.pixscale_at((x0 + x1) / 2., (y0 + y1) / 2.)
                if nearest > (self.getRadius() / pixscale) and not force_sourceOut:
                    return NONE
                if hybrid:
                    return run_mog(mm=modelMask)
                raise RuntimeError('sourceOut, not hybrid')
        else:
            halfsize = self._getUnitFluxPatchSize(img, px=px, py=py, minval=minval)
        sz = psf.getFourierTransformSize(halfsize)
        if sz > render.LARGE_FFT_MAX:
            raise NotImplementedError('Fourier-path patch size %d above the supported %d'
                                      % (sz, render.LARGE_FFT_MAX))
        spec_key, spec, cx, cy = psf.fourier_spectrum(px, py, sz)
        pH = pW = sz
        dx = px - cx
        dy = py - cy
        if modelMask is not None:
            ix0, iy0 = x0, y0
            mux = dx - ix0
            muy = dy - iy0
            sx = int(np.round(mux))
            sy = int(np.round(muy))
            mux -= sx
            muy -= sy
        else:
            ix0 = int(np.round(dx))
            iy0 = int(np.round(dy))
            mux = dx - ix0
            muy = dy - iy0
        assert abs(mux) <= 0.5 and abs(muy) <= 0.5
        amix = self._getShearedProfile(img, px, py)
        fftmix = amix
        mogmix = None
        dfft = None     # a difference item's second mixture: (amp, var) of the FFT part
        dmog = None     # and the pixel-space part's (an affine MixtureOfGaussians)
        if diff_of is not None:
            other = diff_of._getShearedProfile(img, px, py)
            dfft = (other.amp, other.var)
        if hybrid and inner_real_nsigma is not None and outer_real_nsigma is not None:
            nsigma1, nsigma2 = inner_real_nsigma, outer_real_nsigma

            def split(mix):
                # components for pixel space (IM) and for the FFT (IF), and
                # their weights across the ramp between the two
                vv = mix.var[:, 0, 0] + mix.var[:, 1, 1]
                IM = ((pW / 2) ** 2 < (nsigma2 ** 2 * vv))
                IF = ((pW / 2) ** 2 > (nsigma1 ** 2 * vv))
                mw_, fw_ = np.ones(int(IM.sum())), np.ones(int(IF.sum()))
                if np.any(IM * IF):
                    ns = (pW / 2) / np.maximum(1e-6, np.sqrt(vv))
                    mw_ = np.minimum(1., (nsigma2 - ns[IM]) / (nsigma2 - nsigma1))
                    fw_ = np.minimum(1., (ns[IF] - nsigma1) / (nsigma2 - nsigma1))
                return IM, IF, np.any(IM * IF), mw_, fw_
            IM, IF, ramp, mogweights, fftweights = split(amix)
            if diff_of is not None:
                if len(other.amp) != len(amix.amp):
                    raise _NoDifference()
                IM2, IF2, ramp2, mw2, fw2 = split(other)
                if not (np.array_equal(IM, IM2) and np.array_equal(IF, IF2)):
                    raise _NoDifference()
                dfft = (other.amp[IF] * fw2 if ramp2 else other.amp[IF], other.var[IF])
                if np.any(IM):
                    dmog = MixtureOfGaussians(other.amp[IM] * mw2 if ramp2 else other.amp[IM],
                                              amix.mean[IM, :] + np.array([px, py]),
                                              other.var[IM], quick=True)
            if np.any(IM):
                amps = amix.amp[IM]
                if ramp:
                    amps = amps * mogweights
                mogmix = MixtureOfGaussians(amps, amix.mean[IM, :] + np.array([px, py]),
                                            amix.var[IM, :, :], quick=True)
            if np.any(IF):
                amps = amix.amp[IF]
                if ramp:
                    amps = amps * fftweights
                fftmix = MixtureOfGaussians(amps, amix.mean[IF, :], amix.var[IF, :, :], quick=True)
            else:
                fftmix = None
        # output rectangle and the shift of G into it
        if modelMask is not None:
            rx0, ry0, rw, rh = x0, y0, mw, mh
            ssx, ssy = sx, sy
        else:
            # G placed at (ix0, iy0), clipped to [x0, x1) x [y0, y1)
            gx0, gy0 = max(ix0, x0), max(iy0, y0)
            gx1, gy1 = min(ix0 + pW, x1), min(iy0 + pH, y1)
            rx0, ry0, rw, rh = gx0, gy0, max(0, gx1 - gx0), max(0, gy1 - gy0)
            ssx, ssy = ix0 - rx0, iy0 - ry0
        if fftmix is not None and rw > 0 and rh > 0:
            h = plan.add_fft(fftmix.amp, fftmix.var, sz, spec_key, spec, rw, rh, ssx, ssy,
                             mux, muy, diff=dfft)
        else:
            h = ('empty', rh, rw)
        mogp = None
        if mogmix is not None:
            mogp = run_mog(amix=mogmix, mm=modelMask if modelMask is not None else
                           ModelMask(rx0, ry0, rw, rh), damix=dmog)

        def finish():
            G = np.array(plan.get(h), np.float32)
            if mogp is not None:
                mp_ = mogp.result()
                assert mp_.patch.shape == G.shape
                G += mp_.patch
            return Patch(rx0, ry0, G)
        return Pending(finish)


class HoggGalaxy(ProfileGalaxy, Galaxy):
    """tractor/galaxy.py:640-723."""

    def getName(self):
        return 'HoggGalaxy'

    def getRadius(self):
        return self.nre * self.shape.re

    def _tinv(self, img, px, py):
        cdinv = img.getWcs().cdInverseAtPixel(px, py)
        return np.dot(cdinv, self.shape.getRaDecBasis())

    def _getAffineProfile(self, img, px, py):
        return self.getProfile().apply_affine(np.array([px, py]), self._tinv(img, px, py))

    def _getShearedProfile(self, img, px, py):
        return self.getProfile().apply_shear(self._tinv(img, px, py))

    def _getUnitFluxPatchSize(self, img, px=0., py=0., minval=0.):
        if hasattr(self, 'halfsize'):
            return self.halfsize
        pixscale = img.wcs.pixscale_at(px, py)
        halfsize = max(1., self.getRadius() / pixscale)
        h, w = img.shape
        imsize = max(px, w - 1 - px, py, h - 1 - py) + 1
        halfsize = min(halfsize, imsize)
        halfsize = max(halfsize, img.psf.getRadius())
        return int(np.ceil(halfsize))


class GaussianGalaxy(HoggGalaxy):
    nre = 6.

    def __init__(self, *args, **kwargs):
        self.nre = GaussianGalaxy.nre
        super(GaussianGalaxy, self).__init__(*args, **kwargs)

    def getName(self):
        return 'GaussianGalaxy'

    def getProfile(self):
        return profiles.gaussian_mixture()


class ExpGalaxy(HoggGalaxy):
    nre = 4.

    def __init__(self, *args, **kwargs):
        self.nre = ExpGalaxy.nre
        super(ExpGalaxy, self).__init__(*args, **kwargs)

    @staticmethod
    def getExpProfile():
        return profiles.exp_mixture()

    def getName(self):
        return 'ExpGalaxy'

    def getProfile(self):
        return profiles.exp_mixture()


class DevGalaxy(HoggGalaxy):
    nre = 8.

    def __init__(self, *args, **kwargs):
        self.nre = DevGalaxy.nre
        super(DevGalaxy, self).__init__(*args, **kwargs)

    @staticmethod
    def getDevProfile():
        return profiles.dev_mixture()

    def getName(self):
        return 'DevGalaxy'

    def getProfile(self):
        return profiles.dev_mixture()


class SersicIndex(ScalarParam):
    """tractor/sersic.py:344-360: bounds [0.29, 6.3], step 0.01, max step 0.1."""
    stepsize = 0.01

    def __init__(self, val=0):
        super(SersicIndex, self).__init__(val=val)
        self.lower = 0.29
        self.upper = 6.3
        self.maxstep = 0.1

    def isLegal(self):
        return self.lower <= self.val <= self.upper

    def getLogPrior(self):
        return 0. if self.isLegal() else -np.inf


class SersicGalaxy(HoggGalaxy):
    """tractor/sersic.py:362-485."""
    nre = 8.

    @staticmethod
    def getNamedParams():
        return dict(pos=0, brightness=1, shape=2, sersicindex=3)

    def __init__(self, pos, brightness, shape, sersicindex, **kwargs):
        self.nre = SersicGalaxy.nre
        super(SersicGalaxy, self).__init__(pos, brightness, shape, sersicindex)

    def __str__(self):
        return super(SersicGalaxy, self).__str__() + ', Sersic index %.3f' % self.sersicindex.val

    def getName(self):
        return 'SersicGalaxy'

    def getProfile(self):
        return profiles.sersic_mixture().getProfile(self.sersicindex.val)

    def copy(self):
        return SersicGalaxy(self.pos.copy(), self.brightness.copy(), self.shape.copy(),
                            self.sersicindex.copy())

    def _sersic_step(self):
        """The Sersic-index step of getParamDerivatives (sersic.py:416-444):
        0.01, negated if it would pass the upper bound."""
        step = self.sersicindex.getStepSizes()[0]
        newval = self.sersicindex.getParams()[0] + step
        if newval > self.sersicindex.getUpperBounds()[0]:
            step *= -1.
        return step

    def _extra_derivative_renders(self, plan, img, px0, py0, modelMask, minval, counts,
                                  **kwargs):
        """sersic.py:416-444: the index step rendered with the caller's
        modelMask and the default minval.  Where the stepped render and
        patch0 are exact renders of one rectangle with mixtures of as many
        components, the difference newpatch - patch0 is rendered directly
        (difference items: its float32 error is relative to the difference,
        not to the two patches); otherwise newpatch is rendered and
        patch0 subtracted, as the reference does."""
        if self.isParamFrozen('sersicindex'):
            return []
        step = self._sersic_step()
        old = self.sersicindex.getParams()[0]
        other = self.copy()
        other.sersicindex.setParam(0, old + step)
        if self._difference_render_ok(img, other, px0, py0, modelMask, minval):
            try:
                p = self._plan_unit_patch(plan, img, px=px0, py=py0, modelMask=modelMask,
                                          diff_of=other, **kwargs)
                return [(step, p, True)]
            except _NoDifference:
                pass
        self.sersicindex.setParam(0, old + step)
        p = self._plan_unit_patch(plan, img, px=px0, py=py0, modelMask=modelMask, **kwargs)
        self.sersicindex.setParam(0, old)
        return [(step, p, False)]

    def _difference_render_ok(self, img, other, px, py, modelMask, minval):
        """True when patch0 (minval) and other's default-minval render are
        exact renders of the same rectangle by mixtures of equal size: no
        minval cut, equal component counts and, without a mask, equal patch
        extents (a hybrid PSF that splits the two mixtures differently is
        found while planning: _NoDifference)."""
        if minval not in (0., None):
            return False
        if len(self.getProfile().amp) != len(other.getProfile().amp):
            return False
        if modelMask is None:
            if self._no_mask_extent(img, px, py, 0.) != other._no_mask_extent(img, px, py, 0.):
                return False
            if self._getUnitFluxPatchSize(img, px=px, py=py, minval=0.) != \
                    other._getUnitFluxPatchSize(img, px=px, py=py, minval=0.):
                return False
        return True

    def _finish_extra(self, extra, patch0, counts):
        out = []
        for step, p, is_diff in extra:
            newpatch = p.result()
            if newpatch is None:
                out.append(None)
                continue
            if is_diff:
                d = newpatch * (counts / step)
                d.setName('d(%s)/d(%s)' % (self.dname, 'SersicIndex'))
                out.append(d)
                continue
            d = (newpatch - patch0) * (counts / step)
            d.setName('d(%s)/d(%s)' % (self.dname, 'SersicIndex'))
            out.append(d)
        return out

    def _plan_derivatives(self, plan, img, modelMask=None, **kwargs):
        pend = super(SersicGalaxy, self)._plan_derivatives(plan, img, modelMask=modelMask,
                                                           **kwargs)
        nparams = self.numberOfParams()
        if len(pend) < nparams:
            pend = pend + [NONE] * (nparams - len(pend))
        return pend


class FracDev(ScalarParam):
    stepsize = 0.01

    def clipped(self):
        return np.clip(self.getValue(), 0., 1.)

    def derivative(self):
        return 1.


class SoftenedFracDev(FracDev):
    """Sigmoid-softened deV fraction (tractor/galaxy.py:785-801)."""

    def clipped(self):
        return 1. / (1 + np.exp(4. * (0.5 - self.getValue())))

    def derivative(self):
        ef = np.exp(-4. * self.getValue() + 2)
        return 4. * ef / ((ef + 1) ** 2)


class CompositeGalaxy(MultiParams, BasicSource):
    """Exp and deV components sharing a position, each with its own
    brightness and shape (tractor/galaxy.py:1032-1160): rendered as an
    ExpGalaxy plus a DevGalaxy in the same plan."""

    def __init__(self, pos, brightnessExp, shapeExp, brightnessDev, shapeDev):
        MultiParams.__init__(self, pos, brightnessExp, shapeExp, brightnessDev, shapeDev)
        self.name = self.getName()

    @staticmethod
    def getNamedParams():
        return dict(pos=0, brightnessExp=1, shapeExp=2, brightnessDev=3, shapeDev=4)

    def getName(self):
        return 'CompositeGalaxy'

    def __str__(self):
        return (self.name + ' at ' + str(self.pos) + ' with Exp ' + str(self.brightnessExp) +
                ' ' + str(self.shapeExp) + ' and deV ' + str(self.brightnessDev) + ' ' +
                str(self.shapeDev))

    def getBrightness(self):
        return self.brightnessExp + self.brightnessDev

    def getBrightnesses(self):
        return [self.brightnessExp, self.brightnessDev]

    def _parts(self):
        e = ExpGalaxy(self.pos, self.brightnessExp, self.shapeExp)
        d = DevGalaxy(self.pos, self.brightnessDev, self.shapeDev)
        if hasattr(self, 'halfsize'):
            e.halfsize = d.halfsize = self.halfsize
        return e, d

    def _plan_model_patch(self, plan, img, minsb=0., modelMask=None, **kwargs):
        e, d = self._parts()
        kw = dict(kwargs)
        if minsb:
            kw.update(minsb=minsb / 2.)
        pe = e._plan_model_patch(plan, img, modelMask=modelMask, **kw)
        pd = d._plan_model_patch(plan, img, modelMask=modelMask, **kw)
        return Pending(lambda: add_patches(pe.result(), pd.result()))

    def getModelPatch(self, img, minsb=0., modelMask=None, **kwargs):
        plan = RenderPlan()
        return self._plan_model_patch(plan, img, minsb=minsb, modelMask=modelMask,
                                      **kwargs).result()

    def getUnitFluxModelPatches(self, img, minval=0., modelMask=None, **kwargs):
        if minval > 0:
            minval = minval * 0.5   # each component half the error
        e, d = self._parts()
        return (e.getUnitFluxModelPatches(img, minval=minval, modelMask=modelMask, **kwargs) +
                d.getUnitFluxModelPatches(img, minval=minval, modelMask=modelMask, **kwargs))

    def _plan_derivatives(self, plan, img, modelMask=None, **kwargs):
        """galaxy.py:1108-1160: the components' derivatives, the shared
        position's columns summed."""
        e, d = self._parts()
        for frozen, comp, name in (('pos', e, 'pos'), ('pos', d, 'pos'),
                                   ('brightnessExp', e, 'brightness'), ('shapeExp', e, 'shape'),
                                   ('brightnessDev', d, 'brightness'), ('shapeDev', d, 'shape')):
            if self.isParamFrozen(frozen):
                comp.freezeParam(name)
        de = e._plan_derivatives(plan, img, modelMask=modelMask, **kwargs)
        dd = d._plan_derivatives(plan, img, modelMask=modelMask, **kwargs)
        if self.isParamFrozen('pos'):
            return list(de) + list(dd)
        npos = len(self.pos.getStepSizes())

        def pos_sum(i):
            def finish():
                a = de[i].result() if de[i] is not None else None
                b = dd[i].result() if dd[i] is not None else None
                dp = add_patches(a, b)
                if dp is not None:
                    dp.setName('d(comp)/d(pos%i)' % i)
                return dp
            return Pending(finish)
        return [pos_sum(i) for i in range(npos)] + list(de[npos:]) + list(dd[npos:])

    def getParamDerivatives(self, img, modelMask=None, **kwargs):
        plan = RenderPlan()
        return [p.result() if p is not None else None
                for p in self._plan_derivatives(plan, img, modelMask=modelMask, **kwargs)]


class FixedCompositeGalaxy(MultiParams, ProfileGalaxy, SingleProfileSource):
    """deV + exp with a shared position and total brightness and a deV
    fraction (tractor/galaxy.py:798-1029)."""

    def __init__(self, pos, brightness, fracDev, shapeExp, shapeDev):
        if not isinstance(fracDev, ScalarParam):
            fracDev = FracDev(fracDev)
        MultiParams.__init__(self, pos, brightness, fracDev, shapeExp, shapeDev)
        self.name = self.getName()

    def getRadius(self):
        return max(self.shapeExp.re * ExpGalaxy.nre, self.shapeDev.re * DevGalaxy.nre)

    @staticmethod
    def getNamedParams():
        return dict(pos=0, brightness=1, fracDev=2, shapeExp=3, shapeDev=4)

    def getName(self):
        return 'FixedCompositeGalaxy'

    def getSourceType(self):
        return self.name

    def __str__(self):
        return (self.name + ' at ' + str(self.pos) + ' with ' + str(self.brightness) + ', ' +
                str(self.fracDev) + ', exp ' + str(self.shapeExp) + ', deV ' + str(self.shapeDev))

    def _mix(self, img, px, py, affine):
        f = self.fracDev.clipped()
        cdinv = img.getWcs().cdInverseAtPixel(px, py)
        mix = []
        for frac, prof, shape in ((f, profiles.dev_mixture(), self.shapeDev),
                                  (1. - f, profiles.exp_mixture(), self.shapeExp)):
            if (prof is profiles.dev_mixture() and f > 0.) or \
                    (prof is profiles.exp_mixture() and f < 1.):
                T = np.dot(cdinv, shape.getRaDecBasis())
                a = prof.apply_affine(np.array([px, py]), T) if affine else prof.apply_shear(T)
                a.amp = a.amp * frac
                mix.append(a)
        if len(mix) == 1:
            return mix[0]
        return mix[0] + mix[1]

    def _getAffineProfile(self, img, px, py):
        return self._mix(img, px, py, True)

    def _getShearedProfile(self, img, px, py):
        return self._mix(img, px, py, False)

    def _getUnitFluxPatchSize(self, img, px=0., py=0., minval=0.):
        if hasattr(self, 'halfsize'):
            return self.halfsize
        pixscale = img.wcs.pixscale_at(px, py)
        f = self.fracDev.clipped()
        r = 1.
        if f < 1.:
            r = max(r, ExpGalaxy.nre * self.shapeExp.re)
        if f > 0.:
            r = max(r, max(r, DevGalaxy.nre * self.shapeDev.re))
        return r / pixscale + img.psf.getRadius()

    def _plan_derivatives(self, plan, img, modelMask=None, **kwargs):
        """galaxy.py:942-1029: derivatives of exp and deV children, scaled by
        (1 - f) and f, position / brightness columns summed, plus d/dfracDev."""
        e = ExpGalaxy(self.pos, self.brightness, self.shapeExp)
        d = DevGalaxy(self.pos, self.brightness, self.shapeDev)
        e.dname = 'fcomp.exp'
        d.dname = 'fcomp.dev'
        if self.isParamFrozen('pos'):
            e.freezeParam('pos')
            d.freezeParam('pos')
        if self.isParamFrozen('shapeExp'):
            e.freezeParam('shape')
        if self.isParamFrozen('shapeDev'):
            d.freezeParam('shape')
        if hasattr(self, 'halfsize'):
            e.halfsize = self.halfsize
            d.halfsize = self.halfsize
        pe = e._plan_derivatives(plan, img, modelMask=modelMask, **kwargs)
        pd = d._plan_derivatives(plan, img, modelMask=modelMask, **kwargs)
        need_fd = not self.isParamFrozen('fracDev')
        counts = _counts(img, self.brightness)
        ue = ud = None
        if need_fd and counts != 0.:
            ue = e._plan_unit_patch(plan, img, modelMask=modelMask, **kwargs)
            ud = d._plan_unit_patch(plan, img, modelMask=modelMask, **kwargs)
        nparams = self.numberOfParams()
        cache = {}

        def all_derivs():
            if 'd' in cache:
                return cache['d']
            dexp = [p.result() for p in pe]
            ddev = [p.result() for p in pd]
            f = self.fracDev.clipped()
            for x in dexp:
                if x is not None:
                    x *= (1. - f)
            for x in ddev:
                if x is not None:
                    x *= f
            derivs = []
            i0 = 0
            if not self.isParamFrozen('pos'):
                npos = self.pos.numberOfParams()
                for i in range(npos):
                    s = add_patches(dexp[i0 + i], ddev[i0 + i])
                    if s is not None:
                        s.setName('d(fcomp)/d(pos%i)' % i)
                    derivs.append(s)
                i0 += npos
            if not self.isParamFrozen('brightness'):
                nb = self.brightness.numberOfParams()
                for i in range(nb):
                    s = add_patches(dexp[i0 + i], ddev[i0 + i])
                    if s is not None:
                        s.setName('d(fcomp)/d(bright%i)' % i)
                    derivs.append(s)
                i0 += nb
            if not self.isParamFrozen('fracDev'):
                if counts == 0.:
                    derivs.append(None)
                else:
                    uep = ue.result()
                    udp = ud.result()
                    df = self.fracDev.derivative()
                    if uep is not None:
                        uep *= -df
                    if udp is not None:
                        udp *= +df
                    s = add_patches(udp, uep)
                    if s is None:
                        derivs.append(None)
                    else:
                        s *= counts
                        s.setName('d(fcomp)/d(fracDev)')
                        derivs.append(s)
            if not self.isParamFrozen('shapeExp'):
                derivs.extend(dexp[i0:])
            if not self.isParamFrozen('shapeDev'):
                derivs.extend(ddev[i0:])
            cache['d'] = derivs
            return derivs
        return [Pending(lambda k=k: all_derivs()[k]) for k in range(nparams)]
