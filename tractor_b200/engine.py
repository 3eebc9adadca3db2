"""The Tractor engine (tractor/engine.py:40-497) with GPU-batched rendering.

Tractor.getModelImage / getChiImage / getLogProb / getDerivs keep the
reference's signatures and results; all renders of one call (every source in
every image, every derivative step) go into one RenderPlan, i.e. one launch
per kernel type.  Patches are accumulated into float32 model images in
catalog order, as the reference does (engine.py:424-445).
"""
import numpy as np

from .params import MultiParams
from .patch import Patch
from .plan import RenderPlan


def _isint(i):
    try:
        return int(i) == i
    except Exception:
        return False


class Catalog(MultiParams):
    """A list of sources (engine.py:40-76)."""

    def __str__(self):
        return 'Catalog: %i sources, %i parameters' % (len(self), self.numberOfParams())

    def getThawedSources(self):
        return self._getActiveSubs()

    def getFrozenSources(self):
        return (s for s in self._getFrozenArray(self.subs) if s is not None)

    def getNamedParamName(self, j):
        return 'source%i' % j

    def printLong(self):
        print('Catalog with %i sources:' % len(self))
        for i, x in enumerate(self):
            print('  %i:' % i, x)


class Images(MultiParams):
    """A list of images (engine.py:78-88)."""

    def getNamedParamName(self, j):
        return 'image%i' % j


def _once(fn):
    """fn() evaluated at most once."""
    box = []

    def get():
        if not box:
            box.append(fn())
        return box[0]
    return get


class _FiniteDifference(object):
    """A pending forward-difference column of an image parameter:
    Patch(0, 0, (mod - mod0) / step) (engine.py:318-320)."""

    def __init__(self, fin, fin0, step, name):
        self.fin, self.fin0, self.step, self.name = fin, fin0, step, name

    def result(self):
        deriv = Patch(0, 0, (self.fin() - self.fin0()) / self.step)
        deriv.name = self.name
        return deriv


class Tractor(MultiParams):
    """tractor/engine.py:96-497."""

    @staticmethod
    def getName():
        return 'Tractor'

    @staticmethod
    def getNamedParams():
        return dict(images=0, catalog=1)

    def __init__(self, images=None, catalog=None, optimizer=None, model_kwargs=None):
        if images is None:
            images = []
        if catalog is None:
            catalog = []
        if not isinstance(images, Images):
            images = Images(*images)
        if not isinstance(catalog, Catalog):
            catalog = Catalog(*catalog)
        super(Tractor, self).__init__(images, catalog)
        self.modtype = np.float32
        self.modelMasks = None
        self.expectModelMasks = False
        if optimizer is None:
            from .optimizer import B200Optimizer
            optimizer = B200Optimizer()
        self.optimizer = optimizer
        self.model_kwargs = model_kwargs if model_kwargs is not None else {}

    def __str__(self):
        names = [im.name if im.name is not None else '[unnamed]' for im in self.images]
        return ('%s with %i sources and %i images' % (self.getName(), len(self.catalog),
                                                       len(self.images)) +
                ' (' + ', '.join(names) + ')')

    def __call__(self, X):
        self.setParams(X)
        return self.getLogProb()

    def getNImages(self):
        return len(self.images)

    def getImage(self, i):
        return self.images[i]

    def getImages(self):
        return self.images

    def getCatalog(self):
        return self.catalog

    def setCatalog(self, srcs):
        self.catalog = srcs

    def setImages(self, ims):
        self.images = ims

    def addImage(self, img):
        self.images.append(img)

    def addSource(self, src):
        self.catalog.append(src)

    def addSources(self, srcs):
        self.catalog.extend(srcs)

    def removeSource(self, src):
        self.catalog.remove(src)

    # -- optimisation entry points (engine.py:194-240) --------------------
    def optimize(self, **kwargs):
        kw = dict(self.model_kwargs)
        kw.update(kwargs)
        return self.optimizer.optimize(self, **kw)

    def optimize_loop(self, **kwargs):
        kw = dict(self.model_kwargs)
        kw.update(kwargs)
        return self.optimizer.optimize_loop(self, **kw)

    def optimize_forced_photometry(self, **kwargs):
        kw = dict(self.model_kwargs)
        kw.update(kwargs)
        return self.optimizer.forced_photometry(self, **kw)

    # -- model masks (engine.py:341-376) ----------------------------------
    def setModelMasks(self, masks, assumeMasks=True):
        self.modelMasks = masks
        assert (masks is None) or (len(masks) == len(self.images))
        self.expectModelMasks = (masks is not None) and assumeMasks

    def _getModelMaskFor(self, image, src):
        if self.modelMasks is None:
            return None
        i = self.images.index(image)
        return self.modelMasks[i].get(src, None)

    # -- rendering ----------------------------------------------------------
    def _plan_model_patch(self, plan, img, src, **kwargs):
        mask = self._getModelMaskFor(img, src)
        if self.expectModelMasks and mask is None:
            return None
        kw = dict(self.model_kwargs)
        kw.update(kwargs)
        return src._plan_model_patch(plan, img, modelMask=mask, **kw)

    def getModelPatch(self, img, src, **kwargs):
        plan = RenderPlan()
        p = self._plan_model_patch(plan, img, src, **kwargs)
        return None if p is None else p.result()

    def _plan_model_image(self, plan, img, srcs=None, sky=True, minsb=None, **kwargs):
        if _isint(img):
            img = self.getImage(img)
        if srcs is None:
            srcs = self.catalog
        pend = []
        for src in srcs:
            if src is None:
                continue
            p = self._plan_model_patch(plan, img, src, minsb=minsb, **kwargs)
            if p is not None:
                pend.append(p)
        # the sky as it is now (the plan may run after parameters change)
        mod0 = np.zeros(img.getModelShape(), self.modtype)
        if sky:
            img.getSky().addTo(mod0)

        def finish():
            mod = mod0.copy()
            for p in pend:
                patch = p.result()
                if patch is not None:
                    patch.addTo(mod)
            return mod
        return finish

    # Catalogs at least this large on an eligible image go through the scene
    # renderer (tb_scene_render) instead of per-source patches.
    SCENE_MIN_SOURCES = 64

    def getModelImage(self, img, srcs=None, sky=True, minsb=None, **kwargs):
        """engine.py:424-445: all sources rendered in one batched launch --
        for large catalogs with rectangular model masks on a MoG-PSF image,
        one scene render of the whole image (tb_scene_render); otherwise
        per-source patches batched into one launch per kernel type."""
        if _isint(img):
            img = self.getImage(img)
        if not kwargs:
            mod = self._scene_model(img, self.catalog if srcs is None else srcs, sky, minsb)
            if mod is not None:
                return mod
        plan = RenderPlan()
        return self._plan_model_image(plan, img, srcs=srcs, sky=sky, minsb=minsb, **kwargs)()

    def _scene_records(self, img, srcs, minsb):
        """SCENE_SRC records of `srcs` on `img`, or None when the scene
        renderer does not reproduce getModelImage's per-source path here."""
        from . import _lib, psf as psfmod, sources as S, ellipses as E
        from .basics import NullWCS
        from .patch import ModelMask
        psf = img.getPsf()
        if not hasattr(psf, 'getMixtureOfGaussians') or isinstance(psf, psfmod.HybridPSF):
            return None
        if not isinstance(img.getWcs(), NullWCS) or self.modelMasks is None:
            return None
        if (img.modelMinval if minsb is None else minsb) != 0.:
            return None
        rows = []
        for src in srcs:
            if src is None:
                continue
            mask = self._getModelMaskFor(img, src)
            if mask is None:
                if self.expectModelMasks:
                    continue
                return None
            if not isinstance(mask, ModelMask) or mask.mask is not None:
                return None
            counts = S._counts(img, src.getBrightness()) if hasattr(src, 'getBrightness') else None
            if counts is None or not np.isfinite(np.float32(counts)):
                return None
            if counts == 0:
                continue
            r = np.zeros(1, _lib.SCENE_SRC)[0]
            px, py = img.getWcs().positionToPixel(src.getPosition(), src)
            r['px'], r['py'], r['counts'] = px, py, counts
            r['mx0'], r['my0'], r['mw'], r['mh'] = mask.x0, mask.y0, mask.w, mask.h
            shapes = []
            if isinstance(src, S.PointSource):
                r['profile'] = _lib.PROFILE_POINT
            elif isinstance(src, S.FixedCompositeGalaxy):
                r['profile'] = _lib.PROFILE_COMPOSITE
                r['fdev'] = src.fracDev.clipped()
                shapes = [src.shapeExp, src.shapeDev]
            elif isinstance(src, S.SersicGalaxy):
                r['profile'] = _lib.PROFILE_SERSIC
                r['sersic_n'] = src.sersicindex.val
                shapes = [src.shape]
            elif isinstance(src, (S.ExpGalaxy, S.DevGalaxy, S.GaussianGalaxy)):
                r['profile'] = {S.ExpGalaxy: _lib.PROFILE_EXP, S.DevGalaxy: _lib.PROFILE_DEV,
                                S.GaussianGalaxy: _lib.PROFILE_GAUSSIAN}[type(src)]
                shapes = [src.shape]
            else:
                return None
            kinds = set()
            for k, sh in enumerate(shapes):
                if isinstance(sh, E.EllipseESoft):
                    kinds.add(_lib.SHAPE_ELLIPSE_ESOFT)
                elif isinstance(sh, E.EllipseE):
                    kinds.add(_lib.SHAPE_ELLIPSE_E)
                elif isinstance(sh, E.GalaxyShape):
                    kinds.add(_lib.SHAPE_RABPHI)
                else:
                    return None
                vals = [float(v) for v in sh.getAllParams()]
                pre = 'sa' if k == 0 else 'sb'
                r[pre + '0'], r[pre + '1'], r[pre + '2'] = vals
            if len(kinds) > 1:
                return None
            r['shape_type'] = kinds.pop() if kinds else _lib.SHAPE_ELLIPSE_E
            rows.append(r)
        return np.array(rows, _lib.SCENE_SRC) if rows else np.zeros(0, _lib.SCENE_SRC)

    def _scene_model(self, img, srcs, sky, minsb):
        srcs = [s for s in srcs if s is not None]
        if len(srcs) < self.SCENE_MIN_SOURCES or self.modtype != np.float32:
            return None
        recs = self._scene_records(img, srcs, minsb)
        if recs is None:
            return None
        from . import batch
        psf = img.getPsf()
        mog = psf.getMixtureOfGaussians()
        H, W = img.getModelShape()
        cd = img.getWcs().cdInverseAtPixel(0, 0)
        scene = batch.SceneImage(W, H, np.asarray(mog.amp, np.float64),
                                 np.asarray(mog.mean, np.float64), np.asarray(mog.var, np.float64),
                                 pixscale=img.getWcs().pixscale_at(0, 0), cd_inv=cd)
        mod = np.zeros((H, W), np.float32)
        if sky:
            img.getSky().addTo(mod)
        if len(recs):
            r = batch.SceneRenderer([scene], comp_stride=16 * max(len(mog.amp), 1))
            mod += r.image(r.render(recs).numpy(), 0)
        return mod

    def getModelImages(self, **kwargs):
        plan = RenderPlan()
        fins = [self._plan_model_image(plan, img, **kwargs) for img in self.images]
        for f in fins:
            yield f()

    def getChiImage(self, imgi=-1, img=None, srcs=None, minsb=0., **kwargs):
        if img is None:
            img = self.getImage(imgi)
        mod = self.getModelImage(img, srcs=srcs, minsb=minsb, **kwargs)
        return (img.getImage() - mod) * img.getInvError()

    def getChiImages(self, **kwargs):
        plan = RenderPlan()
        fins = [(img, self._plan_model_image(plan, img, minsb=0., **kwargs)) for img in self.images]
        for img, f in fins:
            yield (img.getImage() - f()) * img.getInvError()

    def getLogLikelihood(self, **kwargs):
        chisq = 0.
        for chi in self.getChiImages(**kwargs):
            chisq += (chi.astype(float) ** 2).sum()
        return -0.5 * chisq

    def getLogProb(self, **kwargs):
        """engine.py:481-497."""
        lnprior = self.getLogPrior()
        if lnprior == -np.inf:
            return lnprior
        lnl = self.getLogLikelihood(**kwargs)
        lnp = lnprior + lnl
        if np.isnan(lnp):
            return -np.inf
        return lnp

    # -- derivatives (engine.py:279-339) ----------------------------------
    def _plan_derivs(self, plan, **kwargs):
        allderivs = []
        if self.isParamFrozen('catalog'):
            srcs = []
        else:
            srcs = list(self.catalog.getThawedSources())
        pend = []
        if not self.isParamFrozen('images'):
            # image parameters (PSF, sky, ...) without analytic derivatives:
            # forward differences of the whole model image (engine.py:306-324),
            # the unperturbed and every perturbed model planned into the same
            # batch (a plan renders the state at the time of the call)
            for i in self.images.getThawedParamIndices():
                img = self.images[i]
                derivs = img.getParamDerivatives(self, self.catalog)
                fin0 = None
                for di, deriv in enumerate(derivs):
                    if deriv is False:
                        if fin0 is None:
                            fin0 = _once(self._plan_model_image(plan, img, **kwargs))
                            p0 = img.getParams()
                            stepsizes = img.getStepSizes()
                            paramnames = img.getParamNames()
                        oldval = img.setParam(di, p0[di] + stepsizes[di])
                        fin = self._plan_model_image(plan, img, **kwargs)
                        img.setParam(di, oldval)
                        deriv = _FiniteDifference(fin, fin0, stepsizes[di],
                                                  'd(im%i)/d(%s)' % (i, paramnames[di]))
                    allderivs.append([(deriv, img)])
        for src in srcs:
            per_img = []
            for img in self.images:
                mask = self._getModelMaskFor(img, src)
                if self.expectModelMasks and mask is None:
                    per_img.append((img, [None] * src.numberOfParams()))
                    continue
                per_img.append((img, src._plan_derivatives(plan, img, modelMask=mask, **kwargs)))
            pend.append((src, per_img))

        def finish():
            out = [[(d.result() if isinstance(d, _FiniteDifference) else d, img)
                    for d, img in col] for col in allderivs]
            for src, per_img in pend:
                srcderivs = [[] for _ in range(src.numberOfParams())]
                for img, plist in per_img:
                    for k, p in enumerate(plist):
                        d = p.result() if p is not None else None
                        if d is None:
                            continue
                        srcderivs[k].append((d, img))
                out.extend(srcderivs)
            assert len(out) == self.numberOfParams()
            return out
        return finish

    def getDerivs(self, **kwargs):
        """Nested list, one entry per thawed parameter, of (Patch, Image)
        pairs (engine.py:279-339); all renders in one batch."""
        plan = RenderPlan()
        return self._plan_derivs(plan, **kwargs)()
