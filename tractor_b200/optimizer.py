"""Least-squares optimisers with the reference's Optimizer API
(tractor/optimize.py, tractor/lsqr_optimizer.py,
tractor/constrained_optimizer.py), solving on the GPU.

B200Optimizer is a drop-in beside LsqrOptimizer: the update direction is
the solution of the same column-scaled least-squares problem
(lsqr_optimizer.py:328-644) -- rows = image pixels weighted by the inverse
error plus Gaussian-prior rows, b = chi -- formed as normal equations on
the device (FP32 products, compensated sums, FP64 results) and solved by an
FP64 Cholesky factorisation with one step of iterative refinement.  The line
search renders every trial step of tryUpdates (optimize.py:425-470) in one
batch and applies the reference's sequential acceptance rule to the results.

B200ConstrainedOptimizer adds ConstrainedOptimizer's max-step and bound
handling (constrained_optimizer.py:12-159).
"""
import numpy as np

from . import render
from .plan import RenderPlan


class OptResult(object):
    """Results of a forced-photometry fit (optimize.py: OptResult)."""


def _copy_thaw_state(src, dst):
    """Gives `dst` (a parameter object of the same structure, e.g. a
    subimage) the thawed / frozen state of `src`, recursively."""
    if hasattr(src, 'liquid') and hasattr(dst, 'liquid') and len(src.liquid) == len(dst.liquid):
        dst.liquid[:] = list(src.liquid)
    for a, b in zip(getattr(src, 'subs', None) or [], getattr(dst, 'subs', None) or []):
        _copy_thaw_state(a, b)


def default_alphas():
    """1/1024 .. 1 in factors of 2, then sqrt(2), 2 (optimize.py:426-428)."""
    return np.append(2. ** np.arange(-10, 1), [np.sqrt(2.), 2.])


class B200Optimizer(object):

    # -- update direction --------------------------------------------------
    def getLinearUpdateDirection(self, tractor, damp=0, priors=True, scale_columns=True,
                                 shared_params=True, variance=False, **kwargs):
        """The derivatives and the chi images at the current parameters are
        rendered in one plan (one launch per kernel type and one copy back)
        unless an image's model goes through the scene renderer; the
        log-probability there is kept for tryUpdates' starting value."""
        self._lnp0 = None
        imgs = list(tractor.getImages())
        nsrc = sum(1 for s in tractor.catalog if s is not None)
        chis = None
        if nsrc < tractor.SCENE_MIN_SOURCES or tractor.modtype != np.float32:
            plan = RenderPlan()
            fd = tractor._plan_derivs(plan)
            fm = [tractor._plan_model_image(plan, img, minsb=0.) for img in imgs]
            allderivs = fd()
            chis = [(img.getImage() - f()) * img.getInvError() for img, f in zip(imgs, fm)]
            lnprior = tractor.getLogPrior()
            if lnprior != -np.inf:
                chisq = 0.
                for chi in chis:
                    chisq += (chi.astype(float) ** 2).sum()
                lnp = lnprior - 0.5 * chisq
                self._lnp0 = (tuple(tractor.getParams()), -np.inf if np.isnan(lnp) else lnp)
        else:
            allderivs = tractor.getDerivs()
        return self.getUpdateDirection(tractor, allderivs, damp=damp, priors=priors,
                                       scale_columns=scale_columns, shared_params=shared_params,
                                       variance=variance, chiImages=chis)

    def getUpdateDirection(self, tractor, allderivs, damp=0., priors=True, scale_columns=True,
                           scales_only=False, chiImages=None, variance=False,
                           shared_params=True, get_A_matrix=False):
        """The least-squares update (lsqr_optimizer.py:328-644).  Rows are
        restricted, per image, to the union box of the derivative patches
        (rows outside it are zero in A and do not change the solution)."""
        Ncols = len(allderivs)
        if shared_params:
            p0 = tractor.getParams()
            tractor.setParams(np.arange(len(p0)))
            p1 = tractor.getParams()
            tractor.setParams(p0)
            U, paramindexmap = np.unique(p1, return_inverse=True)
        # per-image ROI: union of derivative extents clipped to the image
        rois = {}
        order = []
        for param in allderivs:
            for deriv, img in param:
                H, W = img.shape
                d = deriv.copy()
                if not d.clipTo(W, H) or d.patch is None:
                    continue
                x0, x1, y0, y1 = d.getExtent()
                if img not in rois:
                    rois[img] = [x0, x1, y0, y1]
                    order.append(img)
                else:
                    r = rois[img]
                    rois[img] = [min(r[0], x0), max(r[1], x1), min(r[2], y0), max(r[3], y1)]
        row0 = {}
        nrows = 0
        for img in order:
            x0, x1, y0, y1 = rois[img]
            row0[img] = nrows
            nrows += (x1 - x0) * (y1 - y0)
        npix_rows = nrows
        # prior rows
        prior = None
        if priors:
            X = tractor.getLogPriorDerivatives()
            if X is not None:
                rA, cA, vA, pb, _ = X
                nr = max([max(r) for r in rA if len(r)] + [-1]) + 1
                prior = (rA, cA, vA, pb, nr)
                nrows += nr
        if nrows == 0:
            return []
        A = np.zeros((Ncols, nrows), np.float32)   # column-major: A[col] is one column
        b = np.zeros(nrows, np.float32)
        anyval = False
        for col, param in enumerate(allderivs):
            for deriv, img in param:
                H, W = img.shape
                d = deriv.copy()
                if not d.clipTo(W, H) or d.patch is None:
                    continue
                x0, x1, y0, y1 = rois[img]
                rw = x1 - x0
                vals = d.patch * img.getInvError()[d.getSlice(img)]
                if not np.any(vals):
                    continue
                anyval = True
                h, w = vals.shape
                # the image's ROI rows of column col as a (rows, rw) view
                roi = A[col, row0[img]:row0[img] + (y1 - y0) * rw].reshape(y1 - y0, rw)
                roi[d.y0 - y0:d.y0 - y0 + h, d.x0 - x0:d.x0 - x0 + w] += vals.astype(np.float32)
        if prior is not None:
            rA, cA, vA, pb, nr = prior
            for ri, ci, vi in zip(rA, cA, vA):
                A[ci, npix_rows + np.array(ri)] = np.array(vi, np.float32)
            b[npix_rows:] = np.hstack(pb)
        if not anyval and prior is None:
            return []
        if not np.all(np.isfinite(A)):
            print('Warning: infinite derivatives; bailing out')
            return None
        colscales = np.sqrt((A.astype(np.float64) ** 2).sum(axis=1))
        if scales_only:
            return colscales
        # b = chi over each image's ROI (float32, as the reference)
        chis = None
        if chiImages is not None:
            chis = dict(zip(tractor.getImages(), chiImages))
        for img in order:
            x0, x1, y0, y1 = rois[img]
            chi = chis.get(img) if chis is not None else None
            if chi is None:
                chi = tractor.getChiImage(img=img)
            assert np.all(np.isfinite(chi))
            b[row0[img]:row0[img] + (x1 - x0) * (y1 - y0)] = chi[y0:y1, x0:x1].ravel()
        var = colscales ** 2 if variance else None
        # scale columns (the reference divides each column by its norm and
        # merges shared parameters afterwards)
        cs = np.where(colscales > 0, colscales, 1.)
        As = A / cs[:, None].astype(np.float32) if scale_columns else A
        if shared_params and not np.array_equal(paramindexmap, np.arange(Ncols)):
            ncols = int(paramindexmap.max()) + 1
            Am = np.zeros((ncols, nrows), np.float32)
            np.add.at(Am, paramindexmap, As)
        else:
            # no parameter shared: the merge would copy every column once
            Am = As
        X = self._solve(Am, b, damp)
        if X is None:
            return np.zeros(len(paramindexmap) if shared_params else Ncols)
        if shared_params:
            X = X[paramindexmap]
        if scale_columns:
            X = np.where(colscales > 0, X / cs, X)
        if variance:
            if shared_params:
                var = var[paramindexmap]
            return X, 1. / var
        return X

    def _solve(self, A_colmajor, b, damp):
        """argmin ||A x - b||^2 + damp^2 ||x||^2 on the device (columns of A
        are rows of A_colmajor)."""
        X, info = render.solve_dense(A_colmajor, b, damp=damp)
        if info != 0:
            return None
        return X

    # -- line search ---------------------------------------------------------
    def _batched_logprobs(self, tractor, p0, X, alphas):
        """log-prob at p0 + alpha X for every alpha: all model images of all
        trial steps rendered in one plan."""
        plan = RenderPlan()
        fins = []
        for alpha in alphas:
            tractor.setParams([p + alpha * d for p, d in zip(p0, X)])
            lnprior = tractor.getLogPrior()
            if lnprior == -np.inf:
                fins.append((lnprior, None))
                continue
            fins.append((lnprior, [(img, tractor._plan_model_image(plan, img, minsb=0.))
                                   for img in tractor.getImages()]))
        tractor.setParams(p0)
        out = []
        for lnprior, imgs in fins:
            if imgs is None:
                out.append(lnprior)
                continue
            chisq = 0.
            for img, f in imgs:
                chi = (img.getImage() - f()) * img.getInvError()
                chisq += (chi.astype(float) ** 2).sum()
            lnp = lnprior - 0.5 * chisq
            out.append(-np.inf if np.isnan(lnp) else lnp)
        return out

    def tryUpdates(self, tractor, X, alphas=None):
        """Optimizer.tryUpdates (optimize.py:425-470)."""
        if alphas is None:
            alphas = default_alphas()
        cached = getattr(self, '_lnp0', None)
        self._lnp0 = None
        if cached is not None and cached[0] == tuple(tractor.getParams()):
            pBefore = cached[1]        # rendered with the update direction's chi images
        else:
            pBefore = tractor.getLogProb()
        pBest = pBefore
        alphaBest = None
        p0 = tractor.getParams()
        lnps = self._batched_logprobs(tractor, p0, X, alphas)
        for alpha, pAfter in zip(alphas, lnps):
            if not np.isfinite(pAfter):
                break
            if pAfter < (pBest - 1.):
                break
            if pAfter > pBest:
                alphaBest = alpha
                pBest = pAfter
        if alphaBest is None:
            tractor.setParams(p0)
            return 0, 0.
        tractor.setParams([p + alphaBest * d for p, d in zip(p0, X)])
        return pBest - pBefore, alphaBest

    # -- optimize / loop (lsqr_optimizer.py:280-326) -----------------------
    def optimize(self, tractor, alphas=None, damp=0, priors=True, scale_columns=True,
                 shared_params=True, variance=False, just_variance=False, **nil):
        X = self.getLinearUpdateDirection(tractor, damp=damp, priors=priors,
                                          scale_columns=scale_columns,
                                          shared_params=shared_params, variance=variance)
        if X is None:
            return (0., None, 0.)
        if variance:
            if len(X) == 0:
                return 0, X, 0, None
            X, var = X
            if just_variance:
                return var
        if len(X) == 0:
            return 0, X, 0.
        dlogprob, alpha = self.tryUpdates(tractor, X, alphas=alphas)
        if variance:
            return dlogprob, X, alpha, var
        return dlogprob, X, alpha

    def optimize_loop(self, tractor, dchisq=0., steps=50, **kwargs):
        R = {}
        for step in range(steps):
            dlnp, X, alpha = self.optimize(tractor, **kwargs)
            if dlnp <= dchisq:
                break
        R.update(steps=step)
        return R

    # -- forced photometry (optimize.py:16-146, lsqr_optimizer.py:11-251) ---
    def forced_photometry(self, tractor, alphas=None, damp=0, priors=False, minsb=0.,
                          mindlnp=1., rois=None, sky=False, minFlux=None, fitstats=False,
                          fitstat_extras=None, justims0=False, variance=False,
                          skyvariance=False, shared_params=True, nonneg=False,
                          nilcounts=-1e30, wantims=True, negfluxval=None, **kwargs):
        """Linear fit of the thawed sources' brightnesses (and, with sky=True,
        of every image's one-parameter sky) with every other parameter fixed
        (Optimizer.forced_photometry, optimize.py:16-145, with
        LsqrOptimizer's loop, lsqr_optimizer.py:11-235): unit-flux models of
        all (image, source) pairs rendered in one batch, the frozen sources'
        model as the base (without the sky when it is fitted), then an
        unscaled least-squares update on the device (getUpdateDirection with
        chi images of the current state; sky columns first), alpha = 1 when
        the fluxes stay above minFlux, otherwise the line search with growing
        damping, until the gain is below mindlnp.  Returns an OptResult with
        ims0 / ims1 (image, model, inverr, chi, roi), with justims0 only the
        first evaluation (lnp0, chis0, ims0), with variance=True IV (the
        sky parameters first with skyvariance), with fitstats=True the
        reference's fit statistics.  nonneg and negfluxval are accepted and,
        as by LsqrOptimizer (lsqr_optimizer.py:11-38), not used.

        rois: one (slice(y0, y1), slice(x0, x1)) per image.  As in
        optimize.py:45-83 and 147-219, the unit-flux models are rendered on
        the full images (with their model masks) and shifted into each ROI,
        and the fit runs on img.subimage(x0, x1, y0, y1): the frozen
        sources' model, chi, update, line search, variances and fit
        statistics all cover the ROI pixels only; a fitted sky is copied back
        to the full images' skies (a one-parameter sky does not depend on the
        origin).  The reference's own ROI path takes chi from the inverse
        error instead of the image (optimize.py:503-506: `im = ie[roi]` after
        `ie = ie[roi]`), which fails on a shape mismatch for any ROI not at
        the origin; here chi is (image - model) x inverr of the ROI, which is
        what the reference computes without ROIs on the same subimages."""
        from .basics import LinearPhotoCal
        result = OptResult()
        imgs = list(tractor.getImages())
        scales = []
        for img in imgs:
            assert isinstance(img.getPhotoCal(), LinearPhotoCal)
            scales.append(img.getPhotoCal().getScale())
        if sky:
            for img in imgs:
                assert img.getSky().numberOfParams() == 1
        srcs = list(tractor.catalog.getThawedSources())
        nparams = tractor.catalog.numberOfParams()
        umodels, umodsforsource = self._unit_models(tractor, srcs, imgs, minsb, **kwargs)
        for um in umodels:
            assert len(um) == nparams
        if rois is not None:
            return self._forced_photometry_rois(
                tractor, rois, umodels, umodsforsource, srcs, nparams, scales, result,
                dict(alphas=alphas, damp=damp, priors=priors, minsb=minsb, mindlnp=mindlnp,
                     sky=sky, minFlux=minFlux, fitstats=fitstats, fitstat_extras=fitstat_extras,
                     justims0=justims0, variance=variance, skyvariance=skyvariance,
                     shared_params=shared_params, nilcounts=nilcounts, wantims=wantims))
        return self._forced_core(tractor, imgs, umodels, umodsforsource, srcs, nparams, scales,
                                 result, alphas=alphas, damp=damp, priors=priors, minsb=minsb,
                                 mindlnp=mindlnp, sky=sky, minFlux=minFlux, fitstats=fitstats,
                                 fitstat_extras=fitstat_extras, justims0=justims0,
                                 variance=variance, skyvariance=skyvariance,
                                 shared_params=shared_params, nilcounts=nilcounts,
                                 wantims=wantims)

    def _forced_photometry_rois(self, tractor, rois, umodels, umodsforsource, srcs, nparams,
                                scales, result, kw):
        """forced_photometry over ROIs: the full images' unit-flux models
        shifted into ROI coordinates (optimize.py:166-184), the fit run with
        the tractor's images replaced by the ROI subimages (their model masks
        shifted alike), the images and masks put back afterwards."""
        from .engine import Images
        from .patch import ModelMask
        imgs = list(tractor.getImages())
        assert len(rois) == len(imgs)
        origins, subimgs, shifted = [], [], []
        for img, roi, umods in zip(imgs, rois, umodels):
            y0, y1 = roi[0].start, roi[0].stop
            x0, x1 = roi[1].start, roi[1].stop
            origins.append((x0, y0))
            sub = img.subimage(x0, x1, y0, y1)
            _copy_thaw_state(img, sub)     # the fit's parameters are the full images' thawed ones
            subimgs.append(sub)
            row = []
            for um in umods:
                if um is not None and um.patch is not None:
                    um = um.copy()
                    um.x0 -= x0
                    um.y0 -= y0
                row.append(um)
            shifted.append(row)
        realims, realmasks = tractor.images, tractor.modelMasks
        masks = None
        if realmasks is not None:
            masks = []
            for (x0, y0), mm in zip(origins, realmasks):
                d = {}
                for src, m in mm.items():
                    if m is None:
                        d[src] = None
                    elif m.mask is not None:
                        d[src] = ModelMask(m.x0 - x0, m.y0 - y0, m.mask)
                    else:
                        d[src] = ModelMask(m.x0 - x0, m.y0 - y0, m.w, m.h)
                masks.append(d)
        tractor.images = Images(*subimgs)
        tractor.modelMasks = masks
        try:
            result = self._forced_core(tractor, subimgs, shifted, umodsforsource, srcs, nparams,
                                       scales, result, **kw)
        finally:
            if kw.get('sky'):
                for img, sub in zip(imgs, subimgs):
                    img.getSky().setParams(sub.getSky().getParams())
            tractor.images = realims
            tractor.modelMasks = realmasks
        return result

    def _forced_core(self, tractor, imgs, umodels, umodsforsource, srcs, nparams, scales,
                     result, alphas=None, damp=0, priors=False, minsb=0., mindlnp=1.,
                     sky=False, minFlux=None, fitstats=False, fitstat_extras=None,
                     justims0=False, variance=False, skyvariance=False, shared_params=True,
                     nilcounts=-1e30, wantims=True):
        """The forced-photometry fit proper (optimize.py:85-145,
        lsqr_optimizer.py:11-235) on `imgs` with their unit-flux models."""
        fsrcs = list(tractor.catalog.getFrozenSources())
        # with the sky fitted, each trial renders it from its parameters
        mod0 = [tractor.getModelImage(img, fsrcs, minsb=minsb, sky=not sky) for img in imgs]
        skyderivs, nsky = None, 0
        if sky:
            skyderivs = []
            for img in imgs:
                for dsky in img.getSky().getParamDerivatives(tractor, img, None):
                    skyderivs.append([(dsky, img)])
            nsky = len(skyderivs)
            assert nsky == tractor.images.numberOfParams()
            assert nsky + nparams == tractor.numberOfParams()
        derivs = [[] for _ in range(nparams)]
        for img, umods, scale in zip(imgs, umodels, scales):
            for um, dd in zip(umods, derivs):
                if um is not None:
                    dd.append((um * scale, img))
        if sky:
            derivs = skyderivs + derivs
        lnp0, chis0, ims0 = None, None, None
        imsBest = None
        damp0 = 1e-3
        damping = damp
        while True:
            tryAgain = False
            quitNow = False
            p0 = tractor.getParams()
            p0sky = None
            if sky:
                p0sky, p0 = p0[:nsky], p0[nsky:]
            if lnp0 is None:
                lnp0, chis0, ims0 = self._lnp_for_update(tractor, mod0, imgs, umodels, None, None,
                                                         p0, scales, None, None, priors, sky,
                                                         minFlux)
                assert np.isfinite(lnp0)
            if justims0:
                result.lnp0, result.chis0, result.ims0 = lnp0, chis0, ims0
                return result
            X = self.getUpdateDirection(tractor, derivs, damp=damping, priors=priors,
                                        scale_columns=False, chiImages=chis0,
                                        shared_params=shared_params)
            if X is None or len(X) == 0:
                break
            Xsky = None
            if sky:
                Xsky, X = X[:nsky], X[nsky:]
            trial = alphas
            if trial is None:
                trial = default_alphas()
            if minFlux is None or np.all((np.array(p0) + X) >= minFlux):
                trial = [1.]
                quitNow = True
            elif damp == 0.:
                damping = damp0
                damp0 *= 10.
                if damp0 < 1e3:
                    tryAgain = True
            lnpBest, alphaBest, chiBest = lnp0, None, None
            alpha = None
            for alpha in trial:
                lnp, chis, ims = self._lnp_for_update(tractor, mod0, imgs, umodels, X, alpha, p0,
                                                      scales, p0sky, Xsky, priors, sky, minFlux)
                if lnp < lnpBest - 1. or not np.isfinite(lnp):
                    break
                if lnp > lnpBest:
                    alphaBest, lnpBest, chiBest, imsBest = alpha, lnp, chis, ims
            if alphaBest is not None:
                pa = [p + alphaBest * d for p, d in zip(p0, X)]
                if minFlux is not None:
                    pa = [max(minFlux, v) for v in pa]
                tractor.catalog.setParams(pa)
                if sky:
                    # as lsqr_optimizer.py:187-189: the sky takes the last
                    # alpha the line search tried
                    tractor.images.setParams([p + alpha * d for p, d in zip(p0sky, Xsky)])
                dlogprob = lnpBest - lnp0
                lnp0, chis0 = lnpBest, chiBest
            else:
                dlogprob = 0.
                if sky:
                    tractor.images.setParams(p0sky)   # the line search moved it
            if dlogprob < mindlnp and not tryAgain:
                break
            if quitNow:
                break
        if wantims or fitstats:
            result.ims0 = ims0
            result.ims1 = imsBest
        if variance:
            result.IV = self._flux_iv(imgs, umodels, scales, nparams,
                                      skyderivs if (sky and skyvariance) else None)
        if fitstats:
            if imsBest is None:
                result.fitstats = None
            else:
                result.fitstats = self._get_fitstats(tractor.catalog, imsBest, srcs, imgs,
                                                     umodsforsource, umodels, scales, nilcounts,
                                                     extras=fitstat_extras)
        return result

    def _unit_models(self, tractor, srcs, imgs, minsb, **kwargs):
        """(n_images, n_params) unit-flux patches and, per source, the indices
        of its patches (Optimizer._get_umodels, optimize.py:147-219),
        rendered in one batch where the source can plan its renders."""
        plan = RenderPlan()
        pend = []
        for img in imgs:
            pcal = img.getPhotoCal()
            row = []
            for src in srcs:
                counts = sum([pcal.brightnessToCounts(b) for b in src.getBrightnesses()])
                mv = 1e-3 if counts <= 0 else minsb / counts
                mask = tractor._getModelMaskFor(img, src)
                if hasattr(src, '_plan_unit_patch'):
                    row.append(('plan', src._plan_unit_patch(plan, img, minval=mv, modelMask=mask,
                                                             **kwargs)))
                else:
                    row.append(('list', src.getUnitFluxModelPatches(img, minval=mv,
                                                                   modelMask=mask, **kwargs)))
            pend.append(row)
        umodels = []
        umodsforsource = [[] for _ in srcs]
        for i, row in enumerate(pend):
            umods = []
            for si, (kind, v) in enumerate(row):
                ums = [v.result()] if kind == 'plan' else list(v)
                for um in ums:
                    if um is not None and um.patch is not None:
                        assert np.all(np.isfinite(um.patch))
                if i == 0:
                    umodsforsource[si].extend(range(len(umods), len(umods) + len(ums)))
                umods.extend(ums)
            umodels.append(umods)
        return umodels, umodsforsource

    @staticmethod
    def _getims(fluxes, imgs, umodels, mod0, scales, sky, minFlux):
        """Image, model, inverr and chi images at the given fluxes (the sky
        rendered from its current parameters when it is fitted)
        (optimize.py:472-520)."""
        ims = []
        for img, umods, m0, scale in zip(imgs, umodels, mod0, scales):
            mod = m0.copy()
            if sky:
                img.getSky().addTo(mod)
            for f, um in zip(fluxes, umods):
                if um is None or um.patch is None:
                    continue
                if minFlux is not None:
                    f = max(f, minFlux)
                counts = f * scale
                if counts == 0.:
                    continue
                (um * counts).addTo(mod)
            ie = img.getInvError()
            im = img.getImage()
            chi = (im - mod) * ie
            ims.append((im, mod, ie, chi, None))
        return ims

    def _lnp_for_update(self, tractor, mod0, imgs, umodels, X, alpha, p0, scales, p0sky, Xsky,
                        priors, sky, minFlux):
        """lsqr_optimizer.py:237-261: the sky is set to its trial value, the
        prior evaluated at the tractor's current state."""
        pa = p0 if X is None else [p + alpha * d for p, d in zip(p0, X)]
        if Xsky is not None:
            tractor.images.setParams([p + alpha * d for p, d in zip(p0sky, Xsky)])
        lnp = 0.
        if priors:
            lnp += tractor.getLogPrior()
            if not np.isfinite(lnp):
                return lnp, None, None
        ims = self._getims(pa, imgs, umodels, mod0, scales, sky, minFlux)
        chis = [chi for _, _, _, chi, _ in ims]
        lnp += -0.5 * sum((chi.astype(np.float64) ** 2).sum() for chi in chis)
        return lnp, chis, ims

    @staticmethod
    def _flux_iv(imgs, umodels, scales, nparams, skyderivs=None):
        """Inverse variances (Optimizer._get_iv, optimize.py:378-423): for
        each sky parameter (when given) the sum of (dsky x inverr)^2, then for
        each flux the sum over images of (unit model x scale x inverr)^2."""
        nsky = len(skyderivs) if skyderivs else 0
        IV = np.zeros(nsky + nparams)
        for di, ((dsky, tim),) in enumerate(skyderivs or []):
            ie = tim.getInvError()
            mm = np.zeros(tim.shape)
            dsky.addTo(mm)
            IV[di] = np.sum((mm * ie) ** 2)
        for img, umods, scale in zip(imgs, umodels, scales):
            ie = img.getInvError()
            H, W = img.shape
            for ui, um in enumerate(umods):
                if um is None or um.patch is None:
                    continue
                d = um.copy()
                if not d.clipTo(W, H) or d.patch is None:
                    continue
                IV[nsky + ui] += np.sum((d.patch * scale * ie[d.getSlice(img)]) ** 2)
        return IV

    @staticmethod
    def _get_fitstats(catalog, imsBest, srcs, imlist, umodsforsource, umodels, scales, nilcounts,
                      extras=None):
        """Optimizer._get_fitstats (optimize.py:233-375): per image the chi^2
        and pixel count; per source the profile-weighted chi^2, pixel count,
        masked fraction, fraction of other sources' flux, other sources'
        flux, pixel count and fraction inside the images (host arithmetic on
        the images the fit produced; `extras` adds profile-weighted sums of
        given images)."""
        if extras is None:
            extras = []

        class FitStats(object):
            pass
        fs = FitStats()
        fs.imchisq = np.array([(chi ** 2).sum() for _, _, _, chi, _ in imsBest])
        fs.imnpix = np.array([(ie > 0).sum() for _, _, ie, _, _ in imsBest])
        n = len(srcs)
        fs.prochi2 = np.zeros(n)
        fs.pronpix = np.zeros(n)
        fs.promasked = np.zeros(n)
        fracflux_num = np.zeros(n)
        fracflux_den = np.zeros(n)
        fs.proflux = np.zeros(n)
        fs.npix = np.zeros(n, int)
        fracin_num = np.zeros(n)
        fracin_den = np.zeros(n)
        for key, x in extras:
            setattr(fs, key, np.zeros(n))
        # others' flux within a profile is measured without the sky
        skies = []
        for tim, (img, mod, ie, chi, roi) in zip(imlist, imsBest):
            tim.getSky().addTo(mod, scale=-1.)
            skies.append(getattr(tim.getSky(), 'val', 0.))
        fs.sky = np.array(skies)
        srcmods = [np.zeros_like(chi) for (img, mod, ie, chi, roi) in imsBest]
        for si, uis in enumerate(umodsforsource):
            src = catalog[si]
            for imi, (umods, scale, tim, (img, mod, ie, chi, roi)) in enumerate(
                    zip(umodels, scales, imlist, imsBest)):
                pcal = tim.getPhotoCal()
                cc = [pcal.brightnessToCounts(b) for b in src.getBrightnesses()]
                sourcecounts = sum(cc)
                if sourcecounts == 0:
                    continue
                srcmod = srcmods[imi]
                xlo = xhi = ylo = yhi = None
                for ui, counts in zip(uis, cc):
                    if counts == 0:
                        continue
                    um = umods[ui]
                    if um is None:
                        continue
                    x0, y0 = um.x0, um.y0
                    uh, uw = um.shape
                    xlo = x0 if xlo is None or x0 < xlo else xlo
                    xhi = x0 + uw if xhi is None or x0 + uw > xhi else xhi
                    ylo = y0 if ylo is None or y0 < ylo else ylo
                    yhi = y0 + uh if yhi is None or y0 + uh > yhi else yhi
                    (um * counts).addTo(srcmod)
                if xlo is None or xhi is None or ylo is None or yhi is None:
                    continue
                slc = slice(ylo, yhi), slice(xlo, xhi)
                srcmod[slc] /= sourcecounts
                nz = np.flatnonzero((srcmod[slc] != 0) * (ie[slc] > 0))
                if len(nz) == 0:
                    srcmod[slc] = 0.
                    continue
                fs.prochi2[si] += np.sum(np.abs(srcmod[slc].flat[nz]) * chi[slc].flat[nz] ** 2)
                fs.pronpix[si] += np.sum(np.abs(srcmod[slc].flat[nz]))
                fs.promasked[si] += np.sum(np.abs(srcmod[slc][ie[slc] == 0]))
                fracflux_num[si] += (np.sum((np.abs(mod[slc] / sourcecounts - srcmod[slc]) *
                                             np.abs(srcmod[slc])).flat[nz]) /
                                     np.sum((srcmod[slc] ** 2).flat[nz]))
                fracflux_den[si] += np.sum(np.abs(srcmod[slc]).flat[nz] / np.abs(sourcecounts))
                fs.proflux[si] += np.sum((np.abs((mod[slc] - srcmod[slc] * sourcecounts) / scale) *
                                          np.abs(srcmod[slc])).flat[nz])
                fs.npix[si] += len(nz)
                fracin_num[si] += np.sum(np.abs(srcmod[slc]))
                fracin_den[si] += 1.
                for key, extraims in extras:
                    x = getattr(fs, key)
                    x[si] += np.sum(np.abs(srcmod[slc].flat[nz]) * extraims[imi][slc].flat[nz])
                srcmod[slc] = 0.
        fs.profracflux = fracflux_num / np.maximum(1, fracflux_den)
        fs.fracin = fracin_num / np.maximum(1, fracin_den)
        for tim, (img, mod, ie, chi, roi) in zip(imlist, imsBest):
            tim.getSky().addTo(mod)
        return fs


class B200ConstrainedOptimizer(B200Optimizer):
    """ConstrainedOptimizer semantics (constrained_optimizer.py:12-159):
    trial steps limited by each parameter's max step and clipped to its
    bounds; the loop stops on dlnp <= dchisq, or <= dchisq_limited after a
    limited step."""

    def __init__(self, *args, **kwargs):
        super(B200ConstrainedOptimizer, self).__init__()
        self.stepLimited = False
        self.tiny_alpha = 1e-8

    def optimize_loop(self, tractor, dchisq=0., steps=100, dchisq_limited=1e-6, check_step=None,
                      **kwargs):
        R = {}
        self.hit_limit = False
        self.last_step_hit_limit = False
        for step in range(steps):
            self.stepLimited = False
            dlnp, X, alpha = self.optimize(tractor, **kwargs)
            if check_step is not None:
                if not check_step(optimizer=self, tractor=tractor, dlnp=dlnp, X=X, alpha=alpha):
                    break
            if not self.stepLimited and dlnp <= dchisq:
                break
            if self.stepLimited and dlnp <= dchisq_limited:
                break
        R.update(steps=step)
        R.update(hit_limit=self.last_step_hit_limit, ever_hit_limit=self.hit_limit)
        return R

    def tryUpdates(self, tractor, X, alphas=None, check_step=None):
        p_best = tractor.getParams()
        logprob_before = tractor.getLogProb()
        logprob_best = logprob_before
        alpha_best = None
        steps = self.getParameterSteps(tractor, X, alphas)
        if len(steps) == 0:
            self.stepLimited = True
            self.last_step_hit_limit = True
            self.hit_limit = True
        p0 = tractor.getParams()
        # evaluate all candidate parameter vectors in one batch
        plan = RenderPlan()
        fins = []
        for alpha, p, step_limit, hit_limit in steps:
            tractor.setParams(p)
            lnprior = tractor.getLogPrior()
            fins.append((lnprior, None if lnprior == -np.inf else
                         [(img, tractor._plan_model_image(plan, img, minsb=0.))
                          for img in tractor.getImages()]))
        tractor.setParams(p0)
        for (alpha, p, step_limit, hit_limit), (lnprior, imgs) in zip(steps, fins):
            if hit_limit:
                self.hit_limit = True
            if check_step is not None:
                tractor.setParams(p)
                ok = check_step(optimizer=self, tractor=tractor, X=X, alpha=alpha)
                tractor.setParams(p0)
                if not ok:
                    break
            if imgs is None:
                logprob = lnprior
            else:
                chisq = 0.
                for img, f in imgs:
                    chi = (img.getImage() - f()) * img.getInvError()
                    chisq += (chi.astype(float) ** 2).sum()
                logprob = lnprior - 0.5 * chisq
                if np.isnan(logprob):
                    logprob = -np.inf
            if not np.isfinite(logprob):
                break
            if logprob < (logprob_best - 1.):
                break
            if logprob > logprob_best:
                self.last_step_hit_limit = hit_limit
                alpha_best = alpha
                logprob_best = logprob
                p_best = p
        tractor.setParams(p_best)
        if alpha_best is None:
            return 0., 0.
        return logprob_best - logprob_before, alpha_best

    def getParameterSteps(self, tractor, step_direction, alphas):
        """constrained_optimizer.py:84-159."""
        if alphas is None:
            alphas = default_alphas()
        p0 = tractor.getParams()
        max_step_size = tractor.getMaxStep()
        lowers = tractor.getLowerBounds()
        uppers = tractor.getUpperBounds()
        assert np.all(np.diff(alphas) > 0)
        step_direction = np.array(step_direction)
        results = []
        for alpha in alphas:
            do_break = False
            step_limit = False
            for i, mx in enumerate(max_step_size):
                if mx is None:
                    continue
                step = alpha * abs(step_direction[i])
                if step > mx:
                    step_limit = True
                    do_break = True
                    alpha = mx / abs(step_direction[i])
                    self.stepLimited = True
            hit_limit = False
            for i, (ps, l, u) in enumerate(zip(p0, lowers, uppers)):
                px = ps + alpha * step_direction[i]
                if l is not None and px < l:
                    alpha = (l - ps) / step_direction[i]
                    hit_limit = True
                if u is not None and px > u:
                    alpha = (u - ps) / step_direction[i]
                    hit_limit = True
            if alpha < self.tiny_alpha:
                break
            p = []
            for ps, s, l, u in zip(p0, step_direction, lowers, uppers):
                px = ps + alpha * s
                if l is not None and px < l:
                    px = l
                if u is not None and px > u:
                    px = u
                p.append(px)
            results.append((alpha, p, step_limit, hit_limit))
            if do_break:
                break
        return results


# The reference's optimizer names: the same semantics, the least-squares
# update solved on the device (lsqr_optimizer.py, constrained_optimizer.py).
LsqrOptimizer = B200Optimizer
ConstrainedOptimizer = B200ConstrainedOptimizer
