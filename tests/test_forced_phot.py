"""Forced photometry (Tractor.optimize_forced_photometry through
B200Optimizer.forced_photometry): the reference's own known answers
(test/test_forced_phot.py:69-147) and a multi-source, two-image fit against
the reference itself (tests/golden/forced_phot.npz, made by
tests/golden/make_golden.py).  Runs on the host stand-ins and on the GPU."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


@pytest.fixture(params=['host', pytest.param('gpu', marks=pytest.mark.gpu)])
def backend(request, monkeypatch):
    if request.param == 'host':
        import fake_device
        fake_device.install(monkeypatch)
    else:
        request.getfixturevalue('tb')
    from tractor_b200 import render
    render._spectra.cache.clear()
    return request.param


def _constant_source_classes():
    import tractor_b200 as T
    from tractor_b200.patch import Patch

    class ConstantSource(T.MultiParams, T.BasicSource):
        """A source whose unit-flux model is 1 on every pixel (the
        reference test's ConstantSource)."""

        def __init__(self, br):
            super(ConstantSource, self).__init__(br)

        @staticmethod
        def getNamedParams():
            return dict(brightness=0)

        def getBrightness(self):
            return self.brightness

        def getBrightnesses(self):
            return [self.brightness]

        def getUnitFluxModelPatches(self, img, modelMask=None, **kwargs):
            shape = img.shape if modelMask is None else modelMask.shape
            return [Patch(0, 0, np.ones(shape, np.float32))]

        def getModelPatch(self, img, modelMask=None, **kwargs):
            counts = img.getPhotoCal().brightnessToCounts(self.brightness)
            if counts == 0:
                return None
            return self.getUnitFluxModelPatches(img, modelMask=modelMask)[0] * counts

        def _plan_model_patch(self, plan, img, modelMask=None, **kwargs):
            from tractor_b200.plan import done
            return done(self.getModelPatch(img, modelMask=modelMask))

    class ConstantSourceWithPrior(T.GaussianPriorsMixin, ConstantSource):
        priorStd = 1.

        def __init__(self, *args, **kwargs):
            super(ConstantSourceWithPrior, self).__init__(*args, **kwargs)
            self.gpriors.add('brightness', 0., self.priorStd, param=self)

    return ConstantSource, ConstantSourceWithPrior


def _pixel_tim(val):
    import tractor_b200 as T
    return T.Image(data=np.zeros((1, 1), np.float32) + val, inverr=np.ones((1, 1), np.float32),
                   photocal=T.LinearPhotoCal(1.))


def test_pixel(backend):
    """test_forced_phot.py:69-88."""
    import tractor_b200 as T
    ConstantSource, _ = _constant_source_classes()
    tim = _pixel_tim(42.)
    src = ConstantSource(T.Flux(10.))
    tr = T.Tractor([tim], [src])
    tr.freezeParam('images')
    tr.optimize_forced_photometry()
    assert abs(src.getParams()[0] - 42.) < 1e-6


def test_pixel_with_prior(backend):
    """test_forced_phot.py:90-147: a Gaussian prior of sigma 1 at 0 halves
    the fitted value; with inverr 2 the fit is the inverse-variance mean."""
    import tractor_b200 as T
    ConstantSource, ConstantSourceWithPrior = _constant_source_classes()
    val = 4.
    tim = _pixel_tim(val)
    src = ConstantSource(T.Flux(0.))
    tr = T.Tractor([tim], [src])
    tr.freezeParam('images')
    tr.optimize_forced_photometry()
    assert abs(src.getParams()[0] - val) < 1e-6
    src = ConstantSourceWithPrior(T.Flux(0.))
    tr = T.Tractor([tim], [src])
    tr.freezeParam('images')
    tr.optimize_forced_photometry(priors=True)
    assert abs(src.getParams()[0] - val / 2.) < 1e-6
    src.setParams([1.])
    tr.optimize_forced_photometry(priors=True)
    assert abs(src.getParams()[0] - val / 2.) < 1e-6
    tim.inverr[:, :] = 2.
    src.setParams([0.])
    tr.optimize_forced_photometry(priors=True)
    pval = (4. * val) / (4. + 1.)
    assert abs(src.getParams()[0] - pval) < 1e-6


def test_fluxes_and_variance_match_reference(backend):
    import tractor_b200 as T
    g = np.load(os.path.join(GOLDEN, 'forced_phot.npz'))
    H, W = g['data'].shape[1:]
    psfs = [T.NCircularGaussianPSF([1.2, 2.6], [0.75, 0.25]),
            T.GaussianMixturePSF(np.array([0.6, 0.3, 0.1]), np.zeros((3, 2)),
                                 np.array([np.eye(2) * s ** 2 for s in (1.5, 3.0, 6.0)]))]
    tims = [T.Image(data=g['data'][b], inverr=np.full((H, W), 2., np.float32), psf=psfs[b],
                    photocal=T.LinearPhotoCal(float(g['scales'][b]))) for b in range(2)]
    srcs = []
    for kind, px, py, fl, re, e1, e2 in g['sources']:
        pos, br = T.PixPos(px, py), T.Flux(fl)
        if int(kind) == 0:
            s = T.PointSource(pos, br)
        elif int(kind) == 1:
            s = T.ExpGalaxy(pos, br, T.EllipseE(re, e1, e2))
        else:
            s = T.DevGalaxy(pos, br, T.EllipseE(re, e1, e2))
        srcs.append(s)
    tr = T.Tractor(tims, srcs)
    tr.freezeParam('images')
    for s in srcs:
        s.freezeAllBut('brightness')
    tr.setParams(g['start'])
    R = tr.optimize_forced_photometry(variance=True, shared_params=False)
    got = np.array(tr.getParams())
    assert np.allclose(got, g['fluxes'], rtol=1e-5, atol=0), (got, g['fluxes'])
    assert np.allclose(R.IV, g['IV'], rtol=1e-4), (R.IV, g['IV'])


def test_sky_fit_fitstats_and_justims0_match_reference(backend):
    """Forced photometry with the images' constant skies fitted along with
    the fluxes (sky=True: sky columns first in the update, the sky rendered
    at each trial), justims0's first evaluation, the fluxes' variance and the
    fit statistics, against the reference (tests/golden/forced_sky.npz)."""
    _sky_fit()


def _sky_fit():
    import tractor_b200 as T
    g = np.load(os.path.join(GOLDEN, 'forced_sky.npz'))
    H, W = g['data'].shape[1:]
    psfs = [T.NCircularGaussianPSF([1.2, 2.6], [0.75, 0.25]),
            T.GaussianMixturePSF(np.array([0.6, 0.3, 0.1]), np.zeros((3, 2)),
                                 np.array([np.eye(2) * s ** 2 for s in (1.5, 3.0, 6.0)]))]
    scales = [1.0, 2.5]
    tims = [T.Image(data=g['data'][b], inverr=np.full((H, W), 2., np.float32), psf=psfs[b],
                    photocal=T.LinearPhotoCal(scales[b]), sky=T.ConstantSky(0.)) for b in range(2)]
    srcs = []
    for kind, px, py, fl, re, e1, e2 in g['sources']:
        pos, br = T.PixPos(px, py), T.Flux(fl)
        if int(kind) == 0:
            s = T.PointSource(pos, br)
        elif int(kind) == 1:
            s = T.ExpGalaxy(pos, br, T.EllipseE(re, e1, e2))
        else:
            s = T.DevGalaxy(pos, br, T.EllipseE(re, e1, e2))
        s.freezeAllBut('brightness')
        srcs.append(s)
    tr = T.Tractor(tims, srcs)
    for tim in tims:
        tim.freezeAllBut('sky')
    tr.setParams(g['start'])
    assert tr.getParamNames() == list(g['names'])
    R0 = tr.optimize_forced_photometry(sky=True, justims0=True, shared_params=False)
    assert np.isclose(R0.lnp0, float(g['lnp0']), rtol=1e-7)
    assert np.abs(np.stack(R0.chis0) - g['chis0']).max() < 1e-3
    assert np.array_equal(tr.getParams(), g['start'])
    R = tr.optimize_forced_photometry(sky=True, variance=True, fitstats=True,
                                      shared_params=False)
    # The reference solves each update by LSQR on unscaled columns (the sky
    # columns span every pixel) and stops on dlnp < 1 close to, not at, the
    # least-squares optimum; the device solve is exact.  So: skies within
    # 1e-4, fluxes within 0.02 sigma of the reference's, and a likelihood at
    # least as high.
    got = np.array(tr.getParams())
    sigma = 1. / np.sqrt(g['IV'])
    assert np.abs(got[:2] - g['params'][:2]).max() < 1e-4
    assert np.all(np.abs(got[2:] - g['params'][2:]) < 0.02 * sigma), (got, g['params'])
    lnl = tr.getLogLikelihood()
    tr.setParams(g['params'])
    assert lnl >= tr.getLogLikelihood() - 1e-6
    tr.setParams(got)
    np.testing.assert_allclose(R.IV, g['IV'], rtol=1e-4)
    # the fit statistics are evaluated at the fitted fluxes (which differ by
    # up to 1.3e-4 relative, above): 1e-3; the port itself is pinned exactly
    # by test_fitstats_port_equals_reference
    fs = R.fitstats
    for k in ('npix', 'imnpix'):
        assert np.array_equal(np.asarray(getattr(fs, k)), g['fs_' + k]), k
    for k in ('prochi2', 'pronpix', 'promasked', 'profracflux', 'proflux', 'fracin', 'imchisq',
              'sky'):
        np.testing.assert_allclose(np.asarray(getattr(fs, k)), g['fs_' + k], rtol=1e-3,
                                   atol=1e-6, err_msg=k)
    return tr, R


@pytest.mark.reference
def test_fitstats_port_equals_reference(monkeypatch):
    """The fit statistics port (B200Optimizer._get_fitstats) against the
    reference's own Optimizer._get_fitstats (optimize.py:233-375) run on
    the same fitted images and unit-flux models: identical."""
    from oracle import refharness
    if not refharness.available():
        pytest.skip('reference source tree not present')
    import fake_device
    fake_device.install(monkeypatch)
    tr, R = _sky_fit()
    from tractor_b200.optimizer import B200Optimizer
    opt = B200Optimizer()
    imgs = list(tr.getImages())
    srcs = list(tr.catalog.getThawedSources())
    umodels, ufs = opt._unit_models(tr, srcs, imgs, 0.)
    scales = [im.getPhotoCal().getScale() for im in imgs]
    ims = R.ims1
    mine = opt._get_fitstats(tr.catalog, ims, srcs, imgs, ufs, umodels, scales, -1e30)
    refharness.load()
    from tractor.optimize import Optimizer
    ref = Optimizer()._get_fitstats(tr.catalog, ims, srcs, imgs, ufs, umodels, scales, -1e30)
    for k in ('prochi2', 'pronpix', 'promasked', 'profracflux', 'proflux', 'npix', 'fracin',
              'imchisq', 'imnpix', 'sky'):
        assert np.array_equal(np.asarray(getattr(mine, k)), np.asarray(getattr(ref, k))), k


def test_nonneg_is_accepted_and_unused(backend):
    """LsqrOptimizer accepts nonneg and does not use it
    (lsqr_optimizer.py:11-38): the same fluxes either way."""
    import tractor_b200 as T
    g = np.load(os.path.join(GOLDEN, 'forced_phot.npz'))
    H, W = g['data'].shape[1:]
    out = []
    for nonneg in (False, True):
        tims = [T.Image(data=g['data'][b], inverr=np.full((H, W), 2., np.float32),
                        psf=T.NCircularGaussianPSF([1.2, 2.6], [0.75, 0.25]),
                        photocal=T.LinearPhotoCal(float(g['scales'][b]))) for b in range(2)]
        srcs = [T.PointSource(T.PixPos(px, py), T.Flux(fl))
                for kind, px, py, fl, re, e1, e2 in g['sources']]
        tr = T.Tractor(tims, srcs)
        tr.freezeParam('images')
        for s in srcs:
            s.freezeAllBut('brightness')
        tr.optimize_forced_photometry(nonneg=nonneg, shared_params=False)
        out.append(np.array(tr.getParams()))
    assert np.array_equal(out[0], out[1])


def _roi_tractor(T, g, sky):
    H, W = g['data'].shape[1:]
    psfs = [T.NCircularGaussianPSF([1.2, 2.6], [0.75, 0.25]),
            T.GaussianMixturePSF(np.array([0.6, 0.3, 0.1]), np.zeros((3, 2)),
                                 np.array([np.eye(2) * s ** 2 for s in (1.5, 3.0, 6.0)]))]
    tims = [T.Image(data=g['data'][b], inverr=np.full((H, W), 2., np.float32), psf=psfs[b],
                    photocal=T.LinearPhotoCal([1.0, 2.5][b]), sky=T.ConstantSky(0.))
            for b in range(2)]
    srcs = []
    for kind, px, py, fl, re, e1, e2 in g['sources']:
        pos, br = T.PixPos(px, py), T.Flux(fl)
        if int(kind) == 0:
            s = T.PointSource(pos, br)
        elif int(kind) == 1:
            s = T.ExpGalaxy(pos, br, T.EllipseE(re, e1, e2))
        else:
            s = T.DevGalaxy(pos, br, T.EllipseE(re, e1, e2))
        s.freezeAllBut('brightness')
        srcs.append(s)
    for tim in tims:
        if sky:
            tim.freezeAllBut('sky')
        else:
            tim.freezeAllParams()
    return tims, srcs


@pytest.mark.parametrize('sky', [False, True])
def test_rois_equal_the_fit_with_zero_weight_outside(backend, sky):
    """forced_photometry(rois=...) (optimize.py:45-83: unit-flux models of the
    full images shifted into each ROI, the fit on the ROI subimages, so
    sources whose centres lie outside an ROI still contribute their wings)
    equals the same fit on the full images with the inverse error set to
    zero outside each ROI: first evaluation, fluxes, variances and fitted
    skies (copied back to the full images).  The images and their model
    masks are put back afterwards."""
    import tractor_b200 as T
    g = np.load(os.path.join(GOLDEN, 'forced_sky.npz'))
    H, W = g['data'].shape[1:]
    rois = [(slice(6, H - 9), slice(4, W - 5)), (slice(0, H - 3), slice(7, W))]
    start = np.array(g['start']) if sky else np.array(g['start'])[2:]
    tims, srcs = _roi_tractor(T, g, sky)
    tr = T.Tractor(tims, srcs)
    tr.setParams(start)
    R0 = tr.optimize_forced_photometry(sky=sky, justims0=True, shared_params=False, rois=rois)
    R = tr.optimize_forced_photometry(sky=sky, variance=True, shared_params=False, rois=rois)
    got = np.array(tr.getParams())
    assert list(tr.getImages()) == tims
    assert tr.modelMasks is None
    # the same fit on the full images, weighted by the ROIs only
    tims2, srcs2 = _roi_tractor(T, g, sky)
    for t, r in zip(tims2, rois):
        ie = np.zeros_like(t.getInvError())
        ie[r] = t.getInvError()[r]
        t.inverr = ie
    tr2 = T.Tractor(tims2, srcs2)
    tr2.setParams(start)
    S0 = tr2.optimize_forced_photometry(sky=sky, justims0=True, shared_params=False)
    S = tr2.optimize_forced_photometry(sky=sky, variance=True, shared_params=False)
    want = np.array(tr2.getParams())
    assert np.isclose(R0.lnp0, S0.lnp0, rtol=1e-9), (R0.lnp0, S0.lnp0)
    for a, b, r in zip(R0.chis0, S0.chis0, rois):
        assert a.shape == b[r].shape
        assert np.abs(a - b[r]).max() < 1e-4
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(R.IV, S.IV, rtol=1e-6)
