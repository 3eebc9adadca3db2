"""Pins the oracle to the reference.

* Against the committed golden fixtures (tests/golden/*.npz, produced by the
  reference itself through tests/golden/make_golden.py): always runs.
* Against the reference's own compiled C and Python, live, where the
  reference source tree is present (marked `reference`, skipped otherwise).
* Against the known answers in the reference's own tests
  (test/test_galaxy.py, test/test_tractor.py).
"""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def _golden(name):
    return np.load(os.path.join(GOLDEN, name))


def test_kernels_match_golden(oracle):
    g = _golden('kernels.npz')
    amp, mean, var = g['amp'], g['mean'], g['var']
    grid = oracle.mog_grid(-5, 26, 3, 27, 7.3, 11.6, amp, mean, var)
    assert np.array_equal(grid, g['grid'])
    out, dx, dy, bbox = oracle.mog_approx3(0, 44, 0, 40, 20.4, 18.7, 1e-4, amp, mean, var,
                                           20, 18, 3, derivs=True)
    assert np.array_equal(out, g['approx'])
    assert np.array_equal(dx, g['approx_dx']) and np.array_equal(dy, g['approx_dy'])
    assert tuple(bbox) == tuple(g['approx_bbox'])
    lz = oracle.lanczos_shift(g['lanczos_in'], 0.37, -0.21)
    assert np.array_equal(lz, g['lanczos_out'])
    ft = oracle.fourier_mog(amp, g['var2'], np.fft.rfftfreq(32), np.fft.fftfreq(32))
    assert np.array_equal(ft, g['fourier'])


def test_fft_path_matches_golden(oracle):
    """The oracle's Fourier-path restatement (galaxy.py:336-519) reproduces the
    reference's SersicGalaxy patches."""
    g = _golden('fft_sersic.npz')
    for i, row in enumerate(g['params']):
        n, re, q, phi, px, py, r, e1, e2 = row
        amp, var = oracle.sersic_profile(n)
        T = oracle.nullwcs_cdinv() @ oracle.ellipseE_basis(r, e1, e2)
        a2, v2 = oracle.sheared(amp, var, T)
        G, _ = oracle.galaxy_fft_masked(a2, v2, px, py, g['psf'], 0, 0, 128, 128)
        ref = g['patches'][i] / 1000.
        assert np.abs(G - ref).max() <= 1e-6 * np.abs(ref).max(), i


def _unpack(g, key):
    n = len(g[key + '.present'])
    out, o = [], 0
    for i in range(n):
        if not g[key + '.present'][i]:
            out.append(None)
            continue
        h, w = int(g[key + '.h'][i]), int(g[key + '.w'][i])
        out.append((int(g[key + '.x0'][i]), int(g[key + '.y0'][i]),
                    g[key + '.pix'][o:o + h * w].reshape(h, w)))
        o += h * w
    return out


def test_mog_paths_match_golden(oracle):
    """Exp galaxy (GalaxyShape) with a GaussianMixturePSF, with and without a
    ModelMask: the oracle's MoG branch equals the reference's patches."""
    g = _golden('mog_sources.npz')
    amp, var = oracle.exp_profile()
    T = oracle.nullwcs_cdinv() @ oracle.galaxyshape_basis(2., 0.5, 45.)
    pamp, pmean = np.array([1.]), np.zeros((1, 2))
    pvar = np.array([[[6., -1.], [-1., 6.]]])
    # no mask: halfsize = max(nre * re, psf radius 25) clipped to the image
    hs = oracle.hogg_halfsize(4 * 2., 49.5, 50., 100, 100, 25)
    x0, x1, y0, y1 = oracle.image_extent(49.5, 50., hs, 100, 100)
    px0, py0, p = oracle.galaxy_mog_patch(amp, var, T, 49.5, 50., pamp, pmean, pvar, x0, x1, y0, y1)
    ref = _unpack(g, 'exp_nomask')[0]
    assert (px0, py0) == ref[:2] and p.shape == ref[2].shape
    assert np.abs(p * 100. - ref[2]).max() < 1e-12 * ref[2].max()
    p2 = oracle.galaxy_mog_masked_rect(amp, var, T, 49.5, 50., pamp, pmean, pvar, 20, 25, 60, 55)
    ref2 = _unpack(g, 'exp_mask')[0]
    assert np.abs(p2 * 100. - ref2[2]).max() < 1e-12 * ref2[2].max()


def test_scene_model_matches_golden(oracle):
    """80 mixed sources (point / exp / deV / composite) with square model
    masks and a 3-component MoG PSF, through the reference's
    Tractor.getModelImage: the oracle's scene model is bit-identical."""
    g = _golden('scene_mog.npz')
    H, W = (int(v) for v in g['shape'])
    mod = oracle.scene_model(g['sources'], g['psf_amp'], g['psf_sigma'], H, W)
    assert mod.dtype == np.float32
    assert np.array_equal(mod, g['model'])


def test_reference_known_answers(oracle):
    """test_galaxy.py:93-96: patch origin (24, 25), shape (52, 53), sum 100;
    test_tractor.py:74-88: peak flux / (2 pi sigma^2), lnp = -143.681."""
    amp, var = oracle.exp_profile()
    T = oracle.nullwcs_cdinv() @ oracle.galaxyshape_basis(2., 0.5, 45.)
    hs = oracle.hogg_halfsize(8., 49.5, 50., 100, 100, 25)
    x0, x1, y0, y1 = oracle.image_extent(49.5, 50., hs, 100, 100)
    px0, py0, p = oracle.galaxy_mog_patch(amp, var, T, 49.5, 50., [1.], np.zeros((1, 2)),
                                          np.array([[[6., -1.], [-1., 6.]]]), x0, x1, y0, y1)
    assert (px0, py0, p.shape) == (24, 25, (52, 53))
    assert abs(100. * p.sum() - 100.) < 1e-3
    chis = []
    for sig in (2., 3.):
        pa, pm, pv = oracle.circular_psf_mog([sig], [1.])
        mod = np.zeros((100, 100), np.float32)
        r = int(np.ceil(5 * sig))   # NCircularGaussianPSF.getRadius, psf.py:887-890
        patch = oracle.mogpsf_point_patch(pa, pm, pv, 50., 50., 50 - r, 50 + r + 1, 50 - r, 50 + r + 1)
        mod[50 - r:50 + r + 1, 50 - r:50 + r + 1] += patch * 100.
        assert abs(mod.max() - 100. / (2 * np.pi * sig ** 2)) < 1e-3
        chis.append(oracle.chi_image(np.zeros((100, 100)), mod, np.ones((100, 100))))
    assert abs(oracle.log_likelihood(chis) - -143.681) < 1e-3


@pytest.mark.reference
def test_oracle_matches_live_reference(oracle):
    from oracle import refharness
    if not refharness.available():
        pytest.skip('reference source tree not present')
    t = refharness.load()
    from tractor import mix, mp_fourier
    from tractor.sersic import SersicMixture
    rng = np.random.default_rng(5)
    for trial in range(20):
        K = int(rng.integers(1, 12))
        amp = rng.uniform(0.1, 1, K)
        mean = rng.normal(scale=2, size=(K, 2))
        var = np.zeros((K, 2, 2))
        for k in range(K):
            a = rng.normal(size=(2, 2))
            var[k] = a @ a.T + 0.2 * np.eye(2)
        W, H = int(rng.integers(5, 60)), int(rng.integers(5, 60))
        x0, y0 = int(rng.integers(-10, 10)), int(rng.integers(-10, 10))
        fx, fy = x0 + W * rng.uniform(), y0 + H * rng.uniform()
        r1 = np.zeros((H, W))
        mix.c_gauss_2d_grid(x0, x0 + W, y0, y0 + H, fx, fy, amp, mean, var, r1)
        assert np.array_equal(r1, oracle.mog_grid(x0, x0 + W, y0, y0 + H, fx, fy, amp, mean, var))
        minval = 10 ** rng.uniform(-6, -2)
        xc, yc = int(fx + rng.integers(-15, 15)), int(fy + rng.integers(-15, 15))
        r2 = np.zeros((H, W))
        dx = np.zeros_like(r2)
        dy = np.zeros_like(r2)
        rt = mix.c_gauss_2d_approx3(x0, x0 + W, y0, y0 + H, fx, fy, minval, amp, mean, var, r2, dx,
                                    dy, xc, yc, 3)
        o, ox, oy, bb = oracle.mog_approx3(x0, x0 + W, y0, y0 + H, fx, fy, minval, amp, mean, var,
                                           xc, yc, 3, derivs=True)
        assert np.array_equal(r2, o) and np.array_equal(dx, ox) and np.array_equal(dy, oy)
        assert tuple(rt[1:]) == tuple(bb)
        n = rng.uniform(0.25, 6.5)
        m = SersicMixture.getProfile(n)
        a, v = oracle.sersic_profile(n)
        assert np.array_equal(m.amp, a) and np.array_equal(m.var[:, 0, 0], v)


def _em_case(g, i):
    """Inputs of golden EM case i after fromStamp's preprocessing
    (tractor/psf.py:549-591)."""
    N, alpha, steps, hasxy, x0, y0, hasp0 = g['cfg%d' % i]
    N, steps = int(N), int(steps)
    st = g['stamp%d' % i].copy()
    st /= st.sum()
    st = np.maximum(st, 0)
    if hasp0:
        w, mu, var = g['p0amp%d' % i].copy(), g['p0mean%d' % i].copy(), g['p0var%d' % i].copy()
    else:
        w = np.ones(N) / N
        mu = np.zeros((N, 2))
        var = np.array([np.eye(2) * (k + 1) for k in range(N)])
    ny, nx = st.shape
    xy = (int(x0), int(y0)) if hasxy else (-(nx // 2), -(ny // 2))
    return st, N, float(alpha), steps, xy, (w, mu, var), bool(hasxy), bool(hasp0)


def test_em_fit_matches_golden(oracle):
    """The oracle's em_fit_2d_reg against GaussianMixturePSF.fromStamp run by
    the reference (emfit.npz): 7 stamps, 1-4 components, prior, origins, P0."""
    g = _golden('emfit.npz')
    for i in range(int(g['n'])):
        st, N, alpha, steps, (xm, ym), (w, mu, var), _, _ = _em_case(g, i)
        assert oracle.em_fit_2d_reg(st, xm, ym, w, mu, var, alpha, steps) == 0
        np.testing.assert_allclose(w, g['amp%d' % i], rtol=1e-11, atol=1e-14)
        np.testing.assert_allclose(mu, g['mean%d' % i], rtol=0, atol=1e-11)
        np.testing.assert_allclose(var, g['var%d' % i], rtol=1e-11, atol=1e-13)


def test_em_fit_failure_leaves_parameters(oracle):
    """A non-positive covariance determinant returns -1 before any update
    (tractor/emfit.i:403-409)."""
    st = np.ones((9, 9)) / 81.
    w, mu = np.array([1.]), np.zeros((1, 2))
    var = np.array([[[1., 2.], [2., 1.]]])
    assert oracle.em_fit_2d_reg(st, -4, -4, w, mu, var, 0., 10) == -1
    assert w[0] == 1. and not mu.any() and var[0, 0, 1] == 2.


@pytest.mark.reference
def test_em_oracle_matches_live_reference(oracle):
    from oracle import refharness
    if not refharness.available():
        pytest.skip('reference source tree not present')
    refharness.load()
    from tractor import emfit
    rng = np.random.default_rng(11)
    for trial in range(6):
        K = int(rng.integers(1, 5))
        h, w_ = int(rng.integers(9, 30)), int(rng.integers(9, 30))
        y, x = np.mgrid[:h, :w_]
        img = np.exp(-0.5 * ((x - w_ / 2.) ** 2 + (y - h / 2.) ** 2) / rng.uniform(1, 9))
        img = np.maximum(img / img.sum() + rng.normal(0, 1e-4, img.shape), 0)
        amp = np.ones(K) / K
        mean = rng.normal(0, 0.5, (K, 2))
        var = np.array([np.eye(2) * (k + 1) for k in range(K)])
        alpha = float(rng.choice([0., 0.3]))
        a2, m2, v2 = amp.copy(), mean.copy(), var.copy()
        r1 = emfit.em_fit_2d_reg(img, -(w_ // 2), -(h // 2), amp, mean, var, alpha, 200)
        r2 = oracle.em_fit_2d_reg(img, -(w_ // 2), -(h // 2), a2, m2, v2, alpha, 200)
        assert r1 == r2 == 0
        np.testing.assert_allclose(a2, amp, rtol=1e-11, atol=1e-14)
        np.testing.assert_allclose(m2, mean, rtol=0, atol=1e-10)
        np.testing.assert_allclose(v2, var, rtol=1e-11, atol=1e-13)


def test_em_sky_oracle_matches_golden(oracle):
    """The oracle's em_fit_2d_reg2 (EM with a flat sky term, emfit2.c)
    against GaussianMixturePSF.fromStamp(v2=True) run by the reference
    (emfit_sky.npz): the mixtures and the sky level."""
    from tractor_b200.emfit import em_init_params
    g = _golden('emfit_sky.npz')
    for i in range(int(g['n'])):
        N, alpha, steps, approx, hasxy, x0, y0 = g['cfg%d' % i]
        st = g['stamp%d' % i]
        h, w_ = st.shape
        xm, ym = (int(x0), int(y0)) if hasxy else (-(w_ // 2), -(h // 2))
        w, mu, var = em_init_params(int(N), None, None, None)
        r, sky = oracle.em_fit_2d_reg2(st, xm, ym, w, mu, var, float(alpha), int(steps),
                                       float(approx))
        assert r == 0
        np.testing.assert_allclose(w, g['amp%d' % i], rtol=1e-11)
        np.testing.assert_allclose(mu, g['mean%d' % i], rtol=0, atol=1e-11)
        np.testing.assert_allclose(var, g['var%d' % i], rtol=1e-11)
        assert abs(sky - float(g['sky%d' % i])) <= 1e-11 * abs(float(g['sky%d' % i]))
