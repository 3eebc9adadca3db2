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
