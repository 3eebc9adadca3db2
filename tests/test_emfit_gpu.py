"""The EM kernel (tb_em_fit_2d) against the oracle's em_fit_2d_reg (pinned
to the reference's own emfit.i): every component count the kernel is
specialised for (1-8), non-square stamps, explicit origins, the alpha
prior, and one launch over many stamps equal to one launch per stamp."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _stamp(rng, h, w, K):
    y, x = np.mgrid[:h, :w]
    img = np.zeros((h, w))
    for k in range(K):
        s = rng.uniform(0.8, 4.0)
        cx, cy = w / 2. + rng.normal(0, 0.7), h / 2. + rng.normal(0, 0.7)
        img += rng.uniform(0.2, 1.) * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * s * s))
    img = img / img.sum() + rng.normal(0, 1e-5, img.shape)
    return np.maximum(img / img.sum(), 0)


def test_em_all_component_counts_match_oracle(tb, oracle):
    from tractor_b200 import emfit
    rng = np.random.default_rng(21)
    for K in range(1, 9):
        h, w = int(rng.integers(15, 34)), int(rng.integers(15, 34))
        img = _stamp(rng, h, w, min(K, 4))
        amp, mean, var = emfit.em_init_params(K, None, None, None)
        mean = mean + rng.normal(0, 0.3, mean.shape)
        alpha = 0.2 if K % 2 else 0.
        x0, y0 = -(w // 2) + int(rng.integers(-2, 3)), -(h // 2) + int(rng.integers(-2, 3))
        a1, m1, v1 = amp.copy(), mean.copy(), var.copy()
        a2, m2, v2 = amp.copy(), mean.copy(), var.copy()
        r1 = emfit.em_fit_2d_reg(img, x0, y0, a1, m1, v1, alpha, 150)
        r2 = oracle.em_fit_2d_reg(img, x0, y0, a2, m2, v2, alpha, 150)
        assert r1 == r2
        if r2 == 0:
            np.testing.assert_allclose(a1, a2, rtol=1e-9, atol=1e-13, err_msg='K=%d' % K)
            np.testing.assert_allclose(m1, m2, rtol=0, atol=1e-9, err_msg='K=%d' % K)
            np.testing.assert_allclose(v1, v2, rtol=1e-9, atol=1e-12, err_msg='K=%d' % K)


def test_em_batch_equals_single_launches(tb):
    from tractor_b200 import emfit
    rng = np.random.default_rng(5)
    imgs = np.stack([_stamp(rng, 21, 27, 3) for _ in range(40)])
    amp, mean, var = emfit.em_init_params(3, None, None, None)
    n = len(imgs)
    a, m, v, st = emfit.em_fit_2d_batch(imgs, np.tile(amp, (n, 1)), np.tile(mean, (n, 1, 1)),
                                        np.tile(var, (n, 1, 1, 1)), 0.1, 120, xy0=(-13, -10))
    assert not st.any()
    for i in (0, 17, 39):
        a1, m1, v1 = amp.copy(), mean.copy(), var.copy()
        assert emfit.em_fit_2d_reg(imgs[i], -13, -10, a1, m1, v1, 0.1, 120) == 0
        assert np.array_equal(a[i], a1) and np.array_equal(m[i], m1) and np.array_equal(v[i], v1)


def _sky_case(g, i):
    cfg = g['cfg%d' % i]
    N, alpha, steps, approx, hasxy, x0, y0 = cfg
    st = g['stamp%d' % i]
    h, w = st.shape
    xy = (int(x0), int(y0)) if hasxy else None
    return st, int(N), float(alpha), int(steps), float(approx), xy


def test_em_sky_fit_matches_reference_golden(tb):
    """GaussianMixturePSF.fromStamp(v2=True) -- the EM fit with a flat sky
    term (tb_em_fit_2d_sky, emfit2.c) -- against the reference's own fits
    (tests/golden/emfit_sky.npz: backgrounds and noise with pixels at or
    below zero, 1-3 components, the prior, two approx cuts, an explicit
    origin): the mixture and the returned sky level."""
    import os
    import tractor_b200 as T
    g = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'emfit_sky.npz'))
    for i in range(int(g['n'])):
        st, N, alpha, steps, approx, xy = _sky_case(g, i)
        psf, sky = T.GaussianMixturePSF.fromStamp(st, N=N, xy0=xy, alpha=alpha, emsteps=steps,
                                                  v2=True, approx=approx)
        np.testing.assert_allclose(psf.mog.amp, g['amp%d' % i], rtol=1e-9, err_msg=str(i))
        np.testing.assert_allclose(psf.mog.mean, g['mean%d' % i], rtol=0, atol=1e-9,
                                   err_msg=str(i))
        np.testing.assert_allclose(psf.mog.var, g['var%d' % i], rtol=1e-9, err_msg=str(i))
        assert abs(sky - float(g['sky%d' % i])) <= 1e-9 * abs(float(g['sky%d' % i])), (i, sky)


def test_em_sky_all_component_counts_match_oracle(tb, oracle):
    """tb_em_fit_2d_sky for every component count (1-8) against the oracle's
    em_fit_2d_reg2 (pinned to the reference), stamps with a background and
    negative noise pixels, and one launch over many stamps equal to one
    launch per stamp."""
    from tractor_b200 import emfit
    rng = np.random.default_rng(23)
    for K in range(1, 9):
        h, w = int(rng.integers(15, 30)), int(rng.integers(15, 30))
        img = _stamp(rng, h, w, min(K, 4)) * 500. + 0.05 + rng.normal(0, 0.03, (h, w))
        amp, mean, var = emfit.em_init_params(K, None, None, None)
        mean = mean + rng.normal(0, 0.3, mean.shape)
        alpha = 0.2 if K % 2 else 0.
        a1, m1, v1 = amp.copy(), mean.copy(), var.copy()
        a2, m2, v2 = amp.copy(), mean.copy(), var.copy()
        r1, s1 = emfit.em_fit_2d_reg2(img, -(w // 2), -(h // 2), a1, m1, v1, alpha, 120, 1e-30)
        r2, s2 = oracle.em_fit_2d_reg2(img, -(w // 2), -(h // 2), a2, m2, v2, alpha, 120, 1e-30)
        assert r1 == r2
        if r2 == 0:
            np.testing.assert_allclose(a1, a2, rtol=1e-9, err_msg='K=%d' % K)
            np.testing.assert_allclose(m1, m2, rtol=0, atol=1e-9, err_msg='K=%d' % K)
            np.testing.assert_allclose(v1, v2, rtol=1e-9, err_msg='K=%d' % K)
            assert abs(s1 - s2) <= 1e-9 * abs(s2), (K, s1, s2)
    imgs = np.stack([_stamp(rng, 21, 23, 2) * 300. + 0.02 + rng.normal(0, 0.02, (21, 23))
                     for _ in range(24)])
    amp, mean, var = emfit.em_init_params(2, None, None, None)
    n = len(imgs)
    a, m, v, sky, st = emfit.em_fit_2d_reg2_batch(imgs, np.tile(amp, (n, 1)),
                                                  np.tile(mean, (n, 1, 1)),
                                                  np.tile(var, (n, 1, 1, 1)), 0.1, 80, 1e-30)
    assert not st.any()
    for i in (0, 11, 23):
        a1, m1, v1 = amp.copy(), mean.copy(), var.copy()
        r, s1 = emfit.em_fit_2d_reg2(imgs[i], -11, -10, a1, m1, v1, 0.1, 80, 1e-30)
        assert r == 0 and s1 == sky[i]
        assert np.array_equal(a[i], a1) and np.array_equal(m[i], m1) and np.array_equal(v[i], v1)
