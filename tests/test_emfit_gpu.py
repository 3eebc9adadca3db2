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
