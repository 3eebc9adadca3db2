"""Batched Fourier-path rendering (the benchmark workload) against the oracle
and against golden patches produced by the reference itself
(tests/golden/fft_sersic.npz, tests/golden/make_golden.py).

Tolerance: model pixels within 1e-5 of the patch peak."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
PEAK_TOL = 1e-5


def _srcs_random(rng, n):
    from tractor_b200 import batch, _lib
    srcs = batch.sersic_sources(n, rng, mask=128)
    srcs['profile'] = rng.integers(0, 4, n)
    srcs['shape_type'] = rng.integers(0, 3, n)
    st = srcs['shape_type']
    # GalaxyShape (re, ab, phi) and EllipseESoft (log re, ee1, ee2) parameters
    srcs['s1'][st == _lib.SHAPE_RABPHI] = rng.uniform(0.2, 1, np.sum(st == _lib.SHAPE_RABPHI))
    srcs['s2'][st == _lib.SHAPE_RABPHI] = rng.uniform(0, 180, np.sum(st == _lib.SHAPE_RABPHI))
    srcs['s0'][st == _lib.SHAPE_ELLIPSE_ESOFT] = np.log(srcs['s0'][st == _lib.SHAPE_ELLIPSE_ESOFT])
    return srcs


def _oracle_source(O, s):
    """(amp, var2x2, K) of a GALAXY_SRC record through the oracle."""
    from tractor_b200 import _lib
    if s['profile'] == _lib.PROFILE_SERSIC:
        amp, var = O.sersic_profile(float(s['sersic_n']))
    elif s['profile'] == _lib.PROFILE_EXP:
        amp, var = O.exp_profile()
    elif s['profile'] == _lib.PROFILE_DEV:
        amp, var = O.dev_profile()
    else:
        amp, var = np.array([1.]), np.array([1.])
    if s['shape_type'] == _lib.SHAPE_RABPHI:
        G = O.galaxyshape_basis(s['s0'], s['s1'], s['s2'])
    elif s['shape_type'] == _lib.SHAPE_ELLIPSE_ESOFT:
        G = O.ellipseE_basis(*O.ellipseESoft_to_E(s['s0'], s['s1'], s['s2']))
    else:
        G = O.ellipseE_basis(s['s0'], s['s1'], s['s2'])
    T = O.nullwcs_cdinv() @ G
    return O.sheared(amp, var, T)


def test_prep_and_render_match_oracle(tb, oracle):
    import torch
    from tractor_b200 import batch, _lib
    rng = np.random.default_rng(11)
    srcs = _srcs_random(rng, 48)
    psf = batch.moffat_psf()
    r = batch.FourierGalaxyRenderer(psf)
    out, flags = r.render(srcs)
    assert np.all(flags == 0)
    out = out.numpy()
    items = r._work(len(srcs))[0].cpu().numpy().view(_lib.FFT_ITEM)
    camp = r._work(len(srcs))[1].cpu().numpy()
    cvar = r._work(len(srcs))[2].cpu().numpy()
    for i, s in enumerate(srcs):
        a2, v2 = _oracle_source(oracle, s)
        it = items[i]
        K = len(a2)
        assert it['K'] == K
        np.testing.assert_allclose(camp[it['c0']:it['c0'] + K], a2, rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(cvar[4 * it['c0']:4 * (it['c0'] + K)].reshape(K, 2, 2), v2,
                                   rtol=1e-10, atol=1e-14)
        ref, (mux, muy, sx, sy, sz) = oracle.galaxy_fft_masked(a2, v2, s['px'], s['py'], psf, 0, 0,
                                                               128, 128)
        assert (it['sz'], it['sx'], it['sy']) == (sz, sx, sy)
        assert abs(it['mux'] - mux) < 1e-12 and abs(it['muy'] - muy) < 1e-12
        got = out[s['out_off']:s['out_off'] + 128 * 128].reshape(128, 128) / s['counts']
        assert np.abs(got - ref).max() / ref.max() < PEAK_TOL, i


def test_renderer_matches_reference_golden(tb):
    """Patches of the reference's own SersicGalaxy.getModelPatch through its
    PixelizedPSF Fourier path (flux 1000, 128x128 ModelMask)."""
    from tractor_b200 import batch, _lib
    g = np.load(os.path.join(GOLDEN, 'fft_sersic.npz'))
    P = g['params']
    srcs = np.zeros(len(P), _lib.GALAXY_SRC)
    srcs['sersic_n'] = P[:, 0]
    srcs['px'] = P[:, 4]
    srcs['py'] = P[:, 5]
    srcs['s0'], srcs['s1'], srcs['s2'] = P[:, 6], P[:, 7], P[:, 8]
    srcs['counts'] = 1000.
    srcs['profile'] = _lib.PROFILE_SERSIC
    srcs['shape_type'] = _lib.SHAPE_ELLIPSE_E
    srcs['mw'] = srcs['mh'] = 128
    srcs['out_off'] = np.arange(len(P)) * 128 * 128
    r = batch.FourierGalaxyRenderer(g['psf'])
    out, flags = r.render(srcs)
    out = out.numpy()
    for i in range(len(P)):
        ref = g['patches'][i]
        got = out[i * 128 * 128:(i + 1) * 128 * 128].reshape(128, 128)
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err < PEAK_TOL, (i, err)


def test_full_workload_properties(tb, oracle):
    """All 256 sources of the benchmark workload: every patch finite, flux
    inside the mask <= total, a sampled subset equal to the oracle."""
    from tractor_b200 import batch
    rng = np.random.default_rng(1000)
    srcs = batch.sersic_sources(256, rng, mask=128)
    psf = batch.moffat_psf()
    r = batch.FourierGalaxyRenderer(psf)
    out, flags = r.render(srcs)
    out = out.numpy().reshape(256, 128, 128)
    assert np.all(flags == 0) and np.all(np.isfinite(out))
    sums = out.sum(axis=(1, 2))
    assert np.all(sums <= srcs['counts'] * (1 + 1e-4)) and np.all(sums > 0.5 * srcs['counts'])
    for i in range(0, 256, 37):
        s = srcs[i]
        a2, v2 = _oracle_source(oracle, s)
        ref, _ = oracle.galaxy_fft_masked(a2, v2, s['px'], s['py'], psf, 0, 0, 128, 128)
        assert np.abs(out[i] / s['counts'] - ref).max() / ref.max() < PEAK_TOL
