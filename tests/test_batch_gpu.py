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
    # the two-launch path leaves the component tables in device memory
    out, flags = r.render(srcs, method='persistent')
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


def test_fused_equals_two_launch_path(tb):
    """tb_galaxy_fft_render (preparation and render in one launch) gives the
    two-launch path's patches bit for bit (the same FP64 products become the
    same FP32 coefficients) and its flags and items: the benchmark's 256
    sources, random profiles and shape types, masks of other sizes (FFT 64 /
    128 / 256), zero counts and a source far outside its mask (no patch),
    one outside its mask within its radius and one whose FFT size would
    exceed 256 (unsupported: zero patches and flag 2)."""
    import numpy as np
    from tractor_b200 import batch, _lib
    rng = np.random.default_rng(29)
    a = batch.sersic_sources(256, rng, mask=128)
    b = _srcs_random(rng, 64)
    srcs = np.concatenate([a, b])
    n = len(srcs)
    sizes = rng.choice([24, 48, 96, 128], n)
    sizes[:256] = 128
    srcs['mw'] = sizes
    srcs['mh'] = np.where(rng.random(n) < 0.8, sizes, np.maximum(sizes // 2, 8))
    srcs['px'] = srcs['mw'] / 2.0 + rng.uniform(-3, 3, n)
    srcs['py'] = srcs['mh'] / 2.0 + rng.uniform(-3, 3, n)
    srcs['counts'][300] = 0.                                  # no patch
    srcs['px'][301], srcs['py'][301] = -500., -500.           # far outside: no patch
    srcs['px'][302] = -2.                                     # just outside: unsupported
    srcs['mw'][303] = srcs['mh'][303] = 300                   # FFT 512: unsupported
    srcs['px'][303], srcs['py'][303] = 150., 150.
    srcs['out_off'] = np.concatenate([[0], np.cumsum(srcs['mw'].astype(np.int64) *
                                                     srcs['mh'])[:-1]])
    r = batch.FourierGalaxyRenderer(batch.moffat_psf())
    got, f1 = r.render(srcs, method='fused')
    got = got.numpy().copy()
    it1 = r._work(n)[0].cpu().numpy().view(_lib.FFT_ITEM).copy()
    want, f2 = r.render(srcs, method='persistent')
    want = want.numpy().copy()
    it2 = r._work(n)[0].cpu().numpy().view(_lib.FFT_ITEM).copy()
    assert np.array_equal(f1, f2)
    assert f1[300] == 1 and f1[301] == 1 and f1[302] == 2 and f1[303] == 2
    assert np.sum(f1 == 0) == n - 4
    for k in it1.dtype.names:
        if k != 'c0':
            assert np.array_equal(it1[k], it2[k]), k
    assert np.all(np.isfinite(got))
    assert np.array_equal(got, want)
