"""Fourier-path galaxies whose FFT size exceeds 256 (half-size above 128 px:
tractor/galaxy.py:336-519 goes on to sizes of 8192): the object API's
getModelPatch / getParamDerivatives through the large-size path
(tb_fourier_spectrum_grid, the inverse real FFT, tb_lanczos3_shift, crop)
against the oracle's restatement of the reference's FFT branch.

Tolerances as for the other sizes: model pixels within 1e-5 of the patch
peak, the shape and Sersic-index columns within 1e-4 of their peak against
the exact FP64 forward differences."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PEAK_TOL = 1e-5
DERIV_TOL = 1e-4


def _check(p, x0, y0, ref, tol, what):
    assert p is not None and p.patch is not None, what
    assert (p.x0, p.y0) == (x0, y0), (what, (p.x0, p.y0), (x0, y0))
    assert p.patch.shape == ref.shape, (what, p.patch.shape, ref.shape)
    err = np.abs(p.patch - ref).max() / np.abs(ref).max()
    assert err < tol, (what, err)


@pytest.mark.parametrize('case', [
    # profile, Sersic n, (re, e1, e2), (px, py), ModelMask (x0, y0, w, h), FFT size
    ('sersic', 2.5, (12., 0.2, -0.1), (170.3, 160.6), (20, 10, 300, 310), 512),
    ('exp', None, (30., -0.3, 0.1), (311.7, 298.2), (0, 0, 620, 600), 1024),
    ('dev', None, (8., 0.1, 0.4), (150., 150.), (0, 0, 300, 300), 512),   # no sub-pixel shift
    ('sersic', 4.0, (5., -0.2, 0.3), (140.2, 352.9), (0, 100, 280, 520), 1024),  # off-centre
])
def test_large_fft_galaxy_matches_oracle(tb, oracle, case):
    import tractor_b200 as T
    from tractor_b200 import batch
    kind, n, (re, e1, e2), (px, py), (mx0, my0, mw, mh), want_sz = case
    psf_img = batch.moffat_psf()
    psf = T.PixelizedPSF(psf_img)
    pos, br, shape = T.PixPos(px, py), T.Flux(1000.), T.EllipseE(re, e1, e2)
    if kind == 'sersic':
        gal = T.SersicGalaxy(pos, br, shape, T.SersicIndex(n))
        amp, var = oracle.sersic_profile(n)
    elif kind == 'exp':
        gal = T.ExpGalaxy(pos, br, shape)
        amp, var = oracle.exp_profile()
    else:
        gal = T.DevGalaxy(pos, br, shape)
        amp, var = oracle.dev_profile()
    H, W = my0 + mh + 8, mx0 + mw + 8
    tim = T.Image(data=np.zeros((H, W), np.float32), inverr=np.ones((H, W), np.float32),
                  psf=psf, photocal=T.LinearPhotoCal(1.))
    mm = T.ModelMask(mx0, my0, mw, mh)
    p = gal.getModelPatch(tim, modelMask=mm)
    Tm = oracle.nullwcs_cdinv() @ oracle.ellipseE_basis(re, e1, e2)
    a2, v2 = oracle.sheared(amp, var, Tm)
    ref, (mux, muy, sx, sy, sz) = oracle.galaxy_fft_masked(a2, v2, px, py, psf_img, mx0, my0,
                                                           mw, mh)
    assert sz == want_sz
    _check(p, mx0, my0, 1000. * ref, PEAK_TOL, '%s %d' % (kind, sz))
    if kind == 'sersic' and sz == 512:
        # the shape and Sersic-index columns (difference items of the
        # large-size path) against FP64 forward differences of step 0.01
        d = gal.getParamDerivatives(tim, modelMask=mm)
        th = [px, py, 1000., re, e1, e2, n]
        base = oracle.sersic_fft_model_f64(th, psf_img, mx0, my0, mw, mh)
        for j in (3, 4, 5, 6):
            th2 = list(th)
            th2[j] += 0.01
            exact = (oracle.sersic_fft_model_f64(th2, psf_img, mx0, my0, mw, mh) - base) / 0.01
            _check(d[j], mx0, my0, exact, DERIV_TOL, 'column %d at size %d' % (j, sz))


def test_large_psf_spectrum_matches_numpy(tb):
    """The PSF spectrum above size 256 (FP64 cuFFT, rounded to complex64, in
    the column-major layout the renderers read) equals np.fft.rfft2 of the
    padded PSF (PixelizedPSF.getFourierTransform, tractor/psf.py:249-280)."""
    from tractor_b200 import batch, render
    img = batch.moffat_psf()
    for sz in (512, 2048):
        spec, cx, cy = render.psf_spectra().compute(img, sz)
        got = spec.cpu().numpy().view(np.complex64).reshape(sz // 2 + 1, sz).T
        pad, cx2, cy2 = render.PsfSpectra.pad(img, sz)
        ref = np.fft.rfft2(pad.astype(np.float64))
        assert (cx, cy) == (cx2, cy2)
        assert np.abs(got - ref).max() < 1e-6 * np.abs(ref).max()
