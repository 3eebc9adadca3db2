"""Generates the golden fixtures in tests/golden/ by running the reference
Tractor itself (imported from its source tree through oracle/refharness.py,
with its own C kernels compiled by oracle/build_ref.sh).

Each fixture stores the scenario's inputs and the reference's outputs, so the
oracle and the CUDA path can be checked against the reference without the
reference being present.  All scenarios are seeded.  Run from the repository
root in the development container:

    python tests/golden/make_golden.py          # every fixture but hybrid_psf
    python tests/golden/make_golden.py hybrid   # hybrid_psf.npz
    python tests/golden/make_golden.py psfex    # psfex.npz
    python tests/golden/make_golden.py emfit    # emfit.npz
    python tests/golden/make_golden.py emfitsky # emfit_sky.npz
    python tests/golden/make_golden.py psfderiv # psf_derivs.npz
    python tests/golden/make_golden.py forcedsky # forced_sky.npz
    python tests/golden/make_golden.py varying  # varying_psf.npz
    python tests/golden/make_golden.py composite # composite.npz
    python tests/golden/make_golden.py fittight # fit_plain_tight.npz
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
OUT = os.path.dirname(os.path.abspath(__file__))


def moffat(size=63, fwhm=4.0, beta=3.0):
    alpha = fwhm / (2 * np.sqrt(2 ** (1 / beta) - 1))
    y, x = np.mgrid[:size, :size] - size // 2
    img = (1 + (x ** 2 + y ** 2) / alpha ** 2) ** (-beta)
    return (img / img.sum()).astype(np.float32)


def patches_to_arrays(plist):
    """[Patch|None] -> (present flags, x0s, y0s, shapes, concatenated pixels)."""
    present, x0, y0, hh, ww, pix = [], [], [], [], [], []
    for p in plist:
        if p is None or p.patch is None:
            present.append(0)
            x0.append(0)
            y0.append(0)
            hh.append(0)
            ww.append(0)
            continue
        present.append(1)
        x0.append(p.x0)
        y0.append(p.y0)
        hh.append(p.patch.shape[0])
        ww.append(p.patch.shape[1])
        pix.append(np.asarray(p.patch, np.float64).ravel())
    return dict(present=np.array(present), x0=np.array(x0), y0=np.array(y0), h=np.array(hh),
                w=np.array(ww), pix=np.concatenate(pix) if pix else np.zeros(0))


def main():
    from oracle import refharness
    t = refharness.load()
    from tractor import (Image, PixPos, Flux, NanoMaggies, LinearPhotoCal, GaussianMixturePSF,
                         NCircularGaussianPSF, PixelizedPSF, PointSource, Tractor, EllipseE,
                         EllipseESoft)
    from tractor.galaxy import ExpGalaxy, DevGalaxy, GalaxyShape, FixedCompositeGalaxy
    from tractor.sersic import SersicGalaxy, SersicIndex
    from tractor.patch import ModelMask
    from tractor import mp_fourier, mix

    # -- 1. kernel-level vectors -------------------------------------------
    rng = np.random.default_rng(100)
    K = 7
    amp = rng.uniform(0.1, 1, K)
    mean = rng.normal(size=(K, 2))
    var = np.zeros((K, 2, 2))
    for k in range(K):
        a = rng.normal(size=(2, 2))
        var[k] = a @ a.T + 0.4 * np.eye(2)
    grid = np.zeros((24, 31))
    mix.c_gauss_2d_grid(-5, 26, 3, 27, 7.3, 11.6, amp, mean, var, grid)
    ap = np.zeros((40, 44))
    axd = np.zeros_like(ap)
    ayd = np.zeros_like(ap)
    rtn, sx0, sx1, sy0, sy1 = mix.c_gauss_2d_approx3(0, 44, 0, 40, 20.4, 18.7, 1e-4, amp, mean,
                                                     var, ap, axd, ayd, 20, 18, 3)
    img = rng.normal(size=(33, 41)).astype(np.float32)
    lz = np.zeros_like(img)
    work = np.zeros((4096, 4096), np.float32)
    mp_fourier.lanczos_shift_3f(img, lz, 0.37, -0.21, work)
    v = np.fft.rfftfreq(32)
    w = np.fft.fftfreq(32)
    var2 = var.copy()
    var2[0] = 0.
    ft = np.zeros((32, 17))
    mp_fourier.gaussian_fourier_transform_zero_mean(amp, var2, v, w, ft)
    np.savez_compressed(os.path.join(OUT, 'kernels.npz'), amp=amp, mean=mean, var=var, var2=var2,
                        grid=grid, approx=ap, approx_dx=axd, approx_dy=ayd,
                        approx_bbox=np.array([sx0, sx1, sy0, sy1]), lanczos_in=img,
                        lanczos_out=lz, fourier=ft)

    # -- 2. MoG galaxies and point sources (exact grid, masks, approx3) ------
    out = {}
    psf = GaussianMixturePSF(1., 0., 0., 6., 6., -1.)
    H, W = 100, 100
    tim = Image(data=np.zeros((H, W), np.float32), inverr=np.ones((H, W), np.float32), psf=psf,
                photocal=LinearPhotoCal(1.))
    srcs = [
        ExpGalaxy(PixPos(49.5, 50.), Flux(100.), GalaxyShape(2., 0.5, 45.)),
        DevGalaxy(PixPos(40.2, 61.7), Flux(250.), EllipseE(3.0, 0.2, -0.1)),
        FixedCompositeGalaxy(PixPos(55.5, 45.3), Flux(500.), 0.3, EllipseE(2.0, -0.1, 0.3),
                             EllipseE(1.5, 0.05, 0.1)),
        SersicGalaxy(PixPos(50.3, 49.8), Flux(300.), EllipseE(2.5, 0.3, 0.1), SersicIndex(2.2)),
        PointSource(PixPos(30.6, 70.1), Flux(80.)),
    ]
    names = ['exp', 'dev', 'comp', 'sersic', 'ptsrc']
    mm = ModelMask(20, 25, 60, 55)
    for name, s in zip(names, srcs):
        p = s.getModelPatch(tim)
        out[name + '_nomask'] = patches_to_arrays([p])
        p = s.getModelPatch(tim, modelMask=mm)
        out[name + '_mask'] = patches_to_arrays([p])
        d = s.getParamDerivatives(tim, modelMask=mm)
        out[name + '_derivs_mask'] = patches_to_arrays(d)
        d = s.getParamDerivatives(tim)
        out[name + '_derivs_nomask'] = patches_to_arrays(d)
    tim.modelMinval = 0.01
    for name, s in zip(names, srcs):
        p = s.getModelPatch(tim)
        out[name + '_minval'] = patches_to_arrays([p])
    tim.modelMinval = 0.
    ncirc = NCircularGaussianPSF([1.5, 3.0], [0.8, 0.2])
    tim2 = Image(data=np.zeros((64, 64), np.float32), inverr=np.ones((64, 64), np.float32),
                 psf=ncirc, photocal=LinearPhotoCal(1.))
    for name, s in zip(names, srcs):
        s2 = s.copy()
        s2.pos.x = s.pos.x - 18
        s2.pos.y = s.pos.y - 18
        p = s2.getModelPatch(tim2)
        out[name + '_ncirc'] = patches_to_arrays([p])
    flat = {}
    for k, dct in out.items():
        for kk, vv in dct.items():
            flat[k + '.' + kk] = vv
    np.savez_compressed(os.path.join(OUT, 'mog_sources.npz'), **flat)

    # -- 3. Fourier path: Sersic galaxies, 63x63 Moffat PixelizedPSF --------
    rng = np.random.default_rng(200)
    mof = moffat()
    ppsf = PixelizedPSF(mof)
    rows = []
    pix = []
    derivs = []
    for i in range(6):
        n = [0.8, 1.7, 3.5, 5.5, 0.45, 1.2][i]
        re = float(np.exp(rng.uniform(np.log(0.5), np.log(8))))
        q = float(rng.uniform(0.2, 1))
        phi = float(rng.uniform(0, 180))
        dx, dy = rng.uniform(-0.5, 0.5, 2)
        px, py = 64 + dx, 64 + dy
        ell = EllipseE.fromRAbPhi(re, q, phi)
        gal = SersicGalaxy(PixPos(px, py), Flux(1000.), ell, SersicIndex(n))
        tim3 = Image(data=np.zeros((128, 128), np.float32), inverr=np.ones((128, 128), np.float32),
                     psf=ppsf, photocal=LinearPhotoCal(1.))
        mask = ModelMask(0, 0, 128, 128)
        p = gal.getModelPatch(tim3, modelMask=mask)
        rows.append([n, re, q, phi, px, py, ell.re, ell.e1, ell.e2])
        pix.append(p.patch.astype(np.float32))
        if i < 2:
            mask64 = ModelMask(32, 32, 64, 64)
            d = gal.getParamDerivatives(tim3, modelMask=mask64)
            derivs.append(np.stack([dd.patch.astype(np.float32) for dd in d]))
    np.savez_compressed(os.path.join(OUT, 'fft_sersic.npz'), params=np.array(rows),
                        psf=mof, patches=np.stack(pix), derivs=np.stack(derivs))

    # -- 4. Plain small fit (ExpGalaxy on 64x64, 2-component MoG PSF) -------
    rng = np.random.default_rng(300)
    truth = ExpGalaxy(PixPos(32., 32.), Flux(1000.), EllipseE.fromRAbPhi(2.0, 0.6, 30.))
    timc = Image(data=np.zeros((64, 64)), invvar=np.ones((64, 64)),
                 psf=NCircularGaussianPSF([1.5, 3.0], [0.8, 0.2]), photocal=LinearPhotoCal(1.))
    trc = Tractor([timc], [truth])
    trc.modtype = np.float64
    clean = trc.getModelImage(0)
    noisy = clean + rng.normal(size=clean.shape)
    timc.data = noisy
    e0 = truth.shape
    start = ExpGalaxy(PixPos(32.5, 32.5), Flux(800.), EllipseE.fromRAbPhi(2.4, 0.6, 30.))
    tr = Tractor([timc], [start])
    tr.modtype = np.float64
    tr.freezeParam('images')
    lnp0 = tr.getLogProb()
    mod0 = tr.getModelImage(0)
    d0 = start.getParamDerivatives(timc)
    X = tr.optimizer.getLinearUpdateDirection(tr)
    p_before = np.array(tr.getParams())
    dlnp, X1, alpha = tr.optimize()
    p_after1 = np.array(tr.getParams())
    R = tr.optimize_loop(dchisq=1e-3)
    p_final = np.array(tr.getParams())
    np.savez_compressed(os.path.join(OUT, 'fit_plain.npz'), data=noisy, clean=clean, mod0=mod0,
                        lnp0=lnp0, X=np.array(X), p_before=p_before, dlnp1=dlnp, X1=np.array(X1),
                        alpha1=alpha, p_after1=p_after1, p_final=p_final, steps=R['steps'],
                        **dict(('d0.' + k, v) for k, v in patches_to_arrays(d0).items()))
    # -- 5. Batched-render scene: mixed sources with square model masks on one
    #       float32 image, 3-component MoG PSF, through Tractor.getModelImage --
    rng = np.random.default_rng(500)
    H, W = 256, 320
    s1 = rng.uniform(1., 2.)
    pamp = np.array([0.7, 0.2, 0.1])
    psig = np.array([s1, 2. * s1, 4. * s1])
    psf5 = GaussianMixturePSF(pamp, np.zeros((3, 2)),
                              np.array([np.eye(2) * s ** 2 for s in psig]))
    tim5 = Image(data=np.zeros((H, W), np.float32), inverr=np.ones((H, W), np.float32),
                 psf=psf5, photocal=LinearPhotoCal(1.))
    rows, srcs5, masks5 = [], [], {}
    for i in range(80):
        kind = rng.choice(4, p=[0.4, 0.3, 0.2, 0.1])
        px, py = rng.uniform(-5, W + 5), rng.uniform(-5, H + 5)
        flux = float(np.exp(rng.uniform(np.log(10.), np.log(1e5))))
        hw = int(np.round(np.exp(rng.uniform(np.log(7), np.log(60)))))
        shp = []
        for _ in range(2):
            re = float(np.exp(rng.uniform(np.log(0.5), np.log(8))))
            shp += [re, float(rng.uniform(0.2, 1)), float(rng.uniform(0, 180))]
        fdev = float(rng.uniform(0, 1))
        ea = EllipseE.fromRAbPhi(*shp[:3])
        eb = EllipseE.fromRAbPhi(*shp[3:])
        pos, br = PixPos(px, py), Flux(flux)
        if kind == 0:
            s = PointSource(pos, br)
        elif kind == 1:
            s = ExpGalaxy(pos, br, ea)
        elif kind == 2:
            s = DevGalaxy(pos, br, ea)
        else:
            s = FixedCompositeGalaxy(pos, br, fdev, ea, eb)
        # square mask centred on the nearest pixel, clipped to the image
        cx, cy = int(np.round(px)), int(np.round(py))
        mx0, mx1 = max(0, cx - hw), min(W, cx + hw + 1)
        my0, my1 = max(0, cy - hw), min(H, cy + hw + 1)
        if mx0 >= mx1 or my0 >= my1:
            continue
        masks5[s] = ModelMask(mx0, my0, mx1 - mx0, my1 - my0)
        srcs5.append(s)
        rows.append([kind, px, py, flux, mx0, my0, mx1 - mx0, my1 - my0, fdev,
                     ea.re, ea.e1, ea.e2, eb.re, eb.e1, eb.e2])
    tr5 = Tractor([tim5], srcs5)
    tr5.setModelMasks([masks5])
    mod5 = tr5.getModelImage(0)
    assert mod5.dtype == np.float32
    np.savez_compressed(os.path.join(OUT, 'scene_mog.npz'), sources=np.array(rows),
                        psf_amp=pamp, psf_sigma=psig, shape=np.array([H, W]), model=mod5)
    # -- 6. Forced photometry: 6 sources of fixed shape / position seen in
    #       two 64 x 72 images of one band (different PSFs and photometric
    #       scales), fluxes fitted, with variance -------------------------
    rng = np.random.default_rng(600)
    H6, W6 = 64, 72
    psf6 = [NCircularGaussianPSF([1.2, 2.6], [0.75, 0.25]),
            GaussianMixturePSF(np.array([0.6, 0.3, 0.1]), np.zeros((3, 2)),
                               np.array([np.eye(2) * s ** 2 for s in (1.5, 3.0, 6.0)]))]
    scales6 = [1.0, 2.5]
    rows6, srcs6 = [], []
    for i in range(6):
        kind = i % 3
        px, py = rng.uniform(8, W6 - 8), rng.uniform(8, H6 - 8)
        fl = rng.uniform(50., 500., 1)
        re = float(rng.uniform(1., 3.))
        e1, e2 = rng.uniform(-0.3, 0.3, 2)
        br = Flux(fl[0])
        if kind == 0:
            s = PointSource(PixPos(px, py), br)
        elif kind == 1:
            s = ExpGalaxy(PixPos(px, py), br, EllipseE(re, e1, e2))
        else:
            s = DevGalaxy(PixPos(px, py), br, EllipseE(re, e1, e2))
        rows6.append([kind, px, py, fl[0], re, e1, e2])
        srcs6.append(s)
    tims6 = []
    for b in range(2):
        tim = Image(data=np.zeros((H6, W6), np.float32), inverr=np.ones((H6, W6), np.float32),
                    psf=psf6[b], photocal=LinearPhotoCal(scales6[b]))
        tims6.append(tim)
    trt = Tractor(tims6, srcs6)
    trt.freezeParam('images')
    datas6 = []
    for b, tim in enumerate(tims6):
        clean = trt.getModelImage(b)
        tim.data = (clean + rng.normal(size=clean.shape) * 0.5).astype(np.float32)
        tim.inverr = np.full((H6, W6), 2., np.float32)
        datas6.append(tim.data.copy())
    # start from wrong fluxes, shapes and positions frozen
    for s in srcs6:
        s.freezeAllBut('brightness')
        s.brightness.setParams([v * 0.7 + 5. for v in s.brightness.getParams()])
    start6 = np.array(trt.getParams())
    R = trt.optimize_forced_photometry(variance=True, shared_params=False)
    np.savez_compressed(os.path.join(OUT, 'forced_phot.npz'), sources=np.array(rows6),
                        data=np.stack(datas6), scales=np.array(scales6), start=start6,
                        fluxes=np.array(trt.getParams()), IV=np.array(R.IV))
    print('golden fixtures written to', OUT)


def hybrid():
    """HybridPixelizedPSF (psf.py:600-655): galaxies rendered by the hybrid
    split of ProfileGalaxy._realGetUnitFluxModelPatch (galaxy.py:412-455,
    510-518) -- all-Fourier, ramped, all-MoG, a source outside its mask
    (MoG), no mask -- and a point source (the pixelized model)."""
    from oracle import refharness
    refharness.load()
    from tractor import (Image, PixPos, Flux, LinearPhotoCal, GaussianMixturePSF, PixelizedPSF,
                         PointSource, EllipseE)
    from tractor.psf import HybridPixelizedPSF
    from tractor.galaxy import ExpGalaxy, DevGalaxy
    from tractor.sersic import SersicGalaxy, SersicIndex
    from tractor.patch import ModelMask
    mof = moffat()
    gauss = dict(amp=np.array([0.8, 0.2]), mean=np.zeros((2, 2)),
                 var=np.array([[[2.0, 0.1], [0.1, 2.2]], [[9.0, 0.], [0., 9.0]]]))
    psf = HybridPixelizedPSF(PixelizedPSF(mof),
                             GaussianMixturePSF(gauss['amp'], gauss['mean'], gauss['var']))
    # kind 0 exp, 1 deV, 2 Sersic, 3 point source; px, py, r_e, b/a, phi, n;
    # mask (x0, y0, w, h), w = 0: none
    cases = [(0, 64.3, 63.8, 2.0, 0.7, 30., 1.0, (0, 0, 128, 128)),
             (0, 64.3, 63.8, 12.0, 0.7, 30., 1.0, (0, 0, 64 + 64, 128)),
             (0, 32.2, 31.6, 9.0, 0.8, 60., 1.0, (0, 0, 64, 64)),
             (1, 32.4, 32.3, 14.0, 0.6, 10., 1.0, (0, 0, 64, 64)),
             (2, 40.1, 36.9, 7.0, 0.5, 120., 3.0, (8, 4, 64, 64)),
             (0, -20.0, 40.0, 10.0, 0.9, 0., 1.0, (0, 0, 64, 64)),
             (0, 50.3, 49.6, 3.0, 0.6, 45., 1.0, (0, 0, 0, 0)),
             (0, 31.7, 32.5, 30.0, 0.8, 75., 1.0, (0, 0, 64, 64)),
             (2, 48.2, 47.7, 20.0, 0.7, 15., 1.5, (0, 0, 96, 96)),
             (3, 33.7, 30.2, 0.0, 1.0, 0., 1.0, (0, 0, 64, 64))]
    out = []
    for kind, px, py, re, ab, phi, n, mk in cases:
        pos, flux = PixPos(px, py), Flux(1000.)
        if kind == 3:
            src = PointSource(pos, flux)
        else:
            ell = EllipseE.fromRAbPhi(re, ab, phi)
            src = (ExpGalaxy(pos, flux, ell) if kind == 0 else DevGalaxy(pos, flux, ell)
                   if kind == 1 else SersicGalaxy(pos, flux, ell, SersicIndex(n)))
        tim = Image(data=np.zeros((100, 100), np.float32), inverr=np.ones((100, 100), np.float32),
                    psf=psf, photocal=LinearPhotoCal(1.))
        mm = ModelMask(*mk) if mk[2] > 0 else None
        out.append(src.getModelPatch(tim, modelMask=mm))
    table = np.array([list(c[:7]) + list(c[7]) for c in cases], np.float64)
    np.savez_compressed(os.path.join(OUT, 'hybrid_psf.npz'), cases=table,
                        psf=mof, gauss_amp=gauss['amp'], gauss_mean=gauss['mean'],
                        gauss_var=gauss['var'], **patches_to_arrays(out))
    print('hybrid fixture written to', OUT)


def psfex():
    """PixelizedPsfEx (psfex.py:428-521) built from a degree-2 model's arrays
    (no FITS file: attributes set as PsfExModel.shifted does): galaxies on the
    Fourier path with the position-dependent spectrum, point sources with the
    position-dependent image, at several positions, and one galaxy with a
    HybridPixelizedPSF around the PsfEx model."""
    from oracle import refharness
    refharness.load()
    from tractor import (Image, PixPos, Flux, LinearPhotoCal, GaussianMixturePSF, PointSource,
                         EllipseE)
    from tractor.psf import HybridPixelizedPSF
    from tractor.psfex import PsfExModel, PixelizedPsfEx
    from tractor.galaxy import ExpGalaxy
    from tractor.sersic import SersicGalaxy, SersicIndex
    from tractor.patch import ModelMask
    base = moffat(33, 4.0, 3.0)
    wide = moffat(33, 5.5, 2.5)
    y, x = np.mgrid[:33, :33] - 16
    bases = np.stack([base, 0.3 * (wide - base), 0.02 * x * base, 0.15 * (wide - base),
                      0.01 * x * y * base, 0.02 * y * base]).astype(np.float32)
    m = PsfExModel()
    m.sampling, m.psfbases, m.degree = 1., bases, 2
    m.x0, m.y0, m.xscale, m.yscale = 50., 40., 100., 80.
    m.radius, m.fwhm = (33 + 1) / 2., 4.0
    psf = PixelizedPsfEx(None, psfex=m)
    mc = m.copy()
    mc.fwhm = m.fwhm     # as PixelizedPsfEx.copy does (shifted() leaves it out)
    hyb = HybridPixelizedPSF(PixelizedPsfEx(None, psfex=mc),
                             GaussianMixturePSF(np.array([1.]), np.zeros((1, 2)),
                                                np.array([[[2.5, 0.], [0., 2.5]]])))
    # kind 0 exp, 1 Sersic, 3 point source, 4 exp with the hybrid PSF; px, py,
    # r_e, b/a, phi, n; mask (x0, y0, w, h)
    cases = [(0, 10.3, 12.7, 3.0, 0.6, 20., 1.0, (0, 0, 32, 32)),
             (1, 88.6, 20.1, 4.0, 0.5, 110., 2.5, (70, 0, 30, 48)),
             (1, 51.2, 85.4, 6.0, 0.8, 60., 0.9, (20, 50, 64, 50)),
             (3, 15.4, 80.2, 0., 1., 0., 1., (0, 60, 40, 40)),
             (3, 90.1, 10.6, 0., 1., 0., 1., (70, 0, 30, 30)),
             (4, 70.2, 70.8, 12.0, 0.7, 45., 1.0, (40, 40, 60, 60))]
    out = []
    for kind, px, py, re, ab, phi, n, mk in cases:
        pos, flux = PixPos(px, py), Flux(1000.)
        if kind == 3:
            src = PointSource(pos, flux)
        else:
            ell = EllipseE.fromRAbPhi(re, ab, phi)
            src = (SersicGalaxy(pos, flux, ell, SersicIndex(n)) if kind == 1
                   else ExpGalaxy(pos, flux, ell))
        tim = Image(data=np.zeros((100, 100), np.float32), inverr=np.ones((100, 100), np.float32),
                    psf=hyb if kind == 4 else psf, photocal=LinearPhotoCal(1.))
        out.append(src.getModelPatch(tim, modelMask=ModelMask(*mk)))
    table = np.array([list(c[:7]) + list(c[7]) for c in cases], np.float64)
    np.savez_compressed(os.path.join(OUT, 'psfex.npz'), cases=table, bases=bases,
                        poly=np.array([m.degree, m.x0, m.y0, m.xscale, m.yscale]),
                        **patches_to_arrays(out))
    print('psfex fixture written to', OUT)


def emfit():
    """GaussianMixturePSF.fromStamp (psf.py:536-597) -- the EM fit of
    em_fit_2d_reg (emfit.i:274-557) after fromStamp's normalisation -- on
    seeded stamps: Moffat and Gaussian-sum profiles with noise, square and
    not, 1 to 4 components, with and without the alpha prior, default and
    explicit origins, and an initial guess P0."""
    from oracle import refharness
    refharness.load()
    from tractor.psf import GaussianMixturePSF
    rng = np.random.default_rng(777)

    def gsum(h, w, parts, noise):
        y, x = np.mgrid[:h, :w]
        x = x - w // 2
        y = y - h // 2
        img = np.zeros((h, w))
        for a, mx, my, sx, sy, rho in parts:
            dx, dy = x - mx, y - my
            q = (dx / sx) ** 2 - 2 * rho * dx * dy / (sx * sy) + (dy / sy) ** 2
            img += a * np.exp(-0.5 * q / (1 - rho ** 2))
        img /= img.sum()
        return img + rng.normal(0., noise, img.shape)

    cases = [
        # stamp, N, alpha, steps, xy0, P0
        (moffat(25, 4.0, 3.0), 3, 0., 1000, None, None),
        (moffat(33, 5.0, 2.5), 2, 0., 500, None, None),
        (moffat(21, 3.0, 4.0), 1, 0.5, 300, None, None),
        (gsum(25, 25, [(0.6, 0., 0., 1.5, 1.5, 0.), (0.3, 0.5, 0., 3., 2.5, 0.2),
                       (0.1, 0., -0.3, 6., 6., 0.)], 1e-4).astype(np.float32),
         3, 0., 1000, None, None),
        (gsum(21, 31, [(0.7, 0.2, 0.1, 1.2, 2.0, -0.3), (0.3, 0., 0., 3.5, 3.0, 0.1)], 3e-4),
         2, 0.1, 800, (-15, -10), None),
        (gsum(29, 29, [(0.5, 0., 0., 1.0, 1.0, 0.), (0.3, 0., 0., 2.0, 2.0, 0.),
                       (0.15, 0., 0., 4.0, 4.0, 0.), (0.05, 0., 0., 8.0, 8.0, 0.)], 2e-5),
         4, 0., 1000, None, None),
        (moffat(25, 4.0, 3.0), 3, 0., 400, None,
         (np.array([0.5, 0.3, 0.2]), np.zeros((3, 2)),
          np.array([np.eye(2) * 1.5, np.eye(2) * 4., np.eye(2) * 12.]))),
    ]
    arrays = {}
    for i, (stamp, N, alpha, steps, xy0, P0) in enumerate(cases):
        P0c = None if P0 is None else tuple(np.array(a, copy=True) for a in P0)
        psf = GaussianMixturePSF.fromStamp(stamp, N=N, P0=P0c, xy0=xy0, alpha=alpha,
                                           emsteps=steps)
        arrays['stamp%d' % i] = stamp
        arrays['cfg%d' % i] = np.array([N, alpha, steps, xy0 is not None,
                                        0 if xy0 is None else xy0[0],
                                        0 if xy0 is None else xy0[1], P0 is not None])
        if P0 is not None:
            arrays['p0amp%d' % i], arrays['p0mean%d' % i], arrays['p0var%d' % i] = P0
        arrays['amp%d' % i] = psf.mog.amp
        arrays['mean%d' % i] = psf.mog.mean
        arrays['var%d' % i] = psf.mog.var
    # HybridPixelizedPSF without its Gaussian approximation fits one to the
    # pixelized model's image (psf.py:606-618)
    from tractor.psf import HybridPixelizedPSF, PixelizedPSF
    hstamp = moffat(33, 4.5, 2.8)
    hyb = HybridPixelizedPSF(PixelizedPSF(hstamp), N=2)
    arrays['hyb_stamp'] = hstamp
    arrays['hyb_amp'] = hyb.gauss.mog.amp
    arrays['hyb_mean'] = hyb.gauss.mog.mean
    arrays['hyb_var'] = hyb.gauss.mog.var
    np.savez_compressed(os.path.join(OUT, 'emfit.npz'), n=len(cases), **arrays)
    print('emfit fixture written to', OUT)


def emfitsky():
    """GaussianMixturePSF.fromStamp(v2=True) (psf.py:579-588) -- the EM fit
    with a flat sky term, em_fit_2d_reg2 (emfit2.c), on the stamp as given --
    on seeded stamps with a background and noise (pixels at or below zero
    go to the sky), 1 to 3 components, with and without the alpha prior,
    two approx cuts, default and explicit origins."""
    from oracle import refharness
    refharness.load()
    from tractor.psf import GaussianMixturePSF
    rng = np.random.default_rng(778)

    def stamp(h, w, sig, bg, noise):
        y, x = np.mgrid[:h, :w]
        x = x - w // 2 + rng.uniform(-0.4, 0.4)
        y = y - h // 2 + rng.uniform(-0.4, 0.4)
        img = np.zeros((h, w))
        for a, s in sig:
            img += a * np.exp(-0.5 * (x ** 2 + y ** 2) / s ** 2) / (2 * np.pi * s ** 2)
        return img + bg + rng.normal(0., noise, img.shape)

    cases = [
        # stamp, N, alpha, steps, approx, xy0
        (stamp(25, 25, [(100., 1.5), (40., 3.5)], 0.05, 0.02), 2, 0., 300, 1e-30, None),
        (stamp(31, 27, [(80., 1.2), (30., 2.5), (10., 6.)], 0.02, 0.01), 3, 0., 500, 1e-30,
         None),
        (stamp(21, 21, [(50., 2.0)], 0.1, 0.05), 1, 0.5, 200, 1e-30, (-10, -10)),
        (stamp(25, 25, [(100., 1.5), (40., 3.5)], 0.0, 0.03), 2, 0.1, 400, 1e-12, None),
    ]
    arrays = {}
    for i, (st, N, alpha, steps, approx, xy0) in enumerate(cases):
        psf, sky = GaussianMixturePSF.fromStamp(st, N=N, xy0=xy0, alpha=alpha, emsteps=steps,
                                                v2=True, approx=approx)
        arrays['stamp%d' % i] = st
        arrays['cfg%d' % i] = np.array([N, alpha, steps, approx, xy0 is not None,
                                        0 if xy0 is None else xy0[0],
                                        0 if xy0 is None else xy0[1]])
        arrays['amp%d' % i] = psf.mog.amp
        arrays['mean%d' % i] = psf.mog.mean
        arrays['var%d' % i] = psf.mog.var
        arrays['sky%d' % i] = np.array(sky)
    np.savez_compressed(os.path.join(OUT, 'emfit_sky.npz'), n=len(cases), **arrays)
    print('emfit_sky fixture written to', OUT)


def psf_scene(tractor_mod, ellipse):
    """A 40 x 36 image with two point sources and an exp galaxy under a
    2-component MoG PSF (GaussianMixturePSF, or GaussianMixtureEllipsePSF
    when `ellipse`) and a constant sky, the PSF and sky thawed, the catalog
    frozen."""
    T = tractor_mod
    from tractor.psf import GaussianMixtureEllipsePSF
    from tractor.sky import ConstantSky
    from tractor.galaxy import ExpGalaxy
    if ellipse:
        psf = GaussianMixtureEllipsePSF(np.array([0.7, 0.3]), np.array([[0.1, -0.05], [0., 0.2]]),
                                        [T.EllipseESoft(0.4, 0.05, -0.1),
                                         T.EllipseESoft(1.1, -0.02, 0.03)])
    else:
        psf = T.GaussianMixturePSF(np.array([0.7, 0.3]), np.array([[0.1, -0.05], [0., 0.2]]),
                                   np.array([[[1.6, 0.2], [0.2, 1.9]], [[7.5, -0.4], [-0.4, 8.2]]]))
    tim = T.Image(data=np.zeros((36, 40), np.float32), inverr=np.ones((36, 40), np.float32),
                  psf=psf, sky=ConstantSky(2.5), photocal=T.LinearPhotoCal(1.))
    srcs = [T.PointSource(T.PixPos(12.3, 10.6), T.Flux(800.)),
            T.PointSource(T.PixPos(27.8, 25.1), T.Flux(450.)),
            ExpGalaxy(T.PixPos(20.4, 17.2), T.Flux(1200.), T.EllipseE(2.5, 0.2, -0.1))]
    tr = T.Tractor([tim], srcs)
    tr.freezeParam('catalog')
    tim.freezeAllBut('psf', 'sky')
    return tr, tim


def psfderiv():
    """Image-parameter derivatives (engine.py:306-324: forward differences of
    the model image for the PSF, the sky's own derivative) for both MoG PSF
    parameterisations, and the optimiser-based PSF fits
    GaussianMixtureEllipsePSF.fromStamp (psf.py:757-789) and
    GaussianMixturePSF.fromStamp(v3=True) (psf.py:563-575)."""
    from oracle import refharness
    T = refharness.load()
    import tractor
    from tractor.psf import GaussianMixturePSF, GaussianMixtureEllipsePSF
    arrays = {}
    for tag, ellipse in (('mog', False), ('ell', True)):
        tr, tim = psf_scene(tractor, ellipse)
        derivs = tr.getDerivs()
        arrays[tag + '_names'] = np.array(tr.getParamNames())
        arrays[tag + '_params'] = np.array(tr.getParams())
        cols = []
        for d in derivs:
            (patch, img), = d
            full = np.zeros(img.shape, np.float64)
            patch.addTo(full)
            cols.append(full)
        arrays[tag + '_derivs'] = np.array(cols)
        arrays[tag + '_model'] = tr.getModelImage(0)
    stamp = moffat(25, 4.0, 3.0)
    p1 = GaussianMixtureEllipsePSF.fromStamp(stamp, N=2)
    arrays['ell_fit'] = np.array(p1.getAllParams())
    p2 = GaussianMixturePSF.fromStamp(stamp, N=2, v3=True)
    arrays['v3_fit'] = np.array(p2.getAllParams())
    arrays['stamp'] = stamp
    np.savez_compressed(os.path.join(OUT, 'psf_derivs.npz'), **arrays)
    print('psf_derivs fixture written to', OUT)


def forced_scene(T, rng, sky_true=None):
    """Six sources of fixed shape / position (point, exp, deV) seen in two
    64 x 72 images of one band with different PSFs and photometric scales;
    noisy data drawn from the true model (plus a constant sky per image when
    `sky_true` is given).  Returns (tractor, images, sources, rows, datas)."""
    from tractor.galaxy import ExpGalaxy, DevGalaxy
    H, W = 64, 72
    psfs = [T.NCircularGaussianPSF([1.2, 2.6], [0.75, 0.25]),
            T.GaussianMixturePSF(np.array([0.6, 0.3, 0.1]), np.zeros((3, 2)),
                                 np.array([np.eye(2) * s ** 2 for s in (1.5, 3.0, 6.0)]))]
    scales = [1.0, 2.5]
    rows, srcs = [], []
    for i in range(6):
        kind = i % 3
        px, py = rng.uniform(8, W - 8), rng.uniform(8, H - 8)
        fl = rng.uniform(50., 500.)
        re = float(rng.uniform(1., 3.))
        e1, e2 = rng.uniform(-0.3, 0.3, 2)
        br = T.Flux(fl)
        if kind == 0:
            s = T.PointSource(T.PixPos(px, py), br)
        elif kind == 1:
            s = ExpGalaxy(T.PixPos(px, py), br, T.EllipseE(re, e1, e2))
        else:
            s = DevGalaxy(T.PixPos(px, py), br, T.EllipseE(re, e1, e2))
        rows.append([kind, px, py, fl, re, e1, e2])
        srcs.append(s)
    from tractor.sky import ConstantSky
    tims = []
    for b in range(2):
        sky = ConstantSky(0. if sky_true is None else sky_true[b])
        tims.append(T.Image(data=np.zeros((H, W), np.float32),
                            inverr=np.ones((H, W), np.float32), psf=psfs[b],
                            photocal=T.LinearPhotoCal(scales[b]), sky=sky))
    tr = T.Tractor(tims, srcs)
    datas = []
    for b, tim in enumerate(tims):
        clean = tr.getModelImage(b)
        tim.data = (clean + rng.normal(size=clean.shape) * 0.5).astype(np.float32)
        tim.inverr = np.full((H, W), 2., np.float32)
        datas.append(tim.data.copy())
    return tr, tims, srcs, rows, datas


def forcedsky():
    """Forced photometry (optimize.py:16-145, lsqr_optimizer.py:11-235) with
    the images' constant skies fitted along with the fluxes (sky=True, the
    fluxes' variance), the fit statistics (optimize.py:233-375),
    and justims0's first evaluation, on the forced-photometry scene with a
    sky added to the data."""
    from oracle import refharness
    refharness.load()
    import tractor
    rng = np.random.default_rng(610)
    tr, tims, srcs, rows, datas = forced_scene(tractor, rng, sky_true=[3.0, -1.5])
    for s in srcs:
        s.freezeAllBut('brightness')
        s.brightness.setParams([v * 0.7 + 5. for v in s.brightness.getParams()])
    for tim in tims:
        tim.freezeAllBut('sky')
        tim.getSky().setParams([0.5])
    start = np.array(tr.getParams())
    R0 = tr.optimize_forced_photometry(sky=True, justims0=True, shared_params=False)
    lnp0 = R0.lnp0
    chis0 = np.stack(R0.chis0)
    # (skyvariance=True fails in the reference: _get_iv unpacks its
    # [(dsky, img)] lists as pairs, optimize.py:381)
    R = tr.optimize_forced_photometry(sky=True, variance=True, fitstats=True,
                                      shared_params=False)
    fs = R.fitstats
    keys = ['prochi2', 'pronpix', 'promasked', 'profracflux', 'proflux', 'npix', 'fracin',
            'imchisq', 'imnpix', 'sky']
    np.savez_compressed(os.path.join(OUT, 'forced_sky.npz'), sources=np.array(rows),
                        data=np.stack(datas), start=start, params=np.array(tr.getParams()),
                        names=np.array(tr.getParamNames()), IV=np.array(R.IV), lnp0=lnp0,
                        chis0=chis0, **{'fs_' + k: np.asarray(getattr(fs, k)) for k in keys})
    print('forced_sky fixture written to', OUT)


def varying():
    """VaryingGaussianPSF (psfex.py:8-150) over the degree-2 PsfEx model of
    psfex.npz (100 x 80 image): (a) GaussianMixtureEllipsePSF on a 4 x 4
    grid through the reference's own _fitParamGrid (each optimiser fit
    started from the previous one); (b) GaussianMixturePSF on a 4 x 4 grid,
    each point fitted by fromStamp's EM from its default start (the
    reference's grid loop cannot pass one EM fit's parameters to the next)
    and splined by the reference's fitSavedData.  The mixture parameters at
    a few positions."""
    from oracle import refharness
    refharness.load()
    from tractor.psf import GaussianMixturePSF, GaussianMixtureEllipsePSF
    from tractor.psfex import PsfExModel, VaryingGaussianPSF
    g = np.load(os.path.join(OUT, 'psfex.npz'))
    deg, x0, y0, xs, ys = g['poly']
    m = PsfExModel()
    m.sampling, m.psfbases, m.degree = 1., g['bases'], int(deg)
    m.x0, m.y0, m.xscale, m.yscale = x0, y0, xs, ys
    m.radius, m.fwhm = (g['bases'].shape[1] + 1) / 2., 4.0

    class Varying(VaryingGaussianPSF):
        def instantiateAt(self, x, y):
            return m.at(x, y)

    pos = np.array([[10.5, 20.25], [60., 45.], [90., 75.], [0., 0.]])
    ve = Varying(100, 80, nx=4, ny=4, K=2, psfClass=GaussianMixtureEllipsePSF)
    ve._fitParamGrid()
    ell = np.array([ve.psfParamsAt(x, y) for x, y in pos])
    K = 2
    vm = Varying(100, 80, nx=4, ny=4, K=K)
    YY, XX = np.linspace(0, 80, 4), np.linspace(0, 100, 4)
    pp = np.array([[GaussianMixturePSF.fromStamp(m.at(x, y), N=K).getAllParams() for x in XX]
                   for y in YY])
    vm.fitSavedData(pp, XX, YY)
    mog = np.array([vm.psfParamsAt(x, y) for x, y in pos])
    np.savez_compressed(os.path.join(OUT, 'varying_psf.npz'), pos=pos, ell=ell, mog=mog,
                        mog_grid=pp)
    print('varying_psf fixture written to', OUT)


def composite():
    """CompositeGalaxy (galaxy.py:1032-1160) on a 60 x 60 image with a
    2-Gaussian PSF: the model patch with and without a mask, and the
    derivatives with the position thawed and frozen."""
    from oracle import refharness
    refharness.load()
    from tractor import (Image, PixPos, Flux, LinearPhotoCal, NCircularGaussianPSF, EllipseE)
    from tractor.galaxy import CompositeGalaxy
    from tractor.patch import ModelMask
    tim = Image(data=np.zeros((60, 60), np.float32), inverr=np.ones((60, 60), np.float32),
                psf=NCircularGaussianPSF([1.5, 3.0], [0.8, 0.2]), photocal=LinearPhotoCal(1.))
    src = CompositeGalaxy(PixPos(30.3, 29.6), Flux(800.), EllipseE(2.5, 0.2, -0.1), Flux(400.),
                          EllipseE(4.0, -0.1, 0.25))
    arrays = {}
    for k, v in patches_to_arrays([src.getModelPatch(tim)]).items():
        arrays['model.' + k] = v
    mm = ModelMask(10, 12, 40, 36)
    for k, v in patches_to_arrays([src.getModelPatch(tim, modelMask=mm)]).items():
        arrays['masked.' + k] = v
    for k, v in patches_to_arrays(src.getParamDerivatives(tim)).items():
        arrays['derivs.' + k] = v
    src.freezeParam('pos')
    for k, v in patches_to_arrays(src.getParamDerivatives(tim)).items():
        arrays['derivs_nopos.' + k] = v
    np.savez_compressed(os.path.join(OUT, 'composite.npz'), **arrays)
    print('composite fixture written to', OUT)


def edges():
    """Empty and degenerate inputs through the object API (engine.py,
    galaxy.py, pointsource.py) on a 50 x 40 image with a constant sky: a
    catalog with no sources; galaxies and point sources entirely off the
    image or of zero flux; a ModelMask off the image.  The model images, the
    log-likelihoods, every patch (None where the reference returns None) and
    getDerivs' entries per parameter (image parameters thawed)."""
    from oracle import refharness
    refharness.load()
    from tractor import (Image, Tractor, PixPos, Flux, LinearPhotoCal, NCircularGaussianPSF,
                         EllipseE, ConstantSky, PointSource, ExpGalaxy)
    from tractor.patch import ModelMask
    data = np.random.default_rng(44).normal(2.5, 1., (40, 50))

    def image():
        return Image(data=data.copy(), invvar=np.ones((40, 50)),
                     psf=NCircularGaussianPSF([1.5, 3.0], [0.8, 0.2]),
                     photocal=LinearPhotoCal(1.), sky=ConstantSky(2.5))
    arrays = {'data': data}
    tr0 = Tractor([image()], [])
    arrays['empty_model'] = tr0.getModelImage(0)
    arrays['empty_lnl'] = tr0.getLogLikelihood()
    tim = image()
    srcs = [ExpGalaxy(PixPos(-200., 20.), Flux(100.), EllipseE(2., 0.1, 0.)),
            PointSource(PixPos(300., 20.), Flux(100.)),
            ExpGalaxy(PixPos(20., 20.), Flux(0.), EllipseE(2., 0.1, 0.)),
            PointSource(PixPos(20., 20.), Flux(0.))]
    patches = [s.getModelPatch(tim) for s in srcs]
    mm = ModelMask(500, 500, 10, 10)
    patches += [s.getModelPatch(tim, modelMask=mm)
                for s in (ExpGalaxy(PixPos(20., 20.), Flux(100.), EllipseE(2., 0.1, 0.)),
                          PointSource(PixPos(20., 20.), Flux(100.)))]
    for k, v in patches_to_arrays(patches).items():
        arrays['patches.' + k] = v
    tr = Tractor([tim], srcs)
    arrays['model'] = tr.getModelImage(0)
    arrays['lnl'] = tr.getLogLikelihood()
    d = tr.getDerivs()
    arrays['deriv_count'] = np.array([len(x) for x in d])
    for k, v in patches_to_arrays([p for x in d for (p, _) in x]).items():
        arrays['derivs.' + k] = v
    # a galaxy much smaller than a pixel: its shape columns are small
    # differences of two FP64 renders
    tiny = ExpGalaxy(PixPos(20.3, 19.6), Flux(100.), EllipseE(0.02, 0.2, -0.1))
    for k, v in patches_to_arrays(tiny.getParamDerivatives(image())).items():
        arrays['tiny.' + k] = v
    np.savez_compressed(os.path.join(OUT, 'edges.npz'), **arrays)
    print('edge-case fixture written to', OUT)


def fittight():
    """The optimum of the small plain fit (scenario 4) in FP64, found on the
    reference's own FP64 model: scipy.optimize.least_squares on
    Tractor.getChiImage (tolerances 1e-15) from the scenario's start.  Stored
    with its log-probability and the Fisher matrix A^T A of the reference's
    derivative columns there (inverse errors 1; the position columns divided
    by NullWCS's cd_inverse of 3600 so that the matrix is per pixel), whose
    inverse gives the parameters' sigmas.  Also the reference's own
    LsqrOptimizer.optimize_loop(dchisq=1e-10) started at the optimum with the
    flux and shape moved (0, 0, +20, +0.05, +0.02, -0.02): its end point and
    step count.  (From the scenario's start the reference's optimizer needs
    many thousands of steps: NullWCS scales the position derivatives by
    3600, which shrinks every position step by that factor.)"""
    from oracle import refharness
    refharness.load()
    from scipy.optimize import least_squares
    from tractor import (Image, PixPos, Flux, LinearPhotoCal, NCircularGaussianPSF, EllipseE,
                         ExpGalaxy, Tractor)
    g = np.load(os.path.join(OUT, 'fit_plain.npz'))
    timc = Image(data=g['data'], invvar=np.ones((64, 64)),
                 psf=NCircularGaussianPSF([1.5, 3.0], [0.8, 0.2]), photocal=LinearPhotoCal(1.))
    src = ExpGalaxy(PixPos(32.5, 32.5), Flux(800.), EllipseE.fromRAbPhi(2.4, 0.6, 30.))
    tr = Tractor([timc], [src])
    tr.modtype = np.float64
    tr.freezeParam('images')

    def resid(p):
        tr.setParams(p)
        return tr.getChiImage(0).ravel().astype(np.float64)
    r = least_squares(resid, np.array(tr.getParams()), x_scale=[0.03, 0.03, 10., 0.05, 0.02, 0.02],
                      xtol=1e-15, ftol=1e-15, gtol=1e-15, diff_step=1e-7)
    p_opt = r.x
    tr.setParams(p_opt)
    lnp = tr.getLogProb()
    cols = []
    for k, d in enumerate(src.getParamDerivatives(timc)):
        full = np.zeros((64, 64))
        d.addTo(full)
        cols.append(full.ravel() / (3600. if k < 2 else 1.))
    A = np.array(cols)
    fisher = A @ A.T
    pert = np.array([0., 0., 20., 0.05, 0.02, -0.02])
    tr.setParams(p_opt + pert)
    R = tr.optimize_loop(dchisq=1e-10, steps=300)
    p_ref = np.array(tr.getParams())
    np.savez_compressed(os.path.join(OUT, 'fit_plain_tight.npz'), p_opt=p_opt, lnp=lnp,
                        fisher=fisher, pert=pert, p_ref_from_pert=p_ref, ref_steps=R['steps'])
    sig = np.sqrt(np.diag(np.linalg.inv(fisher)))
    print('fit_plain_tight fixture written to', OUT, 'reference from the moved start:',
          R['steps'], 'steps,', np.abs(p_ref - p_opt) / sig, 'sigma')


if __name__ == '__main__':
    if sys.argv[1:] == ['fittight']:
        fittight()
    elif sys.argv[1:] == ['hybrid']:
        hybrid()
    elif sys.argv[1:] == ['psfex']:
        psfex()
    elif sys.argv[1:] == ['emfit']:
        emfit()
    elif sys.argv[1:] == ['emfitsky']:
        emfitsky()
    elif sys.argv[1:] == ['psfderiv']:
        psfderiv()
    elif sys.argv[1:] == ['forcedsky']:
        forcedsky()
    elif sys.argv[1:] == ['varying']:
        varying()
    elif sys.argv[1:] == ['composite']:
        composite()
    elif sys.argv[1:] == ['edges']:
        edges()
    else:
        main()
