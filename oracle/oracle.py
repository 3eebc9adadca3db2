"""Oracle (test infrastructure only -- never imported by the product path).

A CPU restatement of the reference Tractor's forward-model hot path in numpy
(FP64) over the plain-C kernels in oracle/oracle_c.c.  tests/, the smoke check
and bench.py's CPU-baseline leg use it as the checker.  Each function cites the
reference lines it restates; paths are relative to the reference project.

Parity pin: tests/test_oracle_pin.py checks these functions against the
reference itself (run from its source tree through oracle/refharness.py, in the
development container) and against the committed fixtures in tests/golden/,
which were generated from the reference by tests/golden/make_golden.py.
"""
import ctypes
import json
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, 'liboracle_c.so')
_TABLES = os.path.join(os.path.dirname(_HERE), 'tractor_b200', 'data', 'profile_tables.json')
_lib = None


def build_lib():
    """Compile oracle_c.c (plain gcc, no device code)."""
    src = os.path.join(_HERE, 'oracle_c.c')
    if (os.path.exists(_LIB_PATH) and
            os.path.getmtime(_LIB_PATH) >= os.path.getmtime(src)):
        return _LIB_PATH
    cmd = 'gcc -O2 -fPIC -shared -std=gnu99 -o %s %s -lm' % (_LIB_PATH, src)
    if os.system(cmd) != 0:
        raise RuntimeError('oracle build failed: ' + cmd)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build_lib()
        L = ctypes.CDLL(_LIB_PATH)
        I, D = ctypes.c_int, ctypes.c_double
        P = ctypes.c_void_p
        L.orc_mog_grid.argtypes = [I, I, I, I, D, D, I, P, P, P, P]
        L.orc_mog_approx3.argtypes = [I, I, I, I, D, D, D, I, P, P, P, P, P, P, I, I, I, P]
        L.orc_mog_masked.argtypes = [I, I, I, I, D, D, I, P, P, P, P, P, P, P]
        L.orc_lanczos3_taps.argtypes = [D, P]
        L.orc_lanczos_shift3f.argtypes = [P, P, I, I, D, D, P]
        L.orc_fourier_mog.argtypes = [I, P, P, I, P, I, P, P]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# ---------------------------------------------------------------------------
# Native kernels
# ---------------------------------------------------------------------------

def mog_grid(x0, x1, y0, y1, fx, fy, amp, mean, var):
    """c_gauss_2d_grid (tractor/mix.i:452-524); float64 (y1-y0, x1-x0)."""
    amp = np.ascontiguousarray(amp, np.float64)
    mean = np.ascontiguousarray(mean, np.float64).reshape(-1, 2)
    var = np.ascontiguousarray(var, np.float64).reshape(-1, 2, 2)
    out = np.zeros((y1 - y0, x1 - x0), np.float64)
    r = lib().orc_mog_grid(int(x0), int(x1), int(y0), int(y1), float(fx), float(fy),
                           len(amp), _p(amp), _p(mean), _p(var), _p(out))
    assert r == 0
    return out


def mog_approx3(x0, x1, y0, y1, fx, fy, minval, amp, mean, var, xc, yc,
                minradius=3, derivs=False):
    """c_gauss_2d_approx3 (tractor/approx3.c); returns (out, dx, dy, bbox)."""
    amp = np.ascontiguousarray(amp, np.float64)
    mean = np.ascontiguousarray(mean, np.float64).reshape(-1, 2)
    var = np.ascontiguousarray(var, np.float64).reshape(-1, 2, 2)
    out = np.zeros((y1 - y0, x1 - x0), np.float64)
    dxo = np.zeros_like(out) if derivs else None
    dyo = np.zeros_like(out) if derivs else None
    bbox = np.zeros(4, np.int32)
    r = lib().orc_mog_approx3(int(x0), int(x1), int(y0), int(y1), float(fx), float(fy),
                              float(minval), len(amp), _p(amp), _p(mean), _p(var), _p(out),
                              _p(dxo) if derivs else None, _p(dyo) if derivs else None,
                              int(xc), int(yc), int(minradius), _p(bbox))
    assert r == 0
    return out, dxo, dyo, tuple(int(b) for b in bbox)


def mog_masked(x0, y0, mask, fx, fy, amp, mean, var, derivs=False):
    """c_gauss_2d_masked (tractor/gauss_masked.c); float32 outputs."""
    amp = np.ascontiguousarray(amp, np.float32)
    mean = np.ascontiguousarray(mean, np.float32).reshape(-1, 2)
    var = np.ascontiguousarray(var, np.float32).reshape(-1, 2, 2)
    mask = np.ascontiguousarray(mask, np.uint8)
    h, w = mask.shape
    out = np.zeros((h, w), np.float32)
    dxo = np.zeros_like(out) if derivs else None
    dyo = np.zeros_like(out) if derivs else None
    lib().orc_mog_masked(int(x0), int(y0), w, h, float(fx), float(fy), len(amp), _p(amp),
                         _p(mean), _p(var), _p(out), _p(dxo) if derivs else None,
                         _p(dyo) if derivs else None, _p(mask))
    return out, dxo, dyo


def lanczos3_taps(dx):
    """lanczos_filter_3 (tractor/mp_fourier.i:355-402)."""
    t = np.zeros(7, np.float64)
    lib().orc_lanczos3_taps(float(dx), _p(t))
    return t


def lanczos_shift(img, dx, dy):
    """lanczos_shift_3f (tractor/mp_fourier.i:405-429) on a float32 image."""
    img = np.ascontiguousarray(img, np.float32)
    H, W = img.shape
    out = np.zeros_like(img)
    work = np.zeros(H * W, np.float32)
    lib().orc_lanczos_shift3f(_p(img), _p(out), H, W, float(dx), float(dy), _p(work))
    return out


def fourier_mog(amp, var, v, w):
    """gaussian_fourier_transform_zero_mean (tractor/mp_fourier.i:431-478)."""
    amp = np.ascontiguousarray(amp, np.float64)
    var = np.ascontiguousarray(var, np.float64).reshape(-1, 2, 2)
    v = np.ascontiguousarray(v, np.float64)
    w = np.ascontiguousarray(w, np.float64)
    out = np.zeros((len(w), len(v)), np.float64)
    lib().orc_fourier_mog(len(amp), _p(amp), _p(var), len(v), _p(v), len(w), _p(w), _p(out))
    return out


# ---------------------------------------------------------------------------
# Profiles
# ---------------------------------------------------------------------------
_tables = None


def tables():
    global _tables
    if _tables is None:
        with open(_TABLES) as f:
            _tables = json.load(f)
    return _tables


def exp_profile():
    """Exp 6-component mixture, tractor/mixture_profiles.py:20-24 (normalised)."""
    t = tables()['exp']
    return np.array(t['amp']), np.array(t['var'])


def dev_profile():
    """deV 8 components + delta core, tractor/mixture_profiles.py:26-38."""
    t = tables()['dev']
    return np.array(t['amp']), np.array(t['var'])


_sersic_splines = None


def sersic_profile(n):
    """SersicMixture._getProfile (tractor/sersic.py:288-342) with scipy's
    InterpolatedUnivariateSpline built from the raw grid as the reference does
    (sersic.py:242-282).  Returns (amp[K], var[K]) sorted by variance."""
    global _sersic_splines
    from scipy.interpolate import InterpolatedUnivariateSpline as IUS
    S = tables()['sersic']
    if _sersic_splines is None:
        fits = []
        for r in S['ranges']:
            grid = r['grid']
            ns = [g[0] for g in grid]
            k = 3 if len(grid) > 3 else 1
            af = [IUS(ns, [g[1][i] for g in grid], k=k) for i in range(r['K'])]
            vf = [IUS(ns, [np.log(g[2][i]) for g in grid], k=k) for i in range(r['K'])]
            fits.append((r['lo'], r['hi'], af, vf))
        core = IUS([c[0] for c in S['cores']], [c[1] for c in S['cores']], k=3)
        _sersic_splines = (fits, core)
    fits, core = _sersic_splines
    lowest, highest = fits[0][0], fits[-1][1]
    if n <= lowest:
        m = fits[0]
        n = lowest
    elif n >= highest:
        m = fits[-1]
        n = highest
    else:
        m = [f for f in fits if f[0] <= n < f[1]]
        assert len(m) == 1
        m = m[0]
    lo, hi, af, vf = m
    amps = np.array([f(n) for f in af])
    amps /= amps.sum()
    varr = np.exp(np.array([f(n) for f in vf]))
    if n > 1.:
        c = core(n)
        amps *= (1. - c) / amps.sum()
        amps = np.append(amps, c)
        varr = np.append(varr, 0.)
    I = np.argsort(varr)
    return amps[I], varr[I]


def diag_var(var):
    """MixtureOfGaussians.set_var for scalar variances (mixture_profiles.py:75-81)."""
    var = np.asarray(var, np.float64)
    V = np.zeros((len(var), 2, 2))
    V[:, 0, 0] = var
    V[:, 1, 1] = var
    return V


# ---------------------------------------------------------------------------
# Shapes (pixel-space transforms)
# ---------------------------------------------------------------------------

def galaxyshape_basis(re, ab, phi):
    """GalaxyShape.getRaDecBasis, tractor/galaxy.py:73-89."""
    p = np.deg2rad(90 - phi)
    re_deg = max(1. / 30, re) / 3600.
    cp, sp = np.cos(p), np.sin(p)
    return re_deg * np.array([[cp, sp * ab], [-sp, cp * ab]])


def ellipseE_basis(re, e1, e2):
    """EllipseE.getRaDecBasis, tractor/ellipses.py:126-155."""
    theta = math.atan2(e2, e1) / 2.
    ct, st = math.cos(theta), math.sin(theta)
    e = math.hypot(e1, e2)
    maxab = 1000.
    ab = maxab if e >= 1. else min(maxab, (1. + e) / (1. - e))
    r_deg = re / 3600.
    return r_deg * np.array([[ct / ab, st], [-st / ab, ct]])


def ellipseESoft_to_E(logre, ee1, ee2, maxe=0.999999):
    """EllipseESoft -> (re, e1, e2), tractor/ellipses.py:55-62, 219-238."""
    re = math.exp(logre)
    ee = math.hypot(ee1, ee2)
    e = min(maxe, 1. - math.exp(-ee))
    theta = math.atan2(ee2, ee1) / 2.
    return re, e * math.cos(2. * theta), e * math.sin(2. * theta)


def ellipseE_from_rabphi(r, ba, phi):
    """EllipseE.fromRAbPhi, tractor/ellipses.py:64-71."""
    ab = 1. / ba
    e = (ab - 1) / (ab + 1)
    angle = math.radians(2. * (-phi))
    return r, e * math.cos(angle), e * math.sin(angle)


def nullwcs_cdinv(pixscale=1.):
    """NullWCS.cd_inverse, tractor/wcs.py:25-28."""
    return np.eye(2) / (pixscale / 3600.)


def sheared(amp, var_scalar, Tinv):
    """apply_shear (mixture_profiles.py:146-155): var -> T V T^T."""
    V = diag_var(var_scalar)
    return np.asarray(amp, np.float64), Tinv @ V @ Tinv.T


def convolve(amp, mean, var, pamp, pmean, pvar):
    """MixtureOfGaussians.convolve, mixture_profiles.py:158-172: for each PSF
    component (outer loop) a block of all galaxy components."""
    K, P = len(amp), len(pamp)
    namp = np.zeros(K * P)
    nmean = np.zeros((K * P, 2))
    nvar = np.zeros((K * P, 2, 2))
    for p in range(P):
        namp[p * K:(p + 1) * K] = amp * pamp[p]
        nmean[p * K:(p + 1) * K] = mean + pmean[p]
        nvar[p * K:(p + 1) * K] = var + pvar[p]
    return namp, nmean, nvar


def circular_psf_mog(sigmas, weights):
    """getCircularMog (tractor/psf.py:931-944): float32 tables."""
    K = len(weights)
    amp = np.array(weights).astype(np.float32)
    mean = np.zeros((K, 2), np.float32)
    var = np.zeros((K, 2, 2), np.float32)
    for k in range(K):
        var[k, 0, 0] = var[k, 1, 1] = sigmas[k] ** 2
    return amp, mean, var


# ---------------------------------------------------------------------------
# Geometry helpers
# ---------------------------------------------------------------------------

def overlapping_region(xlo, xhi, xmin, xmax):
    """tractor/patch.pyx:20-65 (absolute slices)."""
    if xlo > xmax or xhi < xmin or xlo > xhi or xmin > xmax:
        return None
    lo = max(xlo, xmin)
    hi = min(xhi, xmax)
    return slice(lo, hi + 1), slice(lo - xlo, lo - xlo + hi - lo + 1)


def fft_size(radius):
    """PixelizedPSF.getFourierTransformSize, tractor/psf.py:209-212."""
    return int(2 ** int(np.ceil(np.log2(radius * 2.))))


def pad_psf(img, H, W):
    """PixelizedPSF._padInImage, tractor/psf.py:214-247."""
    ph, pw = img.shape
    sub = img
    if H >= ph:
        y0 = (H - ph) // 2
        cy = y0 + ph // 2
    else:
        y0 = 0
        cut = (ph - H) // 2
        sub = sub[cut:cut + H, :]
        cy = ph // 2 - cut
    if W >= pw:
        x0 = (W - pw) // 2
        cx = x0 + pw // 2
    else:
        x0 = 0
        cut = (pw - W) // 2
        sub = sub[:, cut:cut + W]
        cx = pw // 2 - cut
    sh, sw = sub.shape
    pad = np.zeros((H, W), img.dtype)
    pad[y0:y0 + sh, x0:x0 + sw] = sub
    return pad, cx, cy


def psf_fourier(psf_img, sz, normalized=False):
    """PixelizedPSF.getFourierTransform (tractor/psf.py:249-280): complex64
    rfft2 of the padded PSF; NormalizedPsf (psf.py:947-953) divides by |P[0,0]|."""
    pad, cx, cy = pad_psf(np.asarray(psf_img, np.float32), sz, sz)
    P = np.fft.rfft2(pad).astype(np.complex64)
    if normalized:
        n = np.abs(P[0][0])
        if n != 0:
            P /= n
    v = np.fft.rfftfreq(sz)
    w = np.fft.fftfreq(sz)
    return P, (cx, cy), (sz, sz), (v, w)


def fft_halfsize_for_mask(px, py, x0, y0, mw, mh, psfh, psfw):
    """Patch half-size for the FFT path with a ModelMask, galaxy.py:339-351."""
    x1 = x0 + mw
    y1 = y0 + mh
    hs = max(mh / 2., mw / 2.)
    hs = max(hs, max(max(1 + px - x0, 1 + x1 - px), max(1 + py - y0, 1 + y1 - py)))
    hs = max(hs, max(psfw / 2., psfh / 2.))
    return int(np.ceil(hs))


# ---------------------------------------------------------------------------
# Unit-flux galaxy patches
# ---------------------------------------------------------------------------

_work_cache = {}


def _ref_work(shape):
    """Scratch for the reference's lanczos_shift_3f (it indexes a compact
    W x H work array; tractor/psf.py:61 passes a 4096^2 global)."""
    if shape not in _work_cache:
        m = max(shape)
        _work_cache[shape] = np.zeros((m, m), np.float32)
    return _work_cache[shape]


def reference_kernels():
    """The reference's own Fourier / Lanczos C (tractor/mp_fourier.i), built
    into oracle/_ref/ by oracle/build_ref.sh, or None if it is not built."""
    path = os.path.join(_HERE, '_ref', 'libref_mpf.so')
    if not os.path.exists(path):
        return None
    from . import refharness
    return refharness._mpf_module()


def galaxy_fft_masked(amp, var2, px, py, psf_img, mask_x0, mask_y0, mw, mh,
                      normalized_psf=False, force_halfsize=None, kernels=None):
    """ProfileGalaxy._realGetUnitFluxModelPatch FFT branch with a ModelMask and
    a non-hybrid pixelized PSF (tractor/galaxy.py:336-519).  `var2` is the
    sheared (pixel-space) 2x2 covariance per component.  Returns the float32
    (mh, mw) unit-flux patch with origin (mask_x0, mask_y0), plus the split
    (mux, muy, sx, sy, sz) for diagnostics.  `kernels` (from
    reference_kernels()) swaps in the reference's own compiled C for the
    spectrum and the Lanczos shift."""
    psfh, psfw = psf_img.shape
    hs = fft_halfsize_for_mask(px, py, mask_x0, mask_y0, mw, mh, psfh, psfw)
    if force_halfsize is not None:
        hs = int(np.ceil(force_halfsize))
    sz = fft_size(hs)
    P, (cx, cy), (pH, pW), (v, w) = psf_fourier(psf_img, sz, normalized_psf)
    dx = px - cx
    dy = py - cy
    mux = dx - mask_x0
    muy = dy - mask_y0
    sx = int(np.round(mux))
    sy = int(np.round(muy))
    mux -= sx
    muy -= sy
    assert abs(mux) <= 0.5 and abs(muy) <= 0.5
    if kernels is None:
        F = fourier_mog(amp, var2, v, w)
    else:
        F = np.zeros((len(w), len(v)), np.float64)
        kernels.gaussian_fourier_transform_zero_mean(amp, var2, v, w, F)
    G = np.fft.irfftn(F * P)
    G = G.astype(np.float32)
    if mux != 0.0 or muy != 0.0:
        if kernels is None:
            G = lanczos_shift(G, mux, muy)
        else:
            out = np.empty_like(G)
            kernels.lanczos_shift_3f(G, out, mux, muy, _ref_work(G.shape))
            G = out
    gh, gw = G.shape
    if sx != 0 or sy != 0:
        out = np.zeros((mh, mw), np.float32)
        ry = overlapping_region(-sy, -sy + mh - 1, 0, gh - 1)
        rx = overlapping_region(-sx, -sx + mw - 1, 0, gw - 1)
        if ry is not None and rx is not None:
            out[ry[1], rx[1]] = G[ry[0], rx[0]]
        G = out
    if gh > mh or gw > mw:
        G = G[:mh, :mw]
    return G, (mux, muy, sx, sy, sz)


def galaxy_mog_patch(amp, var_scalar, Tinv, px, py, pamp, pmean, pvar,
                     x0, x1, y0, y1, minval=0.):
    """MoG branch without a ModelMask (tractor/galaxy.py:307-326 ->
    mixture_profiles.py:425-438): affine profile at (px, py), convolved with
    the PSF, rendered exactly (minval == 0) or by the ring evaluator.
    Returns (x0, y0, patch float64)."""
    a = np.asarray(amp, np.float64)
    V = Tinv @ diag_var(var_scalar) @ Tinv.T
    mean = np.zeros((len(a), 2)) + np.array([px, py])
    ca, cm, cv = convolve(a, mean, V, np.asarray(pamp, np.float64),
                          np.asarray(pmean, np.float64), np.asarray(pvar, np.float64))
    if minval == 0. or minval is None:
        return x0, y0, mog_grid(x0, x1, y0, y1, 0., 0., ca, cm, cv)
    cx = int(cm[0, 0])
    cy = int(cm[0, 1])
    if cx < x0 - 100 or cx > x1 + 100 or cy < y0 - 100 or cy > y1 + 100:
        return None
    out, _, _, (sx0, sx1, sy0, sy1) = mog_approx3(x0, x1, y0, y1, 0., 0., minval,
                                                  ca, cm, cv, cx, cy, 3)
    return x0 + sx0, y0 + sy0, out[sy0:sy1, sx0:sx1].copy()


def galaxy_mog_masked_rect(amp, var_scalar, Tinv, px, py, pamp, pmean, pvar,
                           mx0, my0, mw, mh):
    """MoG branch with a rectangular ModelMask (galaxy.py:320-326): exact grid
    over the mask."""
    return galaxy_mog_patch(amp, var_scalar, Tinv, px, py, pamp, pmean, pvar,
                            mx0, mx0 + mw, my0, my0 + mh, 0.)[2]


def hogg_halfsize(re_pix_radius, px, py, W, H, psf_radius):
    """HoggGalaxy._getUnitFluxPatchSize, tractor/galaxy.py:678-691 (pixscale 1:
    `re_pix_radius` = nre * re / pixscale)."""
    hs = max(1., re_pix_radius)
    imsize = max(px, W - 1 - px, py, H - 1 - py) + 1
    hs = min(hs, imsize)
    hs = max(hs, psf_radius)
    return int(np.ceil(hs))


def image_extent(px, py, halfsize, W, H):
    """No-mask extent selection, tractor/galaxy.py:274-286."""
    rx = overlapping_region(int(np.floor(px - halfsize)), int(np.ceil(px + halfsize + 1)), 0, W - 1)
    ry = overlapping_region(int(np.floor(py - halfsize)), int(np.ceil(py + halfsize + 1)), 0, H - 1)
    if rx is None or ry is None:
        return None
    return rx[0].start, rx[0].stop, ry[0].start, ry[0].stop


# ---------------------------------------------------------------------------
# Point sources
# ---------------------------------------------------------------------------

def mogpsf_point_patch(pamp, pmean, pvar, px, py, x0, x1, y0, y1):
    """GaussianMixturePSF.getPointSourcePatch exact branch (psf.py:458-528
    with minval == 0): grid of the PSF mixture offset by (px, py)."""
    return mog_grid(x0, x1, y0, y1, px, py, pamp, pmean, pvar)


def pixpsf_point_patch_masked(psf_img, px, py, mx0, my0, mw, mh):
    """PixelizedPSF.getPointSourcePatch with a ModelMask (psf.py:137-207)."""
    img = np.asarray(psf_img, np.float32)
    H, W = img.shape
    ix = int(round(float(px)))
    iy = int(round(float(py)))
    dx = px - ix
    dy = py - iy
    x0 = ix - W // 2
    y0 = iy - H // 2
    if (mx0 >= x0 + W) or (mx0 + mw <= x0) or (my0 >= y0 + H) or (my0 + mh <= y0):
        return None
    L = 3
    mm = np.zeros((mh + 2 * L, mw + 2 * L), np.float32)
    ry = overlapping_region(my0 - y0 - L, my0 - y0 + mh - 1 + L, 0, H - 1)
    rx = overlapping_region(mx0 - x0 - L, mx0 - x0 + mw - 1 + L, 0, W - 1)
    mm[ry[1], rx[1]] = img[ry[0], rx[0]]
    mm = lanczos_shift(mm, dx, dy)
    return mm[L:-L, L:-L]


# ---------------------------------------------------------------------------
# Likelihood and least squares
# ---------------------------------------------------------------------------

# ---------------------------------------------------------------------------
# Batched scenes (Tractor.getModelImage with rectangular model masks)
# ---------------------------------------------------------------------------

SCENE_POINT, SCENE_EXP, SCENE_DEV, SCENE_COMP = 0, 1, 2, 3


def scene_source_mixture(kind, px, py, fdev, shape_a, shape_b, pamp, pmean, pvar,
                         cdinv=None):
    """Pixel-space mixture of one source with the PSF applied, in the order
    the reference evaluates it.  Point source: the PSF mixture itself, offset
    by (px, py) at evaluation (psf.py:458-528), returned with fx, fy = px, py.
    Exp / deV: _getAffineProfile (galaxy.py:648-669) convolved with the PSF
    (galaxy.py:307-326, mixture_profiles.py:158-172).  FixedComposite:
    _getAffineProfile of galaxy.py:847-876 -- deV block (amp x fracDev) then
    exp block (amp x (1 - fracDev)), each present only when its fraction is
    non-zero.  `shape_a` is the exp (or single) EllipseE (re, e1, e2),
    `shape_b` the deV one of a composite.  Returns (amp, mean, var, fx, fy)."""
    pamp = np.asarray(pamp, np.float64)
    pmean = np.asarray(pmean, np.float64)
    pvar = np.asarray(pvar, np.float64)
    if kind == SCENE_POINT:
        return pamp, pmean, pvar, px, py
    cdinv = nullwcs_cdinv() if cdinv is None else cdinv
    blocks = []
    if kind == SCENE_COMP:
        f = min(1., max(0., fdev))
        if f > 0.:
            blocks.append((f, dev_profile(), shape_b))
        if f < 1.:
            blocks.append((1. - f, exp_profile(), shape_a))
    else:
        blocks.append((1., exp_profile() if kind == SCENE_EXP else dev_profile(), shape_a))
    amps, vars_ = [], []
    for frac, (a, v), shp in blocks:
        T = cdinv @ ellipseE_basis(*shp)
        amps.append(np.asarray(a, np.float64) * frac)
        vars_.append(T @ diag_var(v) @ T.T)
    amp = np.concatenate(amps)
    var = np.concatenate(vars_)
    mean = np.zeros((len(amp), 2)) + np.array([px, py])
    ca, cm, cv = convolve(amp, mean, var, pamp, pmean, pvar)
    return ca, cm, cv, 0., 0.


def scene_model(sources, pamp, psig, H, W):
    """Tractor.getModelImage (engine.py:424-445) of a scene whose every source
    has a rectangular ModelMask inside the image: each patch is the exact grid
    over its mask (float64), times counts (LinearPhotoCal(1): counts = flux,
    pointsource.py:36-60), added in catalog order into a float32 image
    (Patch.addTo, patch.py:341-354).  `sources` rows: kind, px, py, flux, mx0,
    my0, mw, mh, fracDev, exp-or-single (re, e1, e2), deV (re, e1, e2)."""
    K = len(pamp)
    pmean = np.zeros((K, 2))
    pvar = np.zeros((K, 2, 2))
    pvar[:, 0, 0] = pvar[:, 1, 1] = np.asarray(psig, np.float64) ** 2
    mod = np.zeros((H, W), np.float32)
    for row in np.asarray(sources, np.float64):
        kind = int(row[0])
        px, py, flux = row[1], row[2], row[3]
        mx0, my0, mw, mh = (int(v) for v in row[4:8])
        ca, cm, cv, fx, fy = scene_source_mixture(kind, px, py, row[8], row[9:12], row[12:15],
                                                  pamp, pmean, pvar)
        p = mog_grid(mx0, mx0 + mw, my0, my0 + mh, fx, fy, ca, cm, cv) * flux
        mod[my0:my0 + mh, mx0:mx0 + mw] += p
    return mod


def chi_image(data, model, inverr):
    """Tractor.getChiImage, tractor/engine.py:455-473."""
    return (data - model) * inverr


def log_likelihood(chis):
    """Tractor.getLogLikelihood, tractor/engine.py:475-479 (FP64 sum)."""
    return -0.5 * sum(float((c.astype(float) ** 2).sum()) for c in chis)


def lsq_update(A_cols, b, priors=None):
    """The solution LsqrOptimizer.getUpdateDirection converges to
    (tractor/lsqr_optimizer.py:328-644): columns of A = J * inverr, scaled to
    unit L2 norm (:423-424, :470-489, dropping |v| <= 1e-8 after scaling),
    b = chi; x = argmin ||A x - b||; X = x / colscale.  Solved densely in FP64.
    `A_cols` is (Nrows, P); `priors` an optional (rows, b) pair appended."""
    A = np.asarray(A_cols, np.float64)
    b = np.asarray(b, np.float64)
    if priors is not None:
        A = np.vstack([A, priors[0]])
        b = np.concatenate([b, priors[1]])
    cs = np.sqrt((A ** 2).sum(axis=0))
    As = np.where(cs > 0, A / np.where(cs > 0, cs, 1.), 0.)
    As[np.abs(As) <= 1e-8] = 0.
    x, *_ = np.linalg.lstsq(As, b, rcond=None)
    X = np.where(cs > 0, x / np.where(cs > 0, cs, 1.), 0.)
    return X


def line_search_alphas():
    """Default step sizes of Optimizer.tryUpdates, tractor/optimize.py:426-428."""
    return np.append(2. ** np.arange(-10, 1), [np.sqrt(2.), 2.])


# ---------------------------------------------------------------------------
# Blob fitting (the batched form of Tractor.optimize_loop over several bands)
# ---------------------------------------------------------------------------

BLOB_NPAR = 9   # x, y, flux[3], log r_e, ee1, ee2, Sersic n


def blob_source_mixture(theta, band, pamp, pmean, pvar, cdinv=None):
    """PSF-convolved mixture of a SersicGalaxy (EllipseESoft shape,
    NanoMaggies counts = flux with LinearPhotoCal(1)) in one band: the
    profile (sersic.py:288-342), the shape (ellipses.py:165-263,
    galaxy.py:659-669), the convolution (mixture_profiles.py:158-172).
    Returns (amp x counts, mean, var)."""
    cdinv = nullwcs_cdinv() if cdinv is None else cdinv
    amp, var = sersic_profile(float(theta[8]))
    T = cdinv @ ellipseE_basis(*ellipseESoft_to_E(theta[5], theta[6], theta[7]))
    a2, v2 = sheared(amp, var, T)
    mean = np.zeros((len(a2), 2)) + np.array([theta[0], theta[1]])
    ca, cm, cv = convolve(a2, mean, v2, np.asarray(pamp, np.float64),
                          np.asarray(pmean, np.float64), np.asarray(pvar, np.float64))
    return ca * theta[2 + band], cm, cv


def blob_model(params, rects, W, H, psf, n_bands):
    """(n_bands, H, W) FP64 model of one blob: every source's grid over its
    mask rectangle clipped to the image (c_gauss_2d_grid, mix.i:452-524),
    summed (Tractor.getModelImage, engine.py:424-445)."""
    mod = np.zeros((n_bands, H, W))
    for k in range(n_bands):
        pamp, pmean, pvar = psf[k]
        for th, (x0, y0, w, h) in zip(params, rects):
            a, m, v = blob_source_mixture(th, k, pamp, pmean, pvar)
            X0, Y0 = max(x0, 0), max(y0, 0)
            X1, Y1 = min(x0 + w, W), min(y0 + h, H)
            if X1 <= X0 or Y1 <= Y0:
                continue
            mod[k, Y0:Y1, X0:X1] += mog_grid(X0, X1, Y0, Y1, 0., 0., a, m, v)
    return mod


def blob_normal_equations(params, rects, W, H, psf, n_bands, data, inverr, steps=None):
    """A^T A, A^T r, chi^2 of one blob in FP64 with A = d model / d params *
    inverr by central differences (fluxes exactly: the model is linear in
    them) and r = (data - model) * inverr (lsqr_optimizer.py:328-520 builds
    the same A and b)."""
    params = np.asarray(params, np.float64)
    n = len(params)
    P = n * BLOB_NPAR
    base = blob_model(params, rects, W, H, psf, n_bands)
    r_all = ((data - base) * inverr).ravel()
    # rows: the pixels some source mask reaches (the others have zero
    # derivatives; their chi^2 is added as is)
    cover = np.zeros((n_bands, H, W), bool)
    for (x0, y0, w, h) in rects:
        cover[:, max(y0, 0):max(min(y0 + h, H), 0), max(x0, 0):max(min(x0 + w, W), 0)] = True
    cover = cover.ravel()
    r = r_all[cover]
    c2_out = float(r_all[~cover] @ r_all[~cover])
    cols = np.zeros((r.size, P))
    h = np.array([1e-5, 1e-5, 0., 0., 0., 1e-6, 1e-6, 1e-6, 1e-6]) if steps is None else steps
    for s in range(n):
        for j in range(BLOB_NPAR):
            if 2 <= j < 5:
                if j - 2 >= n_bands:
                    continue
                one = params[s:s + 1].copy()
                one[0, 2:5] = 0.
                one[0, j] = 1.
                d = blob_model(one, rects[s:s + 1], W, H, psf, n_bands)
            else:
                pp, pm = params.copy(), params.copy()
                pp[s, j] += h[j]
                pm[s, j] -= h[j]
                d = (blob_model(pp[s:s + 1], rects[s:s + 1], W, H, psf, n_bands) -
                     blob_model(pm[s:s + 1], rects[s:s + 1], W, H, psf, n_bands)) / (2 * h[j])
            cols[:, s * BLOB_NPAR + j] = (d * inverr).ravel()[cover]
    return cols.T @ cols, cols.T @ r, float(r @ r) + c2_out


def blob_fit(params0, rects, W, Himg, psf, n_bands, data, inverr, tol=1e-12, max_iter=60,
             lower_n=0.29, upper_n=6.3, frozen=None):
    """FP64 damped Gauss-Newton fit of one blob to a tight optimum (for
    parity: the optimum is a property of the objective, not of the path),
    stopping when the predicted log-likelihood gain of the next step is below
    tol.  `frozen` (bool, the shape of params0) marks parameters held at
    their start values (frozen parameters, tractor/utils.py:195-320).
    Returns (params, H at the optimum, held), `held` marking the parameters
    held at a bound."""
    p = np.array(params0, np.float64)
    fz = np.zeros(p.size, bool) if frozen is None else np.asarray(frozen, bool).ravel()
    H, g, c2 = blob_normal_equations(p, rects, W, Himg, psf, n_bands, data, inverr)
    lam = 1e-3
    for _ in range(max_iter):
        d = np.sqrt(np.maximum(np.diag(H), 0.))
        live = d > 0
        # a Sersic index at a bound that the gradient pushes against is held
        # (projected step: the bound-constrained optimum)
        nidx = np.arange(len(p)) * BLOB_NPAR + 8
        held = ((p[:, 8] >= upper_n) & (g[nidx] > 0)) | ((p[:, 8] <= lower_n) & (g[nidx] < 0))
        live[nidx[held]] = False
        live[fz] = False
        Hs = H[np.ix_(live, live)] / np.outer(d[live], d[live]) + lam * np.eye(live.sum())
        x = np.zeros(len(d))
        xs = np.linalg.solve(Hs, g[live] / d[live])
        x[live] = xs / d[live]
        # predicted log-likelihood gain of the damped step
        pred = 0.5 * (xs @ (g[live] / d[live]) + lam * xs @ xs)
        if pred < tol and lam <= 1.:
            break
        trial = p + x.reshape(p.shape)
        trial[:, 8] = np.clip(trial[:, 8], lower_n, upper_n)
        H2, g2, c22 = blob_normal_equations(trial, rects, W, Himg, psf, n_bands, data,
                                            inverr)
        if c22 <= c2:
            p, H, g, c2 = trial, H2, g2, c22
            lam = max(lam * 0.3, 1e-12)
        else:
            lam *= 10.
            if lam > 1e12:
                break
    nidx = np.arange(len(p)) * BLOB_NPAR + 8
    held = np.zeros(p.size, bool)
    held[nidx] = ((p[:, 8] >= upper_n) & (g[nidx] > 0)) | ((p[:, 8] <= lower_n) & (g[nidx] < 0))
    return p, H, held


# ---------------------------------------------------------------------------
# Fourier path in FP64 throughout (for finite-difference derivative checks)
# ---------------------------------------------------------------------------

def lanczos_shift_f64(img, dx, dy):
    """lanczos_shift_3f's separable Lanczos-3 correlation with zero edges
    (tractor/mp_fourier.i:267-429) in FP64: rows first, then columns;
    out[c] = sum_k taps(dx)[k] in[c - 3 + k]."""
    img = np.asarray(img, np.float64)
    H, W = img.shape
    fx, fy = lanczos3_taps(dx), lanczos3_taps(dy)
    pad = np.zeros((H, W + 6))
    pad[:, 3:W + 3] = img
    tmp = sum(fx[k] * pad[:, k:k + W] for k in range(7))
    pad = np.zeros((H + 6, W))
    pad[3:H + 3, :] = tmp
    return sum(fy[k] * pad[k:k + H, :] for k in range(7))


def galaxy_fft_masked_f64(amp, var2, px, py, psf_img, mask_x0, mask_y0, mw, mh):
    """galaxy_fft_masked without the reference's FP32 roundings (PSF spectrum
    complex128, irfftn output and Lanczos shift in FP64): a smooth function of
    the parameters for central-difference derivative checks."""
    psfh, psfw = psf_img.shape
    hs = fft_halfsize_for_mask(px, py, mask_x0, mask_y0, mw, mh, psfh, psfw)
    sz = fft_size(hs)
    pad, cx, cy = pad_psf(np.asarray(psf_img, np.float64), sz, sz)
    P = np.fft.rfft2(pad)
    v = np.fft.rfftfreq(sz)
    w = np.fft.fftfreq(sz)
    mux = px - cx - mask_x0
    muy = py - cy - mask_y0
    sx = int(np.round(mux))
    sy = int(np.round(muy))
    mux -= sx
    muy -= sy
    G = np.fft.irfftn(fourier_mog(amp, var2, v, w) * P)
    if mux != 0.0 or muy != 0.0:
        G = lanczos_shift_f64(G, mux, muy)
    gh, gw = G.shape
    out = np.zeros((mh, mw))
    ry = overlapping_region(-sy, -sy + mh - 1, 0, gh - 1)
    rx = overlapping_region(-sx, -sx + mw - 1, 0, gw - 1)
    if ry is not None and rx is not None:
        out[ry[1], rx[1]] = G[ry[0], rx[0]]
    return out


def sersic_fft_model_f64(theta, psf_img, mask_x0, mask_y0, mw, mh, shape='E'):
    """FP64 Fourier-path model of a SersicGalaxy, theta = (x, y, counts, s0,
    s1, s2, n) with an EllipseE ('E': re, e1, e2) or EllipseESoft ('ESoft':
    log re, ee1, ee2) shape and NullWCS."""
    x, y, c, s0, s1, s2, n = (float(t) for t in theta)
    amp, var = sersic_profile(n)
    e = (s0, s1, s2) if shape == 'E' else ellipseESoft_to_E(s0, s1, s2)
    T = nullwcs_cdinv() @ ellipseE_basis(*e)
    a2, v2 = sheared(amp, var, T)
    return c * galaxy_fft_masked_f64(a2, v2, x, y, psf_img, mask_x0, mask_y0, mw, mh)


# ---------------------------------------------------------------------------
# EM fit of a Gaussian mixture to an image (tractor/emfit.i)
# ---------------------------------------------------------------------------

def em_fit_2d_reg2(img, x0, y0, amp, mean, var, alpha, steps, approx):
    """em_fit_2d_reg2 (tractor/emfit2.c:1-298): EM with a flat sky term,
    vectorised over pixels.  Each step: per component the symmetrised
    covariance's determinant (a non-positive one returns -1), its inverse,
    amp / sqrt((2 pi)^2 det) and the cut maxD = -2 log(approx sqrt((2 pi)^2
    det)) (emfit2.c:144-166); per pixel: a pixel <= 0 adds |img| to the sky
    and takes no part; z_k = 0 where dsq >= maxD_k; a pixel whose z sum to 0
    adds img to the sky; otherwise the sky's level psky joins the sum and
    img psky / sum goes to the sky, and w_k = img z_k / sum (emfit2.c:
    184-236); then mean = sum w x / sum w, covariance = (alpha I + sum w
    (x - old mean)(x - old mean)^T) / (sum w + alpha), amplitude = sum w,
    and psky = sky sum / npix (emfit2.c:239-248).  psky starts at 0.01 x
    the image mean.  amp / mean / var are updated in place; returns
    (0 or -1, psky)."""
    img = np.asarray(img, np.float64)
    NY, NX = img.shape
    K = len(amp)
    iy, ix = np.mgrid[:NY, :NX]
    x = (x0 + ix).ravel().astype(np.float64)
    y = (y0 + iy).ravel().astype(np.float64)
    I = img.ravel()
    tpd = (2. * np.pi) ** 2
    psky = 0.
    pos = I > 0
    for step in range(steps):
        if step == 0:
            psky = 0.01 * I.sum() / (NX * NY)
        V = var.reshape(K, 4)
        v12 = (V[:, 1] + V[:, 2]) / 2.
        det = V[:, 0] * V[:, 3] - v12 * v12
        if np.any(det <= 0.):
            return -1, psky
        iv0, iv1, iv3 = V[:, 3] / det, -2. * v12 / det, V[:, 0] / det
        scale = amp / np.sqrt(tpd * det)
        maxD = np.log(approx * np.sqrt(tpd * det)) / -0.5
        dx = x[None, :] - mean[:, 0:1]
        dy = y[None, :] - mean[:, 1:2]
        dsq = iv0[:, None] * dx * dx + iv1[:, None] * dx * dy + iv3[:, None] * dy * dy
        Z = np.where(dsq >= maxD[:, None], 0.,
                     scale[:, None] * np.exp(-0.5 * np.where(dsq >= maxD[:, None], 0., dsq)))
        zsum = np.zeros_like(I)
        for k in range(K):
            zsum = zsum + Z[k]
        used = pos & (zsum != 0)
        sky = np.abs(I[~pos]).sum() + I[pos & (zsum == 0)].sum()
        zs = zsum[used] + psky
        sky += (I[used] * (psky / zs)).sum()
        W = np.zeros((K, len(I)))
        W[:, used] = I[used][None, :] * Z[:, used] / zs[None, :]
        wsum = W.sum(axis=1)
        sx = (W * x[None, :]).sum(axis=1)
        sy = (W * y[None, :]).sum(axis=1)
        vxx = alpha + (W * dx * dx).sum(axis=1)
        vxy = (W * dx * dy).sum(axis=1)
        vyy = alpha + (W * dy * dy).sum(axis=1)
        mean[:, 0] = sx / wsum
        mean[:, 1] = sy / wsum
        den = wsum + alpha
        var[:, 0, 0] = vxx / den
        var[:, 0, 1] = vxy / den
        var[:, 1, 0] = vxy / den
        var[:, 1, 1] = vyy / den
        amp[:] = wsum
        psky = sky / (NX * NY)
    return 0, psky


def em_fit_2d_reg(img, x0, y0, amp, mean, var, alpha, steps):
    """em_fit_2d_reg (tractor/emfit.i:274-557), vectorised over pixels: each
    step computes C^-1 and amp / sqrt((2 pi)^2 det) (a non-positive
    determinant returns -1, emfit.i:403-409), the responsibilities
    z_k / sum_j z_j with z = 0 where dsq >= 100 (a pixel whose sum is 0
    keeps its unnormalised z, emfit.i:424-454), then the mean, the
    covariance about the new mean with the alpha prior and the amplitude
    (emfit.i:460-509).  amp / mean / var (float64) are updated in place;
    returns 0 or -1."""
    img = np.asarray(img, np.float64)
    NY, NX = img.shape
    K = len(amp)
    iy, ix = np.mgrid[:NY, :NX]
    x = (x0 + ix).ravel().astype(np.float64)
    y = (y0 + iy).ravel().astype(np.float64)
    I = img.ravel()
    tpd = (2. * np.pi) ** 2
    for step in range(steps):
        V = var.reshape(K, 4)
        det = V[:, 0] * V[:, 3] - V[:, 1] * V[:, 2]
        if np.any(det <= 0.):
            return -1
        iv = np.stack([V[:, 3] / det, -V[:, 1] / det, -V[:, 2] / det, V[:, 0] / det], 1)
        scale = amp / np.sqrt(tpd * det)
        dx = x[None, :] - mean[:, 0:1]
        dy = y[None, :] - mean[:, 1:2]
        dsq = (iv[:, 0:1] * dx * dx + iv[:, 1:2] * dx * dy + iv[:, 2:3] * dx * dy +
               iv[:, 3:4] * dy * dy)
        Z = np.where(dsq >= 100, 0., scale[:, None] * np.exp(-0.5 * np.minimum(dsq, 100.)))
        zsum = np.zeros_like(I)
        for k in range(K):
            zsum = zsum + Z[k]
        nz = zsum != 0
        Z[:, nz] = Z[:, nz] / zsum[nz]
        W = I[None, :] * Z
        wsum = W.sum(axis=1)
        mx = (W * x[None, :]).sum(axis=1) / wsum
        my = (W * y[None, :]).sum(axis=1) / wsum
        mean[:, 0] = mx
        mean[:, 1] = my
        ddx = x[None, :] - mx[:, None]
        ddy = y[None, :] - my[:, None]
        vxx = alpha + (W * ddx * ddx).sum(axis=1)
        vxy = (W * ddx * ddy).sum(axis=1)
        vyy = alpha + (W * ddy * ddy).sum(axis=1)
        den = wsum + alpha
        var[:, 0, 0] = vxx / den
        var[:, 0, 1] = vxy / den
        var[:, 1, 0] = vxy / den
        var[:, 1, 1] = vyy / den
        amp[:] = wsum
    return 0
