"""Test infrastructure (oracle only): import the unmodified reference Tractor
package from its source tree, with its SWIG extensions replaced by the
reference's own C compiled by oracle/build_ref.sh.

This runs only where the reference tree exists (the development container);
tests that need it skip elsewhere.  It is used to generate the golden fixtures
under tests/golden/ and to pin the oracle restatement against the reference.

What is shimmed, and why:
  * tractor.mix / tractor.mp_fourier / tractor.emfit -- the SWIG modules.  Each shim function
    calls the reference's C entry point with the same arguments SWIG would
    pass (tractor/mix.i:311 makes c_gauss_2d_approx3 return
    (rtn, sx0, sx1, sy0, sy1)).
  * tractor.version -- generated by the reference's setup.py.
  * astrometry.util.miscutils.get_overlapping_region -- mirrors the
    reference's own copy in tractor/patch.pyx:20-65 (absolute slices).
  * astrometry.util.miscutils.lanczos_filter -- the un-normalised kernel, as
    tractor/psf.py:45-46 normalises after calling it (used only for images
    of side <= 8).
  * astrometry.util.ttime.Time and plotting / fitsio modules -- imported by
    off-path modules only.
"""
import ctypes
import os
import sys
import types

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REFLIB = os.path.join(_HERE, '_ref')


def reference_root():
    """The reference source tree: $TRACTOR_REFERENCE_ROOT, else the tree
    oracle/build_ref.sh compiled from (recorded in oracle/_ref/REFERENCE_ROOT),
    else None (no reference on this machine)."""
    env = os.environ.get('TRACTOR_REFERENCE_ROOT')
    if env:
        return env
    try:
        with open(os.path.join(_REFLIB, 'REFERENCE_ROOT')) as f:
            return f.read().strip() or None
    except OSError:
        return None


REFERENCE_ROOT = reference_root() or ''

_loaded = None


def available():
    return (os.path.isfile(os.path.join(REFERENCE_ROOT, 'tractor', 'engine.py'))
            and os.path.isfile(os.path.join(_REFLIB, 'libref_mix.so')))


def _mix_module():
    lib = ctypes.PyDLL(os.path.join(_REFLIB, 'libref_mix.so'))
    if lib.ref_mix_init() != 0:
        raise RuntimeError('numpy C-API init failed in libref_mix.so')
    P = ctypes.py_object
    I = ctypes.c_int
    D = ctypes.c_double
    lib.ref_c_gauss_2d_grid.argtypes = [I, I, I, I, D, D, P, P, P, P]
    lib.ref_c_gauss_2d_grid.restype = I
    lib.ref_c_gauss_2d_approx3.argtypes = ([I, I, I, I, D, D, D, P, P, P, P, P, P,
                                            I, I, I] + [ctypes.POINTER(I)] * 4)
    lib.ref_c_gauss_2d_approx3.restype = I
    lib.ref_c_gauss_2d_masked.argtypes = [I, I, I, I, D, D, P, P, P, P, P, P, P]
    lib.ref_c_gauss_2d_masked.restype = I

    m = types.ModuleType('tractor.mix')

    def c_gauss_2d_grid(x0, x1, y0, y1, fx, fy, amp, mean, var, result):
        return lib.ref_c_gauss_2d_grid(int(x0), int(x1), int(y0), int(y1),
                                       float(fx), float(fy), amp, mean, var, result)

    def c_gauss_2d_approx3(x0, x1, y0, y1, fx, fy, minval, amp, mean, var,
                           result, xderiv, yderiv, xc, yc, minradius):
        s = [I(0) for _ in range(4)]
        r = lib.ref_c_gauss_2d_approx3(int(x0), int(x1), int(y0), int(y1),
                                       float(fx), float(fy), float(minval),
                                       amp, mean, var, result, xderiv, yderiv,
                                       int(xc), int(yc), int(minradius),
                                       *[ctypes.byref(v) for v in s])
        return (r,) + tuple(v.value for v in s)

    def c_gauss_2d_masked(x0, y0, W, H, fx, fy, amp, mean, var, result,
                          xderiv, yderiv, mask):
        return lib.ref_c_gauss_2d_masked(int(x0), int(y0), int(W), int(H),
                                         float(fx), float(fy), amp, mean, var,
                                         result, xderiv, yderiv, mask)

    m.c_gauss_2d_grid = c_gauss_2d_grid
    m.c_gauss_2d_approx3 = c_gauss_2d_approx3
    m.c_gauss_2d_masked = c_gauss_2d_masked
    m._lib = lib
    return m


def _f32(a):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _f64(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _mpf_module():
    lib = ctypes.CDLL(os.path.join(_REFLIB, 'libref_mpf.so'))
    m = types.ModuleType('tractor.mp_fourier')

    def lanczos_shift_3f(inimg, outimg, dx, dy, work):
        inimg = np.ascontiguousarray(inimg, np.float32)
        lib.ref_lanczos_shift_3f(_f32(inimg), inimg.shape[0], inimg.shape[1],
                                 _f32(outimg), outimg.shape[0], outimg.shape[1],
                                 ctypes.c_double(dx), ctypes.c_double(dy),
                                 _f32(work), work.shape[0], work.shape[1])

    def correlate7f(img, filtx, filty, work):
        filtx = np.ascontiguousarray(filtx, np.float64)
        filty = np.ascontiguousarray(filty, np.float64)
        lib.ref_correlate7f(_f32(img), img.shape[0], img.shape[1],
                            _f64(filtx), len(filtx), _f64(filty), len(filty),
                            _f32(work), work.shape[0], work.shape[1])

    def correlate7f_inout(inimg, outimg, filtx, filty, work):
        filtx = np.ascontiguousarray(filtx, np.float64)
        filty = np.ascontiguousarray(filty, np.float64)
        lib.ref_correlate7f_inout(_f32(inimg), inimg.shape[0], inimg.shape[1],
                                  _f32(outimg), outimg.shape[0], outimg.shape[1],
                                  _f64(filtx), 7, _f64(filty), 7,
                                  _f32(work), work.shape[0], work.shape[1])

    def lanczos_filter_3(dx):
        f = np.zeros(7, np.float64)
        lib.ref_lanczos_filter_3(_f64(f), ctypes.c_double(dx))
        return f

    def gaussian_fourier_transform_zero_mean(amps, vars, v, w, out):
        amps = np.ascontiguousarray(amps, np.float64)
        vars = np.ascontiguousarray(vars, np.float64)
        v = np.ascontiguousarray(v, np.float64)
        w = np.ascontiguousarray(w, np.float64)
        K = len(amps)
        lib.ref_gaussian_fourier_transform_zero_mean(
            _f64(amps), K, _f64(vars), vars.shape[0], vars.shape[1], vars.shape[2],
            _f64(v), len(v), _f64(w), len(w), _f64(out), out.shape[0], out.shape[1])

    m.lanczos_shift_3f = lanczos_shift_3f
    m.correlate7f = correlate7f
    m.correlate7f_inout = correlate7f_inout
    m.lanczos_filter_3 = lanczos_filter_3
    m.gaussian_fourier_transform_zero_mean = gaussian_fourier_transform_zero_mean
    m._lib = lib
    return m


def _emfit_module():
    lib = ctypes.PyDLL(os.path.join(_REFLIB, 'libref_emfit.so'))
    if lib.ref_emfit_init() != 0:
        raise RuntimeError('numpy C-API init failed in libref_emfit.so')
    P = ctypes.py_object
    I = ctypes.c_int
    D = ctypes.c_double
    lib.ref_em_fit_2d_reg.argtypes = [P, I, I, P, P, P, D, I]
    lib.ref_em_fit_2d_reg.restype = I
    m = types.ModuleType('tractor.emfit')

    def em_fit_2d_reg(img, x0, y0, amp, mean, var, alpha, steps):
        return lib.ref_em_fit_2d_reg(img, int(x0), int(y0), amp, mean, var, float(alpha),
                                     int(steps))

    lib.ref_em_fit_2d_reg2.argtypes = [P, I, I, P, P, P, D, I, D, ctypes.POINTER(D)]
    lib.ref_em_fit_2d_reg2.restype = I

    def em_fit_2d_reg2(img, x0, y0, amp, mean, var, alpha, steps, approx):
        # SWIG's double* OUTPUT: returns [status, skyamp]
        sky = D(0.)
        r = lib.ref_em_fit_2d_reg2(img, int(x0), int(y0), amp, mean, var, float(alpha),
                                   int(steps), float(approx), ctypes.byref(sky))
        return [r, sky.value]

    m.em_fit_2d_reg = em_fit_2d_reg
    m.em_fit_2d_reg2 = em_fit_2d_reg2
    m._lib = lib
    return m


def _get_overlapping_region(xlo, xhi, xmin, xmax):
    # Same contract as tractor/patch.pyx:20-65.
    if xlo > xmax or xhi < xmin or xlo > xhi or xmin > xmax:
        return ([], [])
    xloclamp = max(xlo, xmin)
    Xlo = xloclamp - xlo
    xhiclamp = min(xhi, xmax)
    Xhi = Xlo + (xhiclamp - xloclamp)
    return (slice(xloclamp, xhiclamp + 1), slice(Xlo, Xhi + 1))


def _lanczos_filter_unnormalised(order, x):
    x = np.atleast_1d(np.asarray(x, np.float64))
    out = np.zeros(x.shape, np.float64)
    nz = (x != 0) & (np.abs(x) < order)
    px = np.pi * x[nz]
    out[nz] = order * np.sin(px) * np.sin(px / order) / px**2
    out[x == 0] = 1.
    return out


class _Time(object):
    def __init__(self):
        pass

    def __sub__(self, other):
        return 0.

    def __str__(self):
        return ''


def _install_shims():
    mods = {}
    tmix = _mix_module()
    tmpf = _mpf_module()
    ver = types.ModuleType('tractor.version')
    ver.version = 'reference-source'
    mods['tractor.mix'] = tmix
    mods['tractor.mp_fourier'] = tmpf
    mods['tractor.version'] = ver
    if os.path.isfile(os.path.join(_REFLIB, 'libref_emfit.so')):
        mods['tractor.emfit'] = _emfit_module()

    astro = types.ModuleType('astrometry')
    astro.__path__ = []
    util = types.ModuleType('astrometry.util')
    util.__path__ = []
    misc = types.ModuleType('astrometry.util.miscutils')
    misc.get_overlapping_region = _get_overlapping_region
    misc.lanczos_filter = _lanczos_filter_unnormalised
    ttime = types.ModuleType('astrometry.util.ttime')
    ttime.Time = _Time
    mods.update({'astrometry': astro, 'astrometry.util': util,
                 'astrometry.util.miscutils': misc,
                 'astrometry.util.ttime': ttime})
    # Off-path imports pulled in by `from tractor import *`.
    for name in ['tractor.emfit', 'pylab', 'fitsio', 'astrometry.util.starutil_numpy',
                 'astrometry.util.util', 'astrometry.util.fits',
                 'astrometry.sdss', 'astrometry.libkd',
                 'astrometry.libkd.spherematch', 'astrometry.util.plotutils',
                 'astrometry.util.multiproc']:
        if name not in sys.modules and name not in mods:
            mods[name] = _Stub(name)
    try:
        import matplotlib  # noqa: F401
    except ImportError:
        mods['matplotlib'] = _Stub('matplotlib')
    for k, v in mods.items():
        sys.modules.setdefault(k, v)
    return tmix, tmpf


class _Stub(types.ModuleType):
    def __init__(self, name):
        super().__init__(name)
        self.__path__ = []

    def __getattr__(self, name):
        if name.startswith('__'):
            raise AttributeError(name)
        return _Stub(self.__name__ + '.' + name)

    def __call__(self, *a, **k):
        return None


def load():
    """Import and return the reference `tractor` package (FP64 model type is
    set by callers via Tractor.modtype)."""
    global _loaded
    if _loaded is not None:
        return _loaded
    if not available():
        raise RuntimeError('reference tree or oracle/_ref libraries not present')
    if 'tractor' in sys.modules and not getattr(sys.modules['tractor'], '_from_reference', False):
        raise RuntimeError('another package named tractor is already imported')
    _install_shims()
    sys.path.insert(0, REFERENCE_ROOT)
    try:
        import tractor
        import tractor.sersic  # noqa: F401
        import tractor.galaxy  # noqa: F401
        import tractor.psf  # noqa: F401
        import tractor.constrained_optimizer  # noqa: F401
        import tractor.lsqr_optimizer  # noqa: F401
        import tractor.mixture_profiles  # noqa: F401
        import tractor.ellipses  # noqa: F401
    finally:
        sys.path.remove(REFERENCE_ROOT)
    tractor._from_reference = True
    # Stubbed submodules named in tractor.__all__ must be package attributes
    # for `from tractor import *` to work.
    tractor.emfit = sys.modules['tractor.emfit']
    _loaded = tractor
    return tractor
