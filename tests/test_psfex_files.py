"""PsfEx model files: the numpy FITS binary-table reader / writer
(tractor_b200.fitsbin) and PsfExModel / PixelizedPsfEx built from files.

The reference's own test data (test/psfex-decam-00392360-S31.fits and the
two .psf files) are read where the reference tree is present (marked
`reference`): the models must satisfy the reference test's expectations
(tractor test/test_psfex.py: the image varies over the chip, getShifted
reproduces it exactly, writeto + read returns it exactly), and the
reference's own PsfExModel, reading the same file through the same table
reader, must agree with ours attribute by attribute."""
import os
import types

import numpy as np
import pytest

def _ref_test_dir():
    from oracle import refharness
    return os.path.join(refharness.reference_root() or '', 'test')


REF_TEST = _ref_test_dir()
FILES = ['psfex-decam-00392360-S31.fits', 'c4d_140717_065122_ooi_i_ls11-S2-se.psf']
OVERSAMPLED = 'c4d_140818_002108_ooi_z_v1.ext27.psf'


def test_fits_table_round_trip(tmp_path):
    from tractor_b200 import fitsbin
    rng = np.random.default_rng(3)
    cols = {'psf_mask': rng.normal(size=(2, 3, 5, 7)).astype(np.float32),
            'flux': rng.normal(size=(2,)),
            'ids': np.array([[1, 2], [3, 4]], np.int32)}
    hdr = {'POLNAME1': 'X_IMAGE', 'POLDEG1': 3, 'PSF_SAMP': 1.25, 'PSF_FWHM': 4.5,
           'FLAG': True, 'NOTE': "it's"}
    fn = str(tmp_path / 't.fits')
    fitsbin.write_table(fn, cols, hdr)
    h, got = fitsbin.read_table(fn)
    for k, v in cols.items():
        assert got[k].dtype == v.dtype and np.array_equal(got[k], v)
    for k, v in hdr.items():
        assert h[k] == v
    assert os.path.getsize(fn) % 2880 == 0


def test_psfex_model_write_read(tmp_path):
    from tractor_b200.psfex import PsfExModel, PixelizedPsfEx
    rng = np.random.default_rng(4)
    bases = rng.normal(size=(6, 15, 15)).astype(np.float32)
    m = PsfExModel(bases=bases, degree=2, x0=40., y0=30., xscale=100., yscale=80., fwhm=3.5)
    fn = str(tmp_path / 'm.psf')
    m.writeto(fn)
    r = PsfExModel(fn)
    assert r.degree == 2 and np.array_equal(r.psfbases, bases)
    assert (r.x0, r.y0, r.xscale, r.yscale, r.sampling, r.fwhm) == (40., 30., 100., 80., 1., 3.5)
    p = PixelizedPsfEx(fn)
    assert np.array_equal(p.getImage(12.5, 70.), m.at(12.5, 70.))


def _ref_file(name):
    fn = os.path.join(REF_TEST, name)
    if not os.path.isfile(fn):
        pytest.skip('reference test data not present')
    return fn


@pytest.mark.reference
@pytest.mark.parametrize('name', FILES)
def test_reference_psfex_files(name, tmp_path):
    from tractor_b200.psfex import PixelizedPsfEx, PsfExModel
    psf = PixelizedPsfEx(_ref_file(name))
    # spatial variation (test_psfex.py:43-53)
    dx, dy = 50., 100.
    im0, im = psf.getImage(0., 0.), psf.getImage(dx, dy)
    rms = np.sqrt(np.mean((im0 - im) ** 2))
    assert 0 < rms < 1e-4
    # getShifted (test_psfex.py:55-58)
    sub = psf.getShifted(dx, dy)
    assert np.sqrt(np.mean((sub.getImage(0., 0.) - im) ** 2)) == 0.
    # writeto + read (test_psfex.py:60-76)
    fn = str(tmp_path / 'rt.fits')
    psf.psfex.writeto(fn)
    psf2 = PixelizedPsfEx(None, psfex=PsfExModel(fn=fn))
    assert np.max(np.abs(psf.getImage(0., 0.) - psf2.getImage(0., 0.))) == 0.


@pytest.mark.reference
def test_oversampled_psfex_file_is_refused():
    from tractor_b200.psfex import PixelizedPsfEx, PsfExModel
    fn = _ref_file(OVERSAMPLED)
    m = PsfExModel(fn)
    assert m.sampling != 1. and m.degree == 6
    with pytest.raises(NotImplementedError):
        PixelizedPsfEx(fn)


@pytest.mark.reference
@pytest.mark.parametrize('name', FILES + [OVERSAMPLED])
def test_reference_reader_logic_agrees(name):
    """The reference's PsfExModel(fn) (psfex.py:160-206), given the file's
    table through the same reader, builds the same model."""
    from oracle import refharness
    if not refharness.available():
        pytest.skip('reference source tree not present')
    fn = _ref_file(name)
    refharness.load()
    import sys
    from tractor_b200 import fitsbin
    from tractor_b200.psfex import PsfExModel

    class _Table(object):
        def __init__(self, fn, ext=1):
            self._hdr, cols = fitsbin.read_table(fn, ext)
            for k, v in cols.items():
                setattr(self, k, v)

        def get_header(self):
            return self._hdr

    fits_mod = types.ModuleType('astrometry.util.fits')
    fits_mod.fits_table = _Table
    old = sys.modules.get('astrometry.util.fits')
    sys.modules['astrometry.util.fits'] = fits_mod
    try:
        from tractor.psfex import PsfExModel as RefModel
        ref = RefModel(fn=fn)
    finally:
        if old is not None:
            sys.modules['astrometry.util.fits'] = old
    ours = PsfExModel(fn)
    assert np.array_equal(ours.psfbases, ref.psfbases)
    for k in ('degree', 'x0', 'y0', 'xscale', 'yscale', 'sampling', 'radius', 'fwhm'):
        assert getattr(ours, k) == getattr(ref, k), k
    for x, y in [(0., 0.), (1000., 2000.), (1500.5, 300.25)]:
        assert np.array_equal(ours.at(x, y), ref.at(x, y))
