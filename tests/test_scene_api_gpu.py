"""Tractor.getModelImage through the scene renderer: a catalog of 64 or more
sources with rectangular model masks on a mixture-of-Gaussians-PSF image is
rendered as one scene (tb_scene_render) and must reproduce the reference's
own getModelImage (tests/golden/scene_mog.npz) and the per-source path.

Tolerance: model pixels within 1e-5 of the image's peak."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def _tractor_from_golden(g):
    from tractor_b200 import (Tractor, Image, PixPos, Flux, LinearPhotoCal, GaussianMixturePSF,
                              PointSource, ExpGalaxy, DevGalaxy, FixedCompositeGalaxy, EllipseE,
                              ModelMask)
    H, W = (int(v) for v in g['shape'])
    pamp = np.asarray(g['psf_amp'], np.float64)
    psig = np.asarray(g['psf_sigma'], np.float64)
    psf = GaussianMixturePSF(pamp, np.zeros((3, 2)), np.array([np.eye(2) * s ** 2 for s in psig]))
    tim = Image(data=np.zeros((H, W), np.float32), inverr=np.ones((H, W), np.float32), psf=psf,
                photocal=LinearPhotoCal(1.))
    srcs, masks = [], {}
    for row in g['sources']:
        kind = int(row[0])
        pos, br = PixPos(row[1], row[2]), Flux(row[3])
        ea, eb = EllipseE(*row[9:12]), EllipseE(*row[12:15])
        if kind == 0:
            s = PointSource(pos, br)
        elif kind == 1:
            s = ExpGalaxy(pos, br, ea)
        elif kind == 2:
            s = DevGalaxy(pos, br, ea)
        else:
            s = FixedCompositeGalaxy(pos, br, row[8], ea, eb)
        masks[s] = ModelMask(int(row[4]), int(row[5]), int(row[6]), int(row[7]))
        srcs.append(s)
    tr = Tractor([tim], srcs)
    tr.setModelMasks([masks])
    return tr


def test_getModelImage_scene_path_matches_reference(tb):
    g = np.load(os.path.join(GOLDEN, 'scene_mog.npz'))
    tr = _tractor_from_golden(g)
    assert len(tr.catalog) >= tr.SCENE_MIN_SOURCES
    assert tr._scene_records(tr.getImage(0), list(tr.catalog), None) is not None
    mod = tr.getModelImage(0)
    ref = g['model'].astype(np.float64)
    assert mod.dtype == np.float32
    assert np.abs(mod - ref).max() < 1e-5 * np.abs(ref).max()
    # the per-source path gives the same image
    tr.SCENE_MIN_SOURCES = 10 ** 9
    mod2 = tr.getModelImage(0)
    assert np.abs(mod2.astype(np.float64) - mod).max() < 1e-5 * np.abs(ref).max()
