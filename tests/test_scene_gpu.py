"""Scene rendering (tb_scene_prep + tb_scene_render): many point / exp / deV /
composite / Sersic sources into whole images through mixture-of-Gaussians
PSFs, against the reference's own Tractor.getModelImage (the golden scene of
tests/golden/make_golden.py) and against the oracle.

Tolerance: model pixels within 1e-5 of the image's peak."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')
PEAK_TOL = 1e-5


def golden_rows_to_records(rows, image=0):
    """scene_mog.npz rows (kind, px, py, flux, mx0, my0, mw, mh, fracDev,
    exp-or-single (re, e1, e2), deV (re, e1, e2)) -> SCENE_SRC records."""
    from tractor_b200 import _lib
    rows = np.asarray(rows, np.float64)
    s = np.zeros(len(rows), _lib.SCENE_SRC)
    kinds = np.array([_lib.PROFILE_POINT, _lib.PROFILE_EXP, _lib.PROFILE_DEV,
                      _lib.PROFILE_COMPOSITE])
    s['profile'] = kinds[rows[:, 0].astype(int)]
    s['px'], s['py'], s['counts'] = rows[:, 1], rows[:, 2], rows[:, 3]
    s['mx0'], s['my0'], s['mw'], s['mh'] = (rows[:, 4 + k].astype(int) for k in range(4))
    s['fdev'] = rows[:, 8]
    s['sa0'], s['sa1'], s['sa2'] = rows[:, 9], rows[:, 10], rows[:, 11]
    s['sb0'], s['sb1'], s['sb2'] = rows[:, 12], rows[:, 13], rows[:, 14]
    s['shape_type'] = _lib.SHAPE_ELLIPSE_E
    s['image'] = image
    return s


def records_to_rows(s):
    """Inverse of golden_rows_to_records (for the oracle's scene_model)."""
    from tractor_b200 import _lib
    kind = {_lib.PROFILE_POINT: 0, _lib.PROFILE_EXP: 1, _lib.PROFILE_DEV: 2,
            _lib.PROFILE_COMPOSITE: 3}
    return np.array([[kind[int(r['profile'])], r['px'], r['py'], r['counts'], r['mx0'], r['my0'],
                      r['mw'], r['mh'], r['fdev'], r['sa0'], r['sa1'], r['sa2'], r['sb0'],
                      r['sb1'], r['sb2']] for r in s])


def _peak_err(got, ref):
    return np.abs(got.astype(np.float64) - ref).max() / np.abs(ref).max()


def test_scene_matches_reference_golden(tb):
    """80 mixed sources with square model masks on a 256 x 320 image,
    3-component MoG PSF: the reference's Tractor.getModelImage."""
    from tractor_b200 import batch
    g = np.load(os.path.join(GOLDEN, 'scene_mog.npz'))
    H, W = (int(v) for v in g['shape'])
    img = batch.SceneImage.circular(W, H, g['psf_sigma'], g['psf_amp'])
    r = batch.SceneRenderer([img])
    recs = golden_rows_to_records(g['sources'])
    for th in batch.SCENE_TILE_HEIGHTS:
        out = r.render(recs, tile_h=th).numpy()
        got = r.image(out, 0)
        assert _peak_err(got, g['model']) < PEAK_TOL, th
    flags = r.items(len(recs))['flag']
    assert np.all(flags == 0)


def test_render_is_deterministic_and_tile_shape_independent(tb):
    """Per-pixel summation order (sources in catalog order, components in
    mixture order) does not depend on scheduling: repeated renders are
    bit-identical.  Tile heights change only the FP32 rounding of the
    tile-relative means (far below the tolerance)."""
    from tractor_b200 import batch
    rng = np.random.default_rng(5)
    img = batch.SceneImage.circular(700, 530, [1.3, 2.6, 5.2], [0.7, 0.2, 0.1])
    recs = batch.scene_sources(600, rng, W=700, H=530, hw_range=(4, 90))
    r = batch.SceneRenderer([img])
    outs = {th: r.render(recs, tile_h=th).numpy().copy() for th in batch.SCENE_TILE_HEIGHTS}
    for th in batch.SCENE_TILE_HEIGHTS:
        assert np.array_equal(r.render(recs, tile_h=th).numpy(), outs[th]), th
        assert _peak_err(outs[th], outs[32].astype(np.float64)) < 1e-6, th


def test_multi_image_scene_matches_oracle(tb, oracle):
    """Three images (bands) of different sizes and PSFs, sources seen in
    several images with per-image counts and masks, some masks partly or
    entirely off their image."""
    from tractor_b200 import batch
    rng = np.random.default_rng(17)
    shapes = [(160, 200), (97, 131), (64, 300)]
    sig = [[1.1, 2.2, 4.4], [1.7, 3.4, 6.8], [0.9, 1.8, 3.6]]
    wts = [[0.7, 0.2, 0.1], [0.6, 0.3, 0.1], [0.8, 0.15, 0.05]]
    imgs = [batch.SceneImage.circular(W, H, s, w) for (H, W), s, w in zip(shapes, sig, wts)]
    recs = []
    for i, (H, W) in enumerate(shapes):
        s = batch.scene_sources(40, rng, W=W, H=H, image=i, hw_range=(3, 50))
        s['mx0'] -= rng.integers(-3, 4, len(s))
        recs.append(s)
    recs = np.concatenate(recs)
    recs[5]['mx0'] = -500   # mask entirely off its image: no patch
    r = batch.SceneRenderer(imgs)
    out = r.render(recs).numpy()
    for i, (H, W) in enumerate(shapes):
        sel = recs[(recs['image'] == i)]
        sel = sel[sel['mx0'] > -400]
        # the oracle renders masks inside the image: clip them as Patch.addTo does
        rows = records_to_rows(sel)
        x0 = np.maximum(rows[:, 4], 0)
        y0 = np.maximum(rows[:, 5], 0)
        x1 = np.minimum(rows[:, 4] + rows[:, 6], W)
        y1 = np.minimum(rows[:, 5] + rows[:, 7], H)
        keep = (x1 > x0) & (y1 > y0)
        rows[:, 4], rows[:, 5], rows[:, 6], rows[:, 7] = x0, y0, x1 - x0, y1 - y0
        ref = oracle.scene_model(rows[keep], wts[i], sig[i], H, W)
        assert _peak_err(r.image(out, i), ref) < PEAK_TOL, i
    flags = r.items(len(recs))['flag']
    assert flags[5] == 1
    assert np.sum(flags == 0) == len(recs) - 1


def test_sersic_and_composite_edge_cases(tb, oracle):
    """Sersic sources across the index ranges (delta core for n > 1),
    composites with fracDev 0, 1 and outside [0, 1], zero counts."""
    from tractor_b200 import batch, _lib
    rng = np.random.default_rng(23)
    W, H = 120, 90
    img = batch.SceneImage.circular(W, H, [1.4, 2.8], [0.8, 0.2])
    s = batch.scene_sources(24, rng, W=W, H=H, hw_range=(6, 30), mix=(0., 0., 0., 1.))
    s['fdev'][:6] = [0., 1., -0.3, 1.7, 0.5, 0.999]
    s['counts'][6] = 0.
    ser = batch.scene_sources(12, rng, W=W, H=H, hw_range=(6, 30))
    ser['profile'] = _lib.PROFILE_SERSIC
    ser['sersic_n'] = np.linspace(0.3, 6.2, 12)
    recs = np.concatenate([s, ser])
    r = batch.SceneRenderer([img])
    got = r.image(r.render(recs).numpy(), 0).astype(np.float64)
    ref = np.zeros((H, W))
    pa = np.array([0.8, 0.2])
    pm = np.zeros((2, 2))
    pv = np.zeros((2, 2, 2))
    pv[:, 0, 0] = pv[:, 1, 1] = np.array([1.4, 2.8]) ** 2
    for q in recs:
        if q['counts'] == 0:
            continue
        x0, y0 = max(q['mx0'], 0), max(q['my0'], 0)
        x1, y1 = min(q['mx0'] + q['mw'], W), min(q['my0'] + q['mh'], H)
        if x1 <= x0 or y1 <= y0:
            continue
        if q['profile'] == _lib.PROFILE_SERSIC:
            amp, var = oracle.sersic_profile(float(q['sersic_n']))
            T = oracle.nullwcs_cdinv() @ oracle.ellipseE_basis(q['sa0'], q['sa1'], q['sa2'])
            a2, v2 = oracle.sheared(amp, var, T)
            ca, cm, cv = oracle.convolve(a2, np.zeros((len(a2), 2)) + [q['px'], q['py']], v2,
                                         pa, pm, pv)
            fx = fy = 0.
        else:
            ca, cm, cv, fx, fy = oracle.scene_source_mixture(
                3, q['px'], q['py'], q['fdev'], [q['sa0'], q['sa1'], q['sa2']],
                [q['sb0'], q['sb1'], q['sb2']], pa, pm, pv)
        ref[y0:y1, x0:x1] += oracle.mog_grid(x0, x1, y0, y1, fx, fy, ca, cm, cv) * q['counts']
    assert _peak_err(got, ref) < PEAK_TOL
    assert r.items(len(recs))['flag'][6] == 1


def test_full_size_scene_windows_match_oracle(tb, oracle):
    """The batched-render workload at full size (20,000 sources on one
    4096 x 4096 image, half-widths 7-127 px): the whole image renders in one
    call, and randomly placed 48 x 48 windows match the oracle summed over
    every source reaching them."""
    from tractor_b200 import batch
    rng = np.random.default_rng(3)
    W = H = 4096
    sig = rng.uniform(1., 2.)
    sigmas, wts = [sig, 2 * sig, 4 * sig], [0.7, 0.2, 0.1]
    img = batch.SceneImage.circular(W, H, sigmas, wts)
    recs = batch.scene_sources(20000, rng)
    r = batch.SceneRenderer([img])
    got = r.image(r.render(recs).numpy(), 0)
    assert np.all(np.isfinite(got))
    rows = records_to_rows(recs)
    pa = np.asarray(wts, np.float64)
    pm = np.zeros((3, 2))
    pv = np.zeros((3, 2, 2))
    pv[:, 0, 0] = pv[:, 1, 1] = np.asarray(sigmas) ** 2
    x0s, y0s = rows[:, 4].astype(int), rows[:, 5].astype(int)
    x1s, y1s = x0s + rows[:, 6].astype(int), y0s + rows[:, 7].astype(int)
    for _ in range(6):
        wx, wy = int(rng.integers(0, W - 48)), int(rng.integers(0, H - 48))
        ref = np.zeros((48, 48))
        near = np.flatnonzero((x1s > wx) & (x0s < wx + 48) & (y1s > wy) & (y0s < wy + 48))
        for q in near:
            row = rows[q]
            x0, y0 = max(x0s[q], wx, 0), max(y0s[q], wy, 0)
            x1, y1 = min(x1s[q], wx + 48, W), min(y1s[q], wy + 48, H)
            ca, cm, cv, fx, fy = oracle.scene_source_mixture(int(row[0]), row[1], row[2], row[8],
                                                             row[9:12], row[12:15], pa, pm, pv)
            ref[y0 - wy:y1 - wy, x0 - wx:x1 - wx] += oracle.mog_grid(x0, x1, y0, y1, fx, fy, ca,
                                                                     cm, cv) * row[3]
        win = got[wy:wy + 48, wx:wx + 48].astype(np.float64)
        if len(near):
            assert _peak_err(win, ref) < PEAK_TOL, (wx, wy)
        else:
            assert np.all(win == 0)
