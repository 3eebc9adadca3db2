"""Host-side logic of the scene renderer (no GPU): the (record, tile)
overlap bound that sizes the tile lists, and the synthetic scene generator."""
import numpy as np


def test_max_pairs_counts_every_overlapped_tile():
    from tractor_b200 import batch
    rng = np.random.default_rng(0)
    r = batch.SceneRenderer.__new__(batch.SceneRenderer)
    r.images = [batch.SceneImage.circular(300, 200, [1.], [1.]),
                batch.SceneImage.circular(65, 33, [1.], [1.])]
    recs = np.concatenate([batch.scene_sources(50, rng, W=300, H=200, image=0),
                           batch.scene_sources(20, rng, W=65, H=33, image=1, hw_range=(1, 40))])
    recs['mx0'][:5] = [-400, 299, -10, 0, 5]
    for th in batch.SCENE_TILE_HEIGHTS:
        want = 0
        for q in recs:
            im = r.images[q['image']]
            for ty in range((im.H + th - 1) // th):
                for tx in range((im.W + 31) // 32):
                    x0, x1 = max(q['mx0'], tx * 32), min(q['mx0'] + q['mw'], tx * 32 + 32, im.W)
                    y0, y1 = max(q['my0'], ty * th), min(q['my0'] + q['mh'], ty * th + th, im.H)
                    want += (x1 > max(x0, 0)) and (y1 > max(y0, 0))
        assert r.max_pairs(recs, th) == want


def test_scene_sources_distribution():
    from tractor_b200 import batch, _lib
    rng = np.random.default_rng(1)
    s = batch.scene_sources(20000, rng)
    frac = [np.mean(s['profile'] == p) for p in (_lib.PROFILE_POINT, _lib.PROFILE_EXP,
                                                  _lib.PROFILE_DEV, _lib.PROFILE_COMPOSITE)]
    assert np.allclose(frac, [0.4, 0.3, 0.2, 0.1], atol=0.015)
    hw = (s['mw'] - 1) // 2
    assert hw.min() >= 7 and hw.max() <= 127 and np.all(s['mw'] == s['mh'])
    assert s['counts'].min() >= 10 and s['counts'].max() <= 1e5
