"""Blob segmentation (tractor_b200.blobs) against scipy.ndimage, the
reference's callers' own tool for it: labels and boxes must be identical
(integer work, bit-exact), for both connectivities, on random masks of many
densities and sizes and on the edge cases (empty, full, single pixels, one
row / column, checkerboards, long snakes)."""
import numpy as np
import pytest
import scipy.ndimage as ndi

CROSS = ndi.generate_binary_structure(2, 1)
FULL = np.ones((3, 3), bool)


@pytest.fixture(params=['host', pytest.param('gpu', marks=pytest.mark.gpu)])
def backend(request, monkeypatch):
    if request.param == 'host':
        import fake_device
        fake_device.install(monkeypatch)
    else:
        request.getfixturevalue('tb')
    return request.param


def _serpentine(n):
    """One long snake: every other row set, joined alternately at the right
    and left ends (the worst case for merge chains)."""
    m = np.zeros((n, n), bool)
    m[::2] = True
    for r in range(1, n, 2):
        m[r, n - 1 if (r // 2) % 2 == 0 else 0] = True
    return m


def _cases():
    rng = np.random.default_rng(42)
    out = [np.zeros((7, 9), bool), np.ones((13, 5), bool), np.eye(17, dtype=bool),
           np.ones((1, 50), bool), (rng.random((1, 300)) < 0.5), (rng.random((300, 1)) < 0.5),
           (np.indices((31, 33)).sum(0) % 2).astype(bool), _serpentine(61)]
    z = np.zeros((10, 10), bool)
    z[0, 0] = z[9, 9] = z[0, 9] = z[9, 0] = True
    out.append(z)
    for (h, w, dens) in [(64, 64, 0.3), (100, 257, 0.5), (257, 100, 0.59), (512, 700, 0.45),
                         (333, 333, 0.7), (1000, 1000, 0.55)]:
        out.append(rng.random((h, w)) < dens)
    # smooth blobs: a thresholded smoothed field, as detection maps look
    f = ndi.gaussian_filter(rng.normal(size=(600, 800)), 6)
    out.append(f > 0.02)
    return out


def test_label_and_find_objects_match_scipy(backend):
    from tractor_b200 import blobs
    for m in _cases():
        for st in (None, CROSS, FULL):
            lab, n = blobs.label(m, structure=st)
            ref, nr = ndi.label(m, structure=st)
            assert n == nr and np.array_equal(lab, ref), (m.shape, st is FULL)
            assert blobs.find_objects(lab) == ndi.find_objects(ref)


def test_find_objects_missing_labels(backend):
    """Labels with no pixel give None, as scipy's find_objects does."""
    from tractor_b200 import blobs
    lab = np.zeros((20, 30), np.int32)
    lab[2:5, 3:9] = 1
    lab[10:12, 20:29] = 4
    assert blobs.find_objects(lab) == ndi.find_objects(lab)
    assert blobs.find_objects(lab, max_label=6) == ndi.find_objects(lab, max_label=6)


def test_segment_and_model_masks(backend):
    """Sources go to the blob under their rounded pixel; blob_model_masks
    restricts each to its blob's box (sources off every blob left out)."""
    import tractor_b200 as T
    from tractor_b200 import blobs
    det = np.zeros((60, 80), bool)
    det[5:20, 10:30] = True
    det[30:55, 40:75] = True
    det[30:33, 5:8] = True
    pos = np.array([[12.2, 7.6], [70.4, 50.1], [6.0, 31.4], [0.2, 0.3], [45.0, 40.0]])
    seg = blobs.segment(det, pos)
    assert seg.n == 3
    assert list(seg.blob_of) == [0, 2, 1, -1, 2]
    assert [list(s) for s in seg.sources] == [[0], [2], [1, 4]]
    assert seg.slices[2] == (slice(30, 55), slice(40, 75))
    tim = T.Image(data=np.zeros((60, 80), np.float32), inverr=np.ones((60, 80), np.float32),
                  psf=T.NCircularGaussianPSF([1.5], [1.]))
    srcs = [T.PointSource(T.PixPos(x, y), T.Flux(10.)) for x, y in pos]
    tr = T.Tractor([tim], srcs)
    mm = blobs.blob_model_masks(tr, seg)
    assert len(mm) == 1 and set(mm[0]) == {srcs[0], srcs[1], srcs[2], srcs[4]}
    m = mm[0][srcs[1]]
    assert (m.x0, m.y0, m.w, m.h) == (40, 30, 35, 25)


def test_rejects_unsupported_structure(backend):
    from tractor_b200 import blobs
    with pytest.raises(ValueError):
        blobs.label(np.ones((4, 4)), structure=np.array([[1, 1, 0], [1, 1, 0], [0, 0, 0]]))


@pytest.mark.gpu
def test_label_large_image_matches_scipy(tb):
    """A 4096 x 4096 map near the 4-connected percolation density (one
    component spans most of it, long merge chains) and a smooth field:
    identical to scipy."""
    from tractor_b200 import blobs
    rng = np.random.default_rng(7)
    m = rng.random((4096, 4096)) < 0.593
    lab, n = blobs.label(m)
    ref, nr = ndi.label(m)
    assert n == nr and np.array_equal(lab, ref)
    lab8, n8 = blobs.label(m, structure=FULL)
    ref8, nr8 = ndi.label(m, structure=FULL)
    assert n8 == nr8 and np.array_equal(lab8, ref8)


def test_segment_connectivity_and_empty(backend):
    """8-connectivity joins diagonal neighbours; an empty map has no blobs
    and every source is off-blob."""
    from tractor_b200 import blobs
    det = np.zeros((9, 9), bool)
    det[2, 2] = det[3, 3] = det[6, 6] = True
    s4 = blobs.segment(det, [[2, 2], [3, 3]])
    s8 = blobs.segment(det, [[2, 2], [3, 3]], structure=FULL)
    assert s4.n == 3 and list(s4.blob_of) == [0, 1]
    assert s8.n == 2 and list(s8.blob_of) == [0, 0]
    assert [list(x) for x in s8.sources] == [[0, 1], []]
    assert s8.slices[0] == (slice(2, 4), slice(2, 4))
    e = blobs.segment(np.zeros((5, 7), bool), [[1., 1.], [-3., 2.]])
    assert e.n == 0 and list(e.blob_of) == [-1, -1] and e.sources == [] and e.slices == []
