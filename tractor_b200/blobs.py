"""Blob segmentation on the GPU, for callers that cut images into blobs
before Tractor.setModelMasks (tractor/engine.py:341-361) or the batched
fitter (`fit.fit_tractors`).

`label` and `find_objects` keep scipy.ndimage's signatures and results
(4-connectivity by default, 8 with a full 3 x 3 structure; components
numbered in the raster order of their first pixel; boxes as slice pairs);
`segment` labels a detection map, boxes every blob and assigns sources to
the blob under their pixel; `blob_model_masks` turns that into the
`Tractor.setModelMasks` argument.  There is no CPU path: without the library
or a CUDA device these raise.
"""
import numpy as np
import torch

from . import _lib, render


def _conn8(structure):
    if structure is None:
        return 0
    st = np.asarray(structure).astype(bool)
    if st.shape != (3, 3):
        raise ValueError('structure must be 3 x 3')
    cross = np.array([[0, 1, 0], [1, 1, 1], [0, 1, 0]], bool)
    if np.array_equal(st, cross):
        return 0
    if st.all():
        return 1
    raise ValueError('only the 4-connected cross or the full 3 x 3 structure is supported')


def _label_device(d_mask, H, W, conn8):
    """(labels int32 device tensor (H, W), n) of a device uint8 mask."""
    lib = _lib.load()
    dev = d_mask.device
    nbytes = int(lib.tb_label_workspace_bytes(H, W))
    if nbytes < 0:
        raise ValueError('image too large to label (%d x %d)' % (H, W))
    ws = torch.empty((nbytes + 15) // 16 * 4, dtype=torch.int32, device=dev)
    labels = torch.empty((H, W), dtype=torch.int32, device=dev)
    scal = torch.zeros(2, dtype=torch.int32, device=dev)   # n_labels, error
    _lib.check(lib.tb_label_components(d_mask.data_ptr(), H, W, conn8, labels.data_ptr(),
                                       scal.data_ptr(), ws.data_ptr(), scal.data_ptr() + 4,
                                       _lib.stream_ptr()), 'tb_label_components')
    n, err = (int(v) for v in scal.cpu())
    if err:
        raise RuntimeError('tb_label_components: a merge ran out of its retry bound')
    return labels, n


def _boxes_device(labels, n):
    lib = _lib.load()
    H, W = labels.shape
    boxes = torch.empty((max(n, 1), 4), dtype=torch.int32, device=labels.device)
    _lib.check(lib.tb_component_boxes(labels.data_ptr(), H, W, n, boxes.data_ptr(),
                                      _lib.stream_ptr()), 'tb_component_boxes')
    return boxes[:n]


def _mask_tensor(mask):
    m = np.asarray(mask)
    if m.ndim != 2:
        raise ValueError('2-D mask expected')
    m8 = m.view(np.uint8) if m.dtype == np.bool_ else (m != 0).view(np.uint8)
    return torch.from_numpy(np.ascontiguousarray(m8)).to(render.device()), m.shape


def _run_label(mask, conn8):
    """Host mask -> (labels numpy int32, n)."""
    d, (H, W) = _mask_tensor(mask)
    labels, n = _label_device(d, H, W, conn8)
    return labels.cpu().numpy(), n


def _run_segment(mask, conn8):
    """Host mask -> (labels numpy int32, n, boxes numpy (n, 4)): labels and
    boxes computed on the device, one copy of each back."""
    d, (H, W) = _mask_tensor(mask)
    labels, n = _label_device(d, H, W, conn8)
    boxes = _boxes_device(labels, n)
    return labels.cpu().numpy(), n, boxes.cpu().numpy()


def _run_boxes(labels, n):
    """Host labels -> boxes numpy (n, 4): y0, x0, y1, x1."""
    lab = np.ascontiguousarray(labels, np.int32)
    d = torch.from_numpy(lab).to(render.device())
    return _boxes_device(d, n).cpu().numpy()


def label(input, structure=None):
    """scipy.ndimage.label for 2-D masks: (labels int32, number of
    components)."""
    return _run_label(input, _conn8(structure))


def find_objects(input, max_label=0):
    """scipy.ndimage.find_objects for 2-D label images: for labels 1..n the
    (row slice, column slice) of their bounding box, None for a label with
    no pixel."""
    lab = np.asarray(input)
    n = int(max_label) if max_label > 0 else int(lab.max(initial=0))
    if n == 0:
        return []
    boxes = _run_boxes(lab, n)
    H, W = lab.shape
    out = []
    for y0, x0, y1, x1 in boxes:
        out.append(None if y1 == 0 else (slice(int(y0), int(y1)), slice(int(x0), int(x1))))
    return out


class Segmentation(object):
    """Blobs of a detection map: `labels` (int32, 0 = background), `n`
    blobs, `boxes` (n, 4: y0, x0, y1, x1 exclusive), `slices[b]` the
    bounding box of blob b + 1 as (row slice, column slice), `blob_of[i]`
    the blob (0-based) under source i's pixel or -1, `sources[b]` the
    sources in blob b (in source order).  `slices` and `sources` are built
    on first use."""

    def __init__(self, labels, n, boxes, blob_of):
        self.labels, self.n, self.boxes, self.blob_of = labels, n, boxes, blob_of
        self._slices = None
        self._sources = None

    @property
    def slices(self):
        if self._slices is None:
            self._slices = [None if y1 == 0 else (slice(int(y0), int(y1)),
                                                  slice(int(x0), int(x1)))
                            for y0, x0, y1, x1 in self.boxes]
        return self._slices

    @property
    def sources(self):
        if self._sources is None:
            # group by blob with one stable sort (source order kept in a blob)
            bo, n = self.blob_of, self.n
            if n == 0:
                self._sources = []
            else:
                order = np.argsort(bo, kind='stable')
                counts = np.bincount(bo[bo >= 0], minlength=n)
                start = int(np.count_nonzero(bo < 0))
                self._sources = np.split(order[start:], np.cumsum(counts)[:-1])
        return self._sources


def segment(detmap, positions=None, structure=None):
    """Labels the detection map's connected components (`label`), boxes them
    (`find_objects`) and assigns each source position (x, y), rounded to
    its pixel, to the blob under it (-1 outside the map or on background).
    Returns a Segmentation."""
    labels, n, boxes = _run_segment(detmap, _conn8(structure))
    H, W = labels.shape
    if positions is None:
        blob_of = np.zeros(0, np.int64)
    else:
        xy = np.asarray(positions, np.float64).reshape(-1, 2)
        ix = np.round(xy[:, 0]).astype(np.int64)
        iy = np.round(xy[:, 1]).astype(np.int64)
        inside = (ix >= 0) & (ix < W) & (iy >= 0) & (iy < H)
        blob_of = np.full(len(xy), -1, np.int64)
        blob_of[inside] = labels[iy[inside], ix[inside]].astype(np.int64) - 1
    return Segmentation(labels, n, boxes, blob_of)


def blob_model_masks(tractor, seg, sources=None):
    """The Tractor.setModelMasks argument (one dict per image, source ->
    ModelMask) that restricts each source to the bounding box of its blob
    (sources outside every blob are left out).  `sources` defaults to the
    tractor's catalog, in the order of the positions given to `segment`."""
    from .patch import ModelMask
    srcs = list(tractor.getCatalog()) if sources is None else list(sources)
    if len(srcs) != len(seg.blob_of):
        raise ValueError('one position per source expected')
    d = {}
    for src, b in zip(srcs, seg.blob_of):
        if b < 0:
            continue
        y0, x0, y1, x1 = (int(v) for v in seg.boxes[b])
        d[src] = ModelMask(x0, y0, x1 - x0, y1 - y0)
    return [dict(d) for _ in tractor.getImages()]
