"""Patch and ModelMask with the reference's geometry and arithmetic
(tractor/patch.py:1-446; get_overlapping_region as tractor/patch.pyx:20-65).

A Patch holds a numpy array (host) like the reference's, so callers can use
it with numpy; the GPU paths fill it from device buffers.
"""
import numpy as np


def get_overlapping_region(xlo, xhi, xmin, xmax):
    """Given the wanted integer range [xlo, xhi] and the valid range
    [xmin, xmax], returns (slice of valid coordinates, slice into the wanted
    range), or ([], []) if they do not overlap (tractor/patch.pyx:20-65)."""
    if xlo > xmax or xhi < xmin or xlo > xhi or xmin > xmax:
        return ([], [])
    lo = max(xlo, xmin)
    Xlo = lo - xlo
    hi = min(xhi, xmax)
    Xhi = Xlo + (hi - lo)
    return (slice(lo, hi + 1), slice(Xlo, Xhi + 1))


class ModelMask(object):
    """ModelMask(x0, y0, w, h) or ModelMask(x0, y0, mask) (patch.py:3-56)."""

    def __init__(self, x0, y0, *args):
        self.x0 = x0
        self.y0 = y0
        if len(args) == 2:
            self.w, self.h = args
            self.mask = None
        elif len(args) == 1:
            self.mask = args[0]
            self.h, self.w = self.mask.shape
        else:
            raise ValueError('Wrong number of arguments')

    def __str__(self):
        s = 'ModelMask: origin (%i,%i), w=%i, h=%i' % (self.x0, self.y0, self.w, self.h)
        return s if self.mask is None else s + ', has mask'

    __repr__ = __str__

    @staticmethod
    def fromExtent(x0, x1, y0, y1):
        return ModelMask(x0, y0, x1 - x0, y1 - y0)

    @property
    def shape(self):
        return (self.h, self.w)

    @property
    def x1(self):
        return self.x0 + self.w

    @property
    def y1(self):
        return self.y0 + self.h

    @property
    def extent(self):
        return (self.x0, self.x0 + self.w, self.y0, self.y0 + self.h)


def add_patches(pa, pb):
    p = pa
    if pb is not None:
        if p is None:
            p = pb
        else:
            p += pb
    return p


class Patch(object):
    """A sub-image with an integer origin (patch.py:71-446)."""

    def __init__(self, x0, y0, patch):
        self.x0 = x0
        self.y0 = y0
        self.patch = patch
        self.name = ''

    @property
    def x1(self):
        return self.x0 + self.patch.shape[1]

    @property
    def y1(self):
        return self.y0 + self.patch.shape[0]

    @property
    def shape(self):
        if self.patch is None:
            return (0, 0)
        return self.patch.shape

    @property
    def size(self):
        return 0 if self.patch is None else self.patch.size

    @property
    def extent(self):
        h, w = self.shape
        return (self.x0, self.x0 + w, self.y0, self.y0 + h)

    def __str__(self):
        s = 'Patch: '
        if self.name:
            s += self.name + ' '
        s += 'origin (%i,%i) ' % (self.x0, self.y0)
        if self.patch is not None:
            H, W = self.patch.shape
            s += 'size (%i x %i)' % (W, H)
        else:
            s += '(no image)'
        return s

    __repr__ = __str__

    def set(self, other):
        self.x0, self.y0, self.patch, self.name = other.x0, other.y0, other.patch, other.name

    def setName(self, name):
        self.name = name

    def getName(self):
        return self.name

    def copy(self):
        return Patch(self.x0, self.y0, None if self.patch is None else self.patch.copy())

    def getExtent(self, margin=0):
        h, w = self.shape
        return (self.x0 - margin, self.x0 + w + margin, self.y0 - margin, self.y0 + h + margin)

    def getOrigin(self):
        return (self.x0, self.y0)

    def getPatch(self):
        return self.patch

    getImage = getPatch

    def getX0(self):
        return self.x0

    def getY0(self):
        return self.y0

    def overlapsBbox(self, bbox):
        x0, x1, y0, y1 = self.getExtent()
        ox0, ox1, oy0, oy1 = bbox
        return not (x0 >= ox1 or ox0 >= x1 or y0 >= oy1 or oy0 >= y1)

    def hasBboxOverlapWith(self, other):
        return self.overlapsBbox(other.getExtent())

    def hasNonzeroOverlapWith(self, other):
        """Whether the two patches' product has a positive sum over their
        overlap (patch.py:171-186)."""
        if not self.hasBboxOverlapWith(other):
            return False
        x0, x1, y0, y1 = self.getExtent()
        ox0, ox1, oy0, oy1 = other.getExtent()
        ix, ox = get_overlapping_region(ox0, ox1 - 1, x0, x1 - 1)
        iy, oy = get_overlapping_region(oy0, oy1 - 1, y0, y1 - 1)
        ix = slice(ix.start - x0, ix.stop - x0)
        iy = slice(iy.start - y0, iy.stop - y0)
        sub = self.patch[iy, ix]
        osub = other.patch[oy, ox]
        assert sub.shape == osub.shape
        return np.sum(sub * osub) > 0.

    def getNonZeroMask(self):
        return Patch(self.x0, self.y0, self.patch != 0)

    def trimToNonZero(self):
        """Shrinks to the bounding box of the non-zero pixels (patch.py:136-177)."""
        if self.patch is None:
            return
        H, W = self.patch.shape
        if W == 0 or H == 0:
            return
        nzc = np.flatnonzero(np.any(self.patch != 0, axis=0))
        nzr = np.flatnonzero(np.any(self.patch != 0, axis=1))
        if len(nzc) == 0:
            self.patch = None
            return
        x0, x1 = nzc[0], nzc[-1] + 1
        y0, y1 = nzr[0], nzr[-1] + 1
        if x0 == 0 and y0 == 0 and x1 == W and y1 == H:
            return
        self.patch = self.patch[y0:y1, x0:x1]
        self.x0 += x0
        self.y0 += y0

    def clipTo(self, W, H):
        """patch.py:241-278."""
        if self.patch is None:
            return False
        if self.x0 >= W or self.y0 >= H:
            self.patch = None
            return False
        if self.x0 < 0:
            self.patch = self.patch[:, -self.x0:]
            self.x0 = 0
        if self.y0 < 0:
            self.patch = self.patch[-self.y0:, :]
            self.y0 = 0
        h, w = self.patch.shape
        if self.x0 + w > W:
            self.patch = self.patch[:, :W - self.x0]
        if self.y0 + h > H:
            self.patch = self.patch[:H - self.y0, :]
        return True

    def clipToRoi(self, x0, x1, y0, y1):
        if self.patch is None:
            return False
        if self.x0 >= x1 or self.x1 <= x0 or self.y0 >= y1 or self.y1 <= y0:
            self.patch = None
            return False
        if self.x0 < x0:
            self.patch = self.patch[:, x0 - self.x0:]
            self.x0 = x0
        if self.y0 < y0:
            self.patch = self.patch[y0 - self.y0:, :]
            self.y0 = y0
        h, w = self.shape
        if self.x0 + w > x1:
            self.patch = self.patch[:, :x1 - self.x0]
        if self.y0 + h > y1:
            self.patch = self.patch[:y1 - self.y0, :]
        return True

    def getSlice(self, parent=None):
        if self.patch is None:
            return ([], [])
        ph, pw = self.patch.shape
        if parent is not None:
            H, W = parent.shape
            return (slice(np.clip(self.y0, 0, H), np.clip(self.y0 + ph, 0, H)),
                    slice(np.clip(self.x0, 0, W), np.clip(self.x0 + pw, 0, W)))
        return (slice(self.y0, self.y0 + ph), slice(self.x0, self.x0 + pw))

    def getSlices(self, shape):
        ph, pw = self.shape
        ih, iw = shape
        outx, inx = get_overlapping_region(self.x0, self.x0 + pw - 1, 0, iw - 1)
        outy, iny = get_overlapping_region(self.y0, self.y0 + ph - 1, 0, ih - 1)
        if inx == [] or iny == []:
            return (slice(0, 0), slice(0, 0)), (slice(0, 0), slice(0, 0))
        return (iny, inx), (outy, outx)

    def getPixelIndices(self, parent, dtype=np.int32):
        if self.patch is None:
            return np.array([], dtype)
        h, w = self.shape
        H, W = parent.shape
        return ((np.arange(w, dtype=dtype) + dtype(self.x0))[np.newaxis, :] +
                ((np.arange(h, dtype=dtype) + dtype(self.y0)) * dtype(W))[:, np.newaxis]).ravel()

    def addTo(self, img, scale=1.):
        """Adds into the overlapping part of `img` (patch.py:341-354)."""
        if self.patch is None:
            return
        ih, iw = img.shape
        ph, pw = self.shape
        outx, inx = get_overlapping_region(self.x0, self.x0 + pw - 1, 0, iw - 1)
        outy, iny = get_overlapping_region(self.y0, self.y0 + ph - 1, 0, ih - 1)
        if inx == [] or iny == []:
            return
        img[outy, outx] += self.patch[iny, inx] * scale

    def __imul__(self, f):
        if self.patch is not None:
            self.patch *= f
        return self

    def __itruediv__(self, f):
        if self.patch is not None:
            self.patch /= f
        return self

    def __mul__(self, f):
        return Patch(self.x0, self.y0, None if self.patch is None else self.patch * f)

    def __truediv__(self, f):
        return Patch(self.x0, self.y0, None if self.patch is None else self.patch / f)

    def performArithmetic(self, other, opname, otype=float):
        """Element-wise op on the union of two patches (patch.py:406-446)."""
        assert isinstance(other, Patch)
        if self.x0 == other.x0 and self.y0 == other.y0 and self.shape == other.shape:
            if self.patch is None or other.patch is None:
                return Patch(self.x0, self.y0, None)
            pcopy = self.patch.copy()
            return Patch(self.x0, self.y0, getattr(pcopy, opname)(other.patch))
        ph, pw = self.patch.shape
        ox0, oy0 = other.x0, other.y0
        oh, ow = other.shape
        ux0, uy0 = min(ox0, self.x0), min(oy0, self.y0)
        ux1, uy1 = max(ox0 + ow, self.x0 + pw), max(oy0 + oh, self.y0 + ph)
        p = np.zeros((uy1 - uy0, ux1 - ux0), dtype=otype)
        p[self.y0 - uy0:self.y0 - uy0 + ph, self.x0 - ux0:self.x0 - ux0 + pw] = self.patch
        psub = p[oy0 - uy0:oy0 - uy0 + oh, ox0 - ux0:ox0 - ux0 + ow]
        getattr(psub, opname)(other.getImage())
        return Patch(ux0, uy0, p)

    def __add__(self, other):
        return self.performArithmetic(other, '__iadd__')

    def __sub__(self, other):
        return self.performArithmetic(other, '__isub__')
