"""Host-side batching for the device kernels.

A batch collects work items (one mixture on one rectangle, or one galaxy
through the Fourier path), packs every table into one host buffer, copies it
to the device in a single transfer and launches the kernel once.  Device
outputs stay torch tensors; the Tractor-facing classes copy to numpy only
where the reference API returns numpy arrays.
"""
import numpy as np
import torch

from . import _lib

MOG_STORE, MOG_ACCUM, MOG_ATOMIC = _lib.MOG_STORE, _lib.MOG_ACCUM, _lib.MOG_ATOMIC

# Exponent floors (natural-log units) of the reference evaluators.
FLOOR_GRID = -50.0      # c_gauss_2d_grid: skip Mahalanobis^2 >= 100 (mix.i:505)
FLOOR_MASKED = -30.0    # c_gauss_2d_masked: skip exponents below -30 (gauss_masked.c:88)


def device():
    _lib.require_cuda()
    return torch.device('cuda', torch.cuda.current_device())


class _Packer(object):
    """Accumulates named numpy sections into one 256-byte aligned buffer."""

    def __init__(self):
        self.sections = []
        self.size = 0

    def add(self, arr):
        arr = np.ascontiguousarray(arr)
        off = (self.size + 255) // 256 * 256
        self.sections.append((off, arr))
        self.size = off + arr.nbytes
        return off

    def to_device(self, dev):
        buf = np.zeros(max(self.size, 1), np.uint8)
        for off, arr in self.sections:
            buf[off:off + arr.nbytes] = arr.view(np.uint8).ravel()
        host = torch.from_numpy(buf)
        if dev.type == 'cuda':
            host = host.pin_memory()
        return host.to(dev, non_blocking=True)


def check_status(status_tensor, what):
    """Raises if a kernel reported a bad item or non-finite input."""
    st = status_tensor.cpu().numpy().view(_lib.STATUS)[0]
    if st['code'] != 0:
        kind = {1: 'non-finite value', 2: 'invalid item', 3: 'not positive definite'}
        raise RuntimeError('%s: %s at item %d (detail %d, %d reports)' %
                           (what, kind.get(int(st['code']), 'error'), st['item'], st['detail'],
                            st['count']))


class MogBatch(object):
    """Items for tb_mog_render (c_gauss_2d_grid / c_gauss_2d_masked semantics,
    batched)."""

    def __init__(self):
        self.items = []
        self.amp = []
        self.mean = []
        self.var = []
        self.masks = []
        self.ncomp = 0
        self.nmask = 0
        self.nout = 0

    def __len__(self):
        return len(self.items)

    def add(self, x0, y0, w, h, amp, mean, var, fx=0., fy=0., floor=FLOOR_GRID, scale=1.,
            mask=None, out_off=None, ldo=0, mode=MOG_STORE, minval=None, derivs=False):
        """Adds one mixture evaluated on [x0, x0+w) x [y0, y0+h).  Returns the
        element offset of its output (a packed w x h patch unless `out_off`
        and `ldo` place it inside a larger buffer).  `minval` selects the
        per-component floors of c_gauss_2d_approx3; `derivs` also writes the
        d/dmean_x and d/dmean_y planes right after the patch (packed outputs
        only)."""
        # copies: a plan renders the state at the time of the call even if
        # the caller's arrays change before it runs (line searches, finite
        # differences of image parameters)
        amp = np.array(amp, np.float64).ravel()
        K = len(amp)
        if K > 256:
            raise ValueError('at most 256 components per mixture (got %d)' % K)
        if out_off is None:
            out_off = self.nout
            self.nout += w * h * (3 if derivs else 1)
        elif derivs:
            raise ValueError('derivative planes need a packed output')
        deriv_off = out_off + w * h if derivs else -1
        mask_off = -1
        if mask is not None:
            mask_off = self.nmask
            self.masks.append(np.ascontiguousarray(mask, np.uint8).ravel())
            self.nmask += w * h
        floor_mode = _lib.FLOOR_FIXED
        if minval is not None:
            floor_mode = _lib.FLOOR_MINVAL
            floor = float(minval)
        self.items.append((int(x0), int(y0), int(w), int(h), self.ncomp, K, int(mode), int(ldo),
                           float(fx), float(fy), float(floor), float(scale), floor_mode,
                           int(out_off), int(mask_off), 0, int(deriv_off)))
        self.amp.append(amp)
        self.mean.append(np.array(mean, np.float64).reshape(K, 2))
        self.var.append(np.array(var, np.float64).reshape(K, 2, 2))
        self.ncomp += K
        return out_off

    def run(self, out=None, stream=None, check=True):
        """Launches one tb_mog_render over all items.  `out` (float32 device
        tensor) defaults to a new packed buffer of all patches."""
        lib = _lib.load()
        dev = device()
        if out is None:
            out = torch.empty(max(self.nout, 1), dtype=torch.float32, device=dev)
        if not self.items:
            return out
        items = np.array(self.items, dtype=_lib.MOG_ITEM)
        tiles = ((items['w'] + 31) // 32).astype(np.int64) * ((items['h'] + 31) // 32)
        items['tile0'] = np.concatenate([[0], np.cumsum(tiles)[:-1]])
        n_tiles = int(tiles.sum())
        pk = _Packer()
        o_items = pk.add(items)
        o_amp = pk.add(np.concatenate(self.amp))
        o_mean = pk.add(np.concatenate(self.mean))
        o_var = pk.add(np.concatenate(self.var))
        o_mask = pk.add(np.concatenate(self.masks)) if self.masks else None
        o_ctr = pk.add(np.zeros(4, np.int32))
        o_st = pk.add(np.zeros(1, _lib.STATUS))
        d = pk.to_device(dev)
        base = d.data_ptr()
        rc = lib.tb_mog_render(base + o_items, len(items), n_tiles, base + o_amp, base + o_mean,
                               base + o_var, None if o_mask is None else base + o_mask,
                               out.data_ptr(), base + o_ctr, base + o_st,
                               _lib.stream_ptr(stream))
        _lib.check(rc, 'tb_mog_render')
        self._dev = d
        self.status = d[o_st:o_st + 16]
        if check:
            check_status(self.status, 'tb_mog_render')
        return out


class PsfSpectra(object):
    """Device spectra of pixelized PSFs, one per (PSF image, size), computed
    by tb_psf_spectrum (PixelizedPSF.getFourierTransform, tractor/psf.py:249-280)."""

    def __init__(self):
        self.cache = {}

    @staticmethod
    def pad(img, sz):
        """PixelizedPSF._padInImage (tractor/psf.py:214-247): returns the
        sz x sz padded image and the PSF centre (cx, cy) in it."""
        img = np.asarray(img, np.float32)
        ph, pw = img.shape
        sub = img
        if sz >= ph:
            y0 = (sz - ph) // 2
            cy = y0 + ph // 2
        else:
            y0 = 0
            cut = (ph - sz) // 2
            sub = sub[cut:cut + sz, :]
            cy = ph // 2 - cut
        if sz >= pw:
            x0 = (sz - pw) // 2
            cx = x0 + pw // 2
        else:
            x0 = 0
            cut = (pw - sz) // 2
            sub = sub[:, cut:cut + sz]
            cx = pw // 2 - cut
        sh, sw = sub.shape
        pad = np.zeros((sz, sz), np.float32)
        pad[y0:y0 + sh, x0:x0 + sw] = sub
        return pad, cx, cy

    def get(self, key, img, sz, normalize=False):
        """Returns (device spectrum tensor, cx, cy) for PSF image `img` at FFT
        size sz; `key` identifies the PSF for caching."""
        k = (key, sz, bool(normalize))
        if k not in self.cache:
            self.cache[k] = self.compute(img, sz, normalize)
        return self.cache[k]

    def compute(self, img, sz, normalize=False):
        """(device spectrum tensor, cx, cy) of `img` at FFT size sz, not cached
        (position-dependent PSFs)."""
        lib = _lib.load()
        dev = device()
        pad, cx, cy = self.pad(img, sz)
        dpad = torch.from_numpy(pad).to(dev)
        spec = torch.empty(sz * (sz // 2 + 1) * 2, dtype=torch.float32, device=dev)
        rc = lib.tb_psf_spectrum(dpad.data_ptr(), spec.data_ptr(), 1, sz, int(bool(normalize)),
                                 _lib.stream_ptr())
        _lib.check(rc, 'tb_psf_spectrum')
        return (spec, cx, cy)


_spectra = PsfSpectra()


def psf_spectra():
    return _spectra


class FftBatch(object):
    """Items for tb_fourier_render (the Fourier branch of
    ProfileGalaxy._realGetUnitFluxModelPatch, batched).  Items may use
    different FFT sizes and PSFs; their spectra are gathered into one device
    buffer and each item points at its own."""

    def __init__(self):
        self.items = []
        self.amp = []
        self.var = []
        self.spec_off = {}       # spectrum key -> float offset in the gathered buffer
        self.spec_list = []
        self.nspec = 0
        self.ncomp = 0
        self.nout = 0

    def __len__(self):
        return len(self.items)

    def add(self, amp, var, sz, spec_key, spec, mw, mh, sx, sy, mux, muy, scale=1.,
            out_off=None, ldo=0, mode=MOG_STORE):
        amp = np.array(amp, np.float64).ravel()   # copies, as MogBatch.add
        K = len(amp)
        if K > 128:
            raise ValueError('at most 128 components per galaxy (got %d)' % K)
        if sz not in (32, 64, 128, 256):
            raise ValueError('FFT size %d not supported (32..256)' % sz)
        if out_off is None:
            out_off = self.nout
            self.nout += mw * mh
        key = (sz, spec_key)
        if key not in self.spec_off:
            self.spec_off[key] = self.nspec
            self.spec_list.append(spec)
            self.nspec += spec.numel()
        self.items.append((self.ncomp, K, int(sz), int(mode), int(mw), int(mh), int(sx), int(sy),
                           float(mux), float(muy), float(scale), int(ldo), int(out_off),
                           self.spec_off[key], _lib.FFT_VALUE, 0, 0))
        self.amp.append(amp)
        self.var.append(np.array(var, np.float64).reshape(K, 2, 2))
        self.ncomp += K
        return out_off

    def run(self, out=None, stream=None, check=True):
        lib = _lib.load()
        dev = device()
        if out is None:
            out = torch.empty(max(self.nout, 1), dtype=torch.float32, device=dev)
        if not self.items:
            return out
        items = np.array(self.items, dtype=_lib.FFT_ITEM)
        specs = torch.cat(self.spec_list) if len(self.spec_list) > 1 else self.spec_list[0]
        pk = _Packer()
        o_items = pk.add(items)
        o_amp = pk.add(np.concatenate(self.amp))
        o_var = pk.add(np.concatenate(self.var))
        o_ctr = pk.add(np.zeros(4, np.int32))
        o_st = pk.add(np.zeros(1, _lib.STATUS))
        d = pk.to_device(dev)
        base = d.data_ptr()
        rc = lib.tb_fourier_render(base + o_items, len(items), base + o_amp, base + o_var,
                                   specs.data_ptr(), out.data_ptr(), base + o_ctr, base + o_st,
                                   _lib.stream_ptr(stream))
        _lib.check(rc, 'tb_fourier_render')
        self._keep = (d, specs)
        self.status = d[o_st:o_st + 16]
        if check:
            check_status(self.status, 'tb_fourier_render')
        return out


def lanczos_shift(imgs, shifts, stream=None):
    """Batched Lanczos-3 shift of a (n, h, w) float32 device tensor by
    per-image (dx, dy) (lanczos_shift_3f, tractor/mp_fourier.i:405-429)."""
    lib = _lib.load()
    imgs = imgs.contiguous()
    n, h, w = imgs.shape
    out = torch.empty_like(imgs)
    sh = torch.as_tensor(np.asarray(shifts, np.float64).reshape(n, 2), device=imgs.device)
    rc = lib.tb_lanczos3_shift(imgs.data_ptr(), out.data_ptr(), sh.data_ptr(), n, h, w,
                               _lib.stream_ptr(stream))
    _lib.check(rc, 'tb_lanczos3_shift')
    return out


def chi2(data, model, inverr, offsets, npix, stream=None):
    """Per-image chi^2 (FP64 results) of flat float32 device tensors."""
    lib = _lib.load()
    n = len(offsets)
    out = torch.empty(n, dtype=torch.float64, device=data.device)
    off = torch.as_tensor(np.asarray(offsets, np.int64), device=data.device)
    npx = torch.as_tensor(np.asarray(npix, np.int64), device=data.device)
    rc = lib.tb_chi2(data.data_ptr(), model.data_ptr(), inverr.data_ptr(), off.data_ptr(),
                     npx.data_ptr(), n, out.data_ptr(), _lib.stream_ptr(stream))
    _lib.check(rc, 'tb_chi2')
    return out


def normal_equations(A, rhs, a_off, r_off, lda, P, R, stream=None):
    """A^T A and A^T r (FP64) of column-major FP32 problems in flat device
    tensors A and rhs.  Returns (AtA, Atr, ata_off, atr_off) device tensors."""
    lib = _lib.load()
    dev = A.device
    P = np.asarray(P, np.int32)
    n = len(P)
    ata_off = np.concatenate([[0], np.cumsum(P.astype(np.int64) ** 2)[:-1]]).astype(np.int64)
    atr_off = np.concatenate([[0], np.cumsum(P.astype(np.int64))[:-1]]).astype(np.int64)
    AtA = torch.zeros(int((P.astype(np.int64) ** 2).sum()), dtype=torch.float64, device=dev)
    Atr = torch.zeros(int(P.sum()), dtype=torch.float64, device=dev)
    t = lambda a, dt: torch.as_tensor(np.asarray(a, dt), device=dev)  # noqa: E731
    args = [t(a_off, np.int64), t(r_off, np.int64), t(lda, np.int32), t(P, np.int32),
            t(R, np.int32), t(ata_off, np.int64), t(atr_off, np.int64)]
    rc = lib.tb_normal_equations(A.data_ptr(), rhs.data_ptr(), *[a.data_ptr() for a in args],
                                 AtA.data_ptr(), Atr.data_ptr(), n, int(P.max()),
                                 _lib.stream_ptr(stream))
    _lib.check(rc, 'tb_normal_equations')
    return AtA, Atr, args[5], args[6]


def solve_update(AtA, Atr, ata_off, atr_off, P, damp=0., stream=None):
    """Column-scaled FP64 Cholesky solve + one refinement step per problem.
    Returns (X float64 device tensor, info int32 device tensor, x_off)."""
    lib = _lib.load()
    dev = AtA.device
    P = np.asarray(P, np.int32)
    n = len(P)
    maxp = int(P.max())
    x_off = np.concatenate([[0], np.cumsum(P.astype(np.int64))[:-1]]).astype(np.int64)
    X = torch.zeros(int(P.sum()), dtype=torch.float64, device=dev)
    info = torch.zeros(n, dtype=torch.int32, device=dev)
    work = torch.empty(n * maxp * maxp, dtype=torch.float64, device=dev)
    dP = torch.as_tensor(P, device=dev)
    dxo = torch.as_tensor(x_off, device=dev)
    rc = lib.tb_solve_update(AtA.data_ptr(), Atr.data_ptr(), ata_off.data_ptr(),
                             atr_off.data_ptr(), dP.data_ptr(), dxo.data_ptr(), X.data_ptr(),
                             info.data_ptr(), float(damp), n, maxp, work.data_ptr(),
                             _lib.stream_ptr(stream))
    _lib.check(rc, 'tb_solve_update')
    return X, info, x_off
