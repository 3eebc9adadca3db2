"""Host-side batching for the device kernels.

A batch collects work items (one mixture on one rectangle, or one galaxy
through the Fourier path), packs every table into one host buffer, copies it
to the device in a single transfer and launches the kernel once.  Device
outputs stay torch tensors; the Tractor-facing classes copy to numpy only
where the reference API returns numpy arrays.
"""
import ctypes

import threading

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


class _PinnedPool(object):
    """Reusable pinned host staging buffers for host-to-device copies.
    Pinning memory costs far more than a small copy, so buffers are kept;
    a buffer is handed out again only once the copy that last read it has
    completed (an event recorded after that copy on its stream)."""

    MAX_BUFFERS = 16

    def __init__(self):
        self.bufs = []      # [pinned uint8 tensor, event or None]

    def get(self, nbytes):
        for entry in self.bufs:
            t, ev = entry
            if t.numel() >= nbytes and (ev is None or ev.query()):
                return entry
        if len(self.bufs) >= self.MAX_BUFFERS:
            # all busy or too small: wait for the oldest copy and replace it
            t, ev = self.bufs.pop(0)
            if ev is not None:
                ev.synchronize()
        size = 1 << max(16, int(np.ceil(np.log2(max(nbytes, 1)))))
        entry = [torch.empty(size, dtype=torch.uint8).pin_memory(), None]
        self.bufs.append(entry)
        return entry


_pinned = _PinnedPool()


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
        size = max(self.size, 1)
        if dev.type != 'cuda':
            buf = np.zeros(size, np.uint8)
            for off, arr in self.sections:
                buf[off:off + arr.nbytes] = arr.view(np.uint8).ravel()
            return torch.from_numpy(buf)
        entry = _pinned.get(size)
        host = entry[0][:size]
        buf = host.numpy()      # padding between sections is never read
        for off, arr in self.sections:
            buf[off:off + arr.nbytes] = arr.view(np.uint8).ravel()
        out = torch.empty(size, dtype=torch.uint8, device=dev)
        out.copy_(host, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        entry[1] = ev
        return out


class _PinnedOut(threading.local):
    """Pinned host staging for device-to-host copies of finished renders
    (one reused buffer per thread): the copy lands in pinned memory
    (pageable destinations take a slower, staged path), the stream is
    synchronised and the bytes are copied out into a new array."""

    buf = None

    def to_host(self, t, dtype, stream):
        n = t.numel() * t.element_size()
        if self.buf is None or self.buf.numel() < n:
            size = 1 << max(16, int(np.ceil(np.log2(max(n, 1)))))
            self.buf = torch.empty(size, dtype=torch.uint8).pin_memory()
        host = self.buf[:n]
        host.copy_(t.reshape(-1).view(torch.uint8), non_blocking=True)
        stream.synchronize()
        return host.numpy().view(dtype).copy()


_pinned_out = _PinnedOut()


def to_host(t, dtype, stream=None):
    """numpy copy of device tensor `t` (contiguous) as `dtype`, after the
    stream (default: the current one) has finished writing it."""
    if stream is None:
        stream = torch.cuda.current_stream()
    return _pinned_out.to_host(t, dtype, stream)


def check_status_host(raw, what):
    """check_status of a status word already on the host (16 bytes)."""
    st = np.ascontiguousarray(raw).view(np.uint8).view(_lib.STATUS)[0]
    if st['code'] != 0:
        kind = {1: 'non-finite value', 2: 'invalid item', 3: 'not positive definite'}
        raise RuntimeError('%s: %s at item %d (detail %d, %d reports)' %
                           (what, kind.get(int(st['code']), 'error'), st['item'], st['detail'],
                            st['count']))


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
        self.rings = []

    def __len__(self):
        return len(self.items)

    def add_ring(self, val_off, w, h, minval, minradius, start=None, default_start=(0, 0),
                 edge_col=None, edge_row=None, deriv_off=-1):
        """Adds an approx3 region walk (tb_approx3_region) over the w x h
        values at val_off (an item added with `minval`): start = box-relative
        (xc, yc) inside the box, or None to start at the largest value of
        edge_col = (x, offset of its h values) / edge_row = (y, offset of its
        w values), default_start when none is above 0.  Returns the index of
        its extent (sx0, sx1, sy0, sy1) in `extents` after run()."""
        if w > _lib.RING_MAX or h > _lib.RING_MAX:
            raise ValueError('approx3 boxes up to %d pixels a side' % _lib.RING_MAX)
        r = np.zeros(1, _lib.RING_ITEM)[0]
        r['val_off'], r['deriv_off'] = val_off, deriv_off
        r['edge_col_off'] = edge_col[1] if edge_col else -1
        r['edge_row_off'] = edge_row[1] if edge_row else -1
        r['edge_x'] = edge_col[0] if edge_col else 0
        r['edge_y'] = edge_row[0] if edge_row else 0
        r['w'], r['h'] = w, h
        r['start_inside'] = start is not None
        r['xc'], r['yc'] = start if start is not None else (0, 0)
        r['dcx'], r['dcy'] = default_start
        r['minradius'] = minradius
        r['minval'] = minval
        self.rings.append(r)
        return len(self.rings) - 1

    def add(self, x0, y0, w, h, amp, mean, var, fx=0., fy=0., floor=FLOOR_GRID, scale=1.,
            mask=None, out_off=None, ldo=0, mode=MOG_STORE, minval=None, derivs=False,
            diff=None):
        """Adds one mixture evaluated on [x0, x0+w) x [y0, y0+h).  Returns the
        element offset of its output (a packed w x h patch unless `out_off`
        and `ldo` place it inside a larger buffer).  `minval` selects the
        per-component floors of c_gauss_2d_approx3; `derivs` also writes the
        d/dmean_x and d/dmean_y planes right after the patch (packed outputs
        only).  `diff` = (amp2, var2), a second mixture of the same size and
        means: the item renders (mixture 2) - (this mixture), computed with
        its error relative to the difference."""
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
        diff_c0 = -1
        if diff is not None:
            if minval is not None or derivs:
                raise ValueError('difference items take a fixed floor and no derivative planes')
            diff_c0 = self.ncomp + K
        self.items.append((int(x0), int(y0), int(w), int(h), self.ncomp, K, int(mode), int(ldo),
                           float(fx), float(fy), float(floor), float(scale), floor_mode,
                           int(out_off), int(mask_off), 0, int(deriv_off), diff_c0, 0))
        mean = np.array(mean, np.float64).reshape(K, 2)
        self.amp.append(amp)
        self.mean.append(mean)
        self.var.append(np.array(var, np.float64).reshape(K, 2, 2))
        self.ncomp += K
        if diff is not None:
            amp2 = np.array(diff[0], np.float64).ravel()
            if len(amp2) != K:
                raise ValueError('a difference item needs two mixtures of one size')
            self.amp.append(amp2)
            self.mean.append(mean.copy())
            self.var.append(np.array(diff[1], np.float64).reshape(K, 2, 2))
            self.ncomp += K
        return out_off

    def run(self, out=None, stream=None, check=True):
        """Launches one tb_mog_render over all items.  `out` (float32 device
        tensor) defaults to a new packed buffer of all patches followed by
        the launch's 16-byte status word (its last 4 elements)."""
        lib = _lib.load()
        dev = device()
        self.status_in_out = out is None
        if out is None:
            # the launch's status word rides at the end of the packed output,
            # so one copy brings both back
            out = torch.empty(max(self.nout, 1) + 4, dtype=torch.float32, device=dev)
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
        o_ring = pk.add(np.array(self.rings, _lib.RING_ITEM)) if self.rings else None
        o_rst = pk.add(np.zeros(1, _lib.STATUS))
        d = pk.to_device(dev)
        base = d.data_ptr()
        st_ptr = out.data_ptr() + 4 * (out.numel() - 4) if self.status_in_out else base + o_st
        rc = lib.tb_mog_render(base + o_items, len(items), n_tiles, base + o_amp, base + o_mean,
                               base + o_var, None if o_mask is None else base + o_mask,
                               out.data_ptr(), base + o_ctr, st_ptr,
                               _lib.stream_ptr(stream))
        _lib.check(rc, 'tb_mog_render')
        self.extents = None
        self.ring_status = None
        if self.rings:
            self.extents = torch.empty(4 * len(self.rings), dtype=torch.int32, device=dev)
            rc = lib.tb_approx3_region(base + o_ring, len(self.rings), out.data_ptr(),
                                       self.extents.data_ptr(), base + o_rst,
                                       _lib.stream_ptr(stream))
            _lib.check(rc, 'tb_approx3_region')
            self.ring_status = d[o_rst:o_rst + 16]
        self._dev = d
        self.status = (out[-4:].view(torch.uint8) if self.status_in_out else d[o_st:o_st + 16])
        if check:
            check_status(self.status, 'tb_mog_render')
            if self.ring_status is not None:
                check_status(self.ring_status, 'tb_approx3_region')
        return out


    def run_host(self, stream=None):
        """Renders all items with tb_mog_render_host and returns the packed
        float32 output (nout elements) as a host array: inputs staged, the
        launch made, the output and status word read back and the stream
        synchronised in one library call.  Plans without approx3 region
        walks take this path."""
        lib = _lib.load()
        if self.rings:
            raise ValueError('approx3 region walks need the device output (run)')
        out = np.empty(max(self.nout, 1), np.float32)
        if not self.items:
            out[:] = 0.
            return out[:self.nout]
        items = np.array(self.items, dtype=_lib.MOG_ITEM)
        tiles = ((items['w'] + 31) // 32).astype(np.int64) * ((items['h'] + 31) // 32)
        items['tile0'] = np.concatenate([[0], np.cumsum(tiles)[:-1]])
        amp = np.concatenate(self.amp)
        mean = np.concatenate(self.mean)
        var = np.concatenate(self.var)
        masks = np.concatenate(self.masks) if self.masks else None
        nmask = 0 if masks is None else masks.size
        nbytes = ctypes.c_int64()
        _lib.check(lib.tb_mog_render_host_bytes(len(items), amp.size, nmask, self.nout,
                                                ctypes.byref(nbytes)),
                   'tb_mog_render_host_bytes')
        pinned, ws = _host_staging.get(nbytes.value, device())
        st = np.zeros(1, _lib.STATUS)
        rc = lib.tb_mog_render_host(items.ctypes.data, len(items), int(tiles.sum()),
                                    amp.ctypes.data, mean.ctypes.data, var.ctypes.data,
                                    amp.size, None if masks is None else masks.ctypes.data,
                                    nmask, out.ctypes.data, self.nout, st.ctypes.data,
                                    pinned.data_ptr(), ws.data_ptr(), ws.numel(),
                                    _lib.stream_ptr(stream))
        _lib.check(rc, 'tb_mog_render_host')
        check_status_host(st, 'tb_mog_render')
        return out[:self.nout]


class _HostStaging(threading.local):
    """One page-locked host buffer and one device workspace per thread for
    tb_mog_render_host (grown to the next power of two; the call
    synchronises its stream, so both are free again when it returns)."""

    pinned = None
    ws = None

    def get(self, nbytes, dev):
        if self.ws is None or self.ws.numel() < nbytes or self.ws.device != dev:
            size = 1 << max(16, int(np.ceil(np.log2(max(nbytes, 1)))))
            self.pinned = torch.empty(size, dtype=torch.uint8).pin_memory()
            self.ws = torch.empty(size, dtype=torch.uint8, device=dev)
        return self.pinned, self.ws


_host_staging = _HostStaging()


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
        (position-dependent PSFs).  Sizes above 256 (beyond tb_psf_spectrum)
        are transformed in FP64 by cuFFT and rounded to complex64, as the
        reference's np.fft.rfft2 + astype(complex64), into the same
        column-major layout."""
        lib = _lib.load()
        dev = device()
        if sz > 256:
            pad, cx, cy = self.pad(img, sz)
            P = torch.fft.rfft2(torch.from_numpy(pad.astype(np.float64)).to(dev))
            if normalize:
                P = P / torch.abs(P[0, 0])
            P = P.to(torch.complex64).transpose(0, 1).contiguous()   # [v][w]
            return (torch.view_as_real(P).reshape(-1), cx, cy)
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
        self.dcoef = []
        self.ndc = 0
        self.large = []          # items above FFT size 256 (run_large)

    def __len__(self):
        return len(self.items) + len(self.large)

    def add(self, amp, var, sz, spec_key, spec, mw, mh, sx, sy, mux, muy, scale=1.,
            out_off=None, ldo=0, mode=MOG_STORE, diff=None):
        """Adds one galaxy.  `diff` = (amp2, var2), a second mixture of the
        same size: the item renders (mixture 2) - (this mixture) through the
        same geometry (TB_FFT_DIFF), with its error relative to the
        difference."""
        amp = np.array(amp, np.float64).ravel()   # copies, as MogBatch.add
        K = len(amp)
        if K > 128:
            raise ValueError('at most 128 components per galaxy (got %d)' % K)
        if sz < 32 or sz > LARGE_FFT_MAX or (sz & (sz - 1)) != 0:
            raise ValueError('FFT size %d not supported (powers of two, 32..%d)'
                             % (sz, LARGE_FFT_MAX))
        if out_off is None:
            out_off = self.nout
            self.nout += mw * mh
        if sz > 256:
            # beyond the fused renderer: run_large's spectrum grid + cuFFT
            dc = None
            var2 = np.array(var, np.float64).reshape(K, 2, 2)
            if diff is not None:
                amp2 = np.array(diff[0], np.float64).ravel()
                if len(amp2) != K:
                    raise ValueError('a difference item needs two mixtures of one size')
                dv = np.array(diff[1], np.float64).reshape(K, 2, 2) - var2
                dc = np.stack([amp2 - amp, dv[:, 0, 0], 0.5 * (dv[:, 0, 1] + dv[:, 1, 0]),
                               dv[:, 1, 1]], axis=1)
            self.large.append((amp, var2, dc, int(sz), spec, int(mw), int(mh), int(sx), int(sy),
                               float(mux), float(muy), float(scale), int(out_off), int(ldo),
                               int(mode)))
            return out_off
        key = (sz, spec_key)
        if key not in self.spec_off:
            self.spec_off[key] = self.nspec
            self.spec_list.append(spec)
            self.nspec += spec.numel()
        var = np.array(var, np.float64).reshape(K, 2, 2)
        dmode, dc0 = _lib.FFT_VALUE, 0
        if diff is not None:
            amp2 = np.array(diff[0], np.float64).ravel()
            if len(amp2) != K:
                raise ValueError('a difference item needs two mixtures of one size')
            dv = np.array(diff[1], np.float64).reshape(K, 2, 2) - var
            dc = np.stack([amp2 - amp, dv[:, 0, 0], 0.5 * (dv[:, 0, 1] + dv[:, 1, 0]),
                           dv[:, 1, 1]], axis=1)
            dmode, dc0 = _lib.FFT_DIFF, self.ndc
            self.dcoef.append(dc)
            self.ndc += K
        self.items.append((self.ncomp, K, int(sz), int(mode), int(mw), int(mh), int(sx), int(sy),
                           float(mux), float(muy), float(scale), int(ldo), int(out_off),
                           self.spec_off[key], dmode, dc0, 0))
        self.amp.append(amp)
        self.var.append(var)
        self.ncomp += K
        return out_off

    def run(self, out=None, stream=None, check=True):
        lib = _lib.load()
        dev = device()
        self.status_in_out = out is None
        if out is None:
            out = torch.empty(max(self.nout, 1) + 4, dtype=torch.float32, device=dev)
        if self.large:
            self.run_large(out, stream)
        if not self.items:
            if self.status_in_out:
                out[-4:].zero_()
            self.status = out[-4:].view(torch.uint8) if self.status_in_out else None
            return out
        items = np.array(self.items, dtype=_lib.FFT_ITEM)
        specs = torch.cat(self.spec_list) if len(self.spec_list) > 1 else self.spec_list[0]
        pk = _Packer()
        o_items = pk.add(items)
        o_amp = pk.add(np.concatenate(self.amp))
        o_var = pk.add(np.concatenate(self.var))
        o_dc = pk.add(np.concatenate(self.dcoef)) if self.dcoef else None
        o_ctr = pk.add(np.zeros(4, np.int32))
        o_st = pk.add(np.zeros(1, _lib.STATUS))
        d = pk.to_device(dev)
        base = d.data_ptr()
        st_ptr = out.data_ptr() + 4 * (out.numel() - 4) if self.status_in_out else base + o_st
        fourier_render(base + o_items, len(items), base + o_amp, base + o_var, specs.data_ptr(),
                       out.data_ptr(), st_ptr,
                       dcoef_ptr=None if o_dc is None else base + o_dc, stream=stream)
        self._keep = (d, specs)
        self.status = (out[-4:].view(torch.uint8) if self.status_in_out else d[o_st:o_st + 16])
        if check:
            check_status(self.status, 'tb_fourier_render')
        return out


    def run_large(self, out, stream=None):
        """Items whose FFT size exceeds 256 (ProfileGalaxy's FFT branch,
        tractor/galaxy.py:457-519, for galaxies with a half-size above 128):
        the mixture spectrum times the PSF spectrum on the full rfft grid
        (tb_fourier_spectrum_grid), the inverse 2-D real transform as irfftn
        does it (a complex inverse FFT along w, the DC and Nyquist columns'
        imaginary parts dropped, a real inverse FFT along v; cuFFT), the
        Lanczos-3 shift of the whole sz x sz image with zero edges
        (tb_lanczos3_shift, the reference's lanczos_shift_image), then the
        integer shift and crop into the item's rectangle of `out`."""
        lib = _lib.load()
        dev = out.device
        s = _lib.stream_ptr(stream)
        for (amp, var, dc, N, spec, mw, mh, sx, sy, mux, muy, scale, off, ldo,
             mode) in self.large:
            K = len(amp)
            NH = N // 2 + 1
            a_d = torch.as_tensor(amp, device=dev)
            v_d = torch.as_tensor(var.reshape(K, 4), device=dev)
            dc_d = None if dc is None else torch.as_tensor(dc, device=dev)
            S = torch.empty(N * NH * 2, dtype=torch.float32, device=dev)
            rc = lib.tb_fourier_spectrum_grid(a_d.data_ptr() if K else None,
                                              v_d.data_ptr() if K else None,
                                              None if dc_d is None else dc_d.data_ptr(), K,
                                              spec.data_ptr(), N, S.data_ptr(), s)
            _lib.check(rc, 'tb_fourier_spectrum_grid')
            G1 = torch.fft.ifft(torch.view_as_complex(S.view(N, NH, 2)), dim=0)
            G1[:, 0].imag.zero_()
            G1[:, N // 2].imag.zero_()
            G = torch.fft.irfft(G1, n=N, dim=1).to(torch.float32)
            if mux != 0. or muy != 0.:
                G = lanczos_shift(G[None], [(mux, muy)], stream=stream)[0]
            ld = ldo if ldo > 0 else mw
            view = out[off:off + (mh - 1) * ld + mw].as_strided((mh, mw), (ld, 1))
            gr0, gr1 = max(0, -sy), min(N, mh - sy)
            gc0, gc1 = max(0, -sx), min(N, mw - sx)
            if mode == _lib.MOG_STORE:
                view.zero_()
            if gr0 < gr1 and gc0 < gc1:
                blk = G[gr0:gr1, gc0:gc1] * scale
                if mode == _lib.MOG_STORE:
                    view[gr0 + sy:gr1 + sy, gc0 + sx:gc1 + sx] = blk
                else:
                    view[gr0 + sy:gr1 + sy, gc0 + sx:gc1 + sx] += blk


LARGE_FFT_MAX = 8192     # the reference warns above a half-size of 4096 (galaxy.py:376)

_fourier_ws = {}


def fourier_workspace(n_items, dev=None):
    """Device scratch of tb_fourier_render_split for n_items items (one
    buffer per device, grown when needed and reused: launches on one stream
    use it one after another)."""
    lib = _lib.load()
    dev = dev or device()
    nb = ctypes.c_int64()
    _lib.check(lib.tb_fourier_workspace(int(n_items), ctypes.byref(nb)), 'tb_fourier_workspace')
    ws = _fourier_ws.get(dev.index)
    if ws is None or ws.numel() < nb.value:
        ws = torch.empty(max(nb.value, 1 << 20), dtype=torch.uint8, device=dev)
        _fourier_ws[dev.index] = ws
    return ws


FOURIER_METHODS = ('persistent', 'split')
fourier_method = {'default': 'persistent'}   # per device index, set by autotune_fourier


def fourier_render(items_ptr, n_items, amp_ptr, var_ptr, spec_ptr, out_ptr, status_ptr,
                   dcoef_ptr=None, dots_ptr=None, stream=None, method=None):
    """Renders device Fourier items: 'persistent' -- tb_fourier_render(_deriv),
    one CTA per galaxy holding its whole transpose in shared memory -- or
    'split' -- tb_fourier_render_split, column and row kernels through an
    L2-resident scratch.  The default is the device's autotuned choice
    (autotune_fourier), else 'persistent'."""
    lib = _lib.load()
    if method is None:
        dev = device()
        method = fourier_method.get(dev.index, fourier_method['default'])
    s = _lib.stream_ptr(stream)
    if method == 'split':
        ws = fourier_workspace(n_items)
        rc = lib.tb_fourier_render_split(items_ptr, int(n_items), amp_ptr, var_ptr, dcoef_ptr,
                                         spec_ptr, out_ptr, dots_ptr, ws.data_ptr(), ws.numel(),
                                         status_ptr, s)
        _lib.check(rc, 'tb_fourier_render_split')
        return
    ctr = _counter(device())
    if dcoef_ptr is None and dots_ptr is None:
        rc = lib.tb_fourier_render(items_ptr, int(n_items), amp_ptr, var_ptr, spec_ptr, out_ptr,
                                   ctr.data_ptr(), status_ptr, s)
    else:
        rc = lib.tb_fourier_render_deriv(items_ptr, int(n_items), amp_ptr, var_ptr, dcoef_ptr,
                                         spec_ptr, out_ptr, dots_ptr, ctr.data_ptr(), status_ptr,
                                         s)
    _lib.check(rc, 'tb_fourier_render')


_counters = {}


def _counter(dev):
    """A device int32 work counter for the persistent kernels (zeroed by each
    launch on its stream before use)."""
    c = _counters.get(dev.index)
    if c is None:
        c = _counters[dev.index] = torch.zeros(4, dtype=torch.int32, device=dev)
    return c


def autotune_fourier(run, reps=3):
    """Times run(method) for each Fourier method (device events, after a
    warm-up) and makes the fastest this device's default.  Returns
    {method: ms}."""
    dev = device()
    times = {}
    for m in FOURIER_METHODS:
        run(m)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            run(m)
        e1.record()
        e1.synchronize()
        times[m] = e0.elapsed_time(e1) / reps
    fourier_method[dev.index] = min(times, key=times.get)
    return times


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


def solve_dense(A_colmajor, b, damp=0., stream=None):
    """argmin ||A x - b||^2 + damp^2 ||x||^2 of one dense problem given on
    the host (A's columns are the rows of the float32 array A_colmajor, b
    float32): tb_normal_equations + tb_solve_update with one host-to-device
    copy of everything and one device-to-host copy of (x, info).  Returns
    (x float64 numpy array, info)."""
    lib = _lib.load()
    dev = device()
    A_colmajor = np.ascontiguousarray(A_colmajor, np.float32)
    P, R = A_colmajor.shape
    pk = _Packer()
    o_A = pk.add(A_colmajor.ravel())
    o_b = pk.add(np.ascontiguousarray(b, np.float32))
    o_i64 = pk.add(np.array([0, 0, 0, 0, 0], np.int64))     # a_off r_off ata_off atr_off x_off
    o_i32 = pk.add(np.array([R, P, R], np.int32))            # lda P R
    d = pk.to_device(dev)
    base = d.data_ptr()
    ws = torch.empty(P * P + P + P * P + P + 1, dtype=torch.float64, device=dev)
    wb = ws.data_ptr()
    AtA, Atr, work, X, info = wb, wb + 8 * P * P, wb + 8 * (P * P + P), \
        wb + 8 * (2 * P * P + P), wb + 8 * (2 * P * P + 2 * P)
    s = _lib.stream_ptr(stream)
    rc = lib.tb_normal_equations(base + o_A, base + o_b, base + o_i64, base + o_i64 + 8,
                                 base + o_i32, base + o_i32 + 4, base + o_i32 + 8,
                                 base + o_i64 + 16, base + o_i64 + 24, AtA, Atr, 1, P, s)
    _lib.check(rc, 'tb_normal_equations')
    rc = lib.tb_solve_update(AtA, Atr, base + o_i64 + 16, base + o_i64 + 24, base + o_i32 + 4,
                             base + o_i64 + 32, X, info, float(damp), 1, P, work, s)
    _lib.check(rc, 'tb_solve_update')
    host = ws[2 * P * P + P:].cpu().numpy()
    x = host[:P].copy()
    info_v = int(host[P:P + 1].view(np.int32)[0])
    return x, info_v


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
