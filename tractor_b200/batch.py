"""Batched GPU rendering of many sources at once.

FourierGalaxyRenderer renders thousands of galaxies through the
pixelized-PSF Fourier path of ProfileGalaxy._realGetUnitFluxModelPatch
(tractor/galaxy.py:336-519): tb_galaxy_fft_prep turns source parameters into
work items and component tables on the device, and tb_fourier_render_split
renders every item (column and row kernels, 256 items per pair, and the
persistent kernel for the few items they do not cover).
"""
import ctypes

import numpy as np
import torch

from . import _lib, profiles, render

GALAXY_SRC = _lib.GALAXY_SRC
COMP_STRIDE = 10
FFT_SIZES = (32, 64, 128, 256)


class DeviceProfileTables(object):
    """The exp / deV / Sersic profile tables in device memory, in the layout
    tb_profile_tables describes."""

    def __init__(self, device=None):
        t = profiles.tables()
        S = t['sersic']
        lohi, rinfo, sinfo, knots, coefs = [], [], [], [], []

        def add_spline(sp):
            sinfo.append([len(knots), len(sp['t']), len(coefs), sp['k']])
            knots.extend(sp['t'])
            coefs.extend(sp['c'])
            return len(sinfo) - 1

        for r in S['ranges']:
            lohi.extend([r['lo'], r['hi']])
            a0 = len(sinfo)
            for sp in r['amp_splines']:
                add_spline(sp)
            v0 = len(sinfo)
            for sp in r['logvar_splines']:
                add_spline(sp)
            # 1: every spline of the range has the same knots and degree (at
            # most 32 knots), so a warp finds one knot span for all of them
            sps = r['amp_splines'] + r['logvar_splines']
            shared = int(len(sps[0]['t']) <= 32 and
                         all(np.array_equal(sp['t'], sps[0]['t']) and sp['k'] == sps[0]['k']
                             for sp in sps))
            rinfo.append([r['K'], a0, v0, shared])
        core = add_spline(S['core_spline'])
        exp_m, dev_m = profiles.exp_mixture(), profiles.dev_mixture()
        arrays = dict(
            range_lohi=np.array(lohi, np.float64), range_info=np.array(rinfo, np.int32),
            spline_info=np.array(sinfo, np.int32), knots=np.array(knots, np.float64),
            coefs=np.array(coefs, np.float64), exp_amp=exp_m.amp.astype(np.float64),
            exp_var=exp_m.var[:, 0, 0].astype(np.float64), dev_amp=dev_m.amp.astype(np.float64),
            dev_var=dev_m.var[:, 0, 0].astype(np.float64))
        pk = render._Packer()
        offs = dict((k, pk.add(v)) for k, v in arrays.items())
        self.buf = pk.to_device(device or render.device())
        base = self.buf.data_ptr()
        st = _lib.ProfileTables()
        st.n_ranges = len(S['ranges'])
        st.core_spline = core
        for k, o in offs.items():
            setattr(st, k, base + o)
        st.exp_K = len(exp_m.amp)
        st.dev_K = len(dev_m.amp)
        st.n_splines = len(sinfo)
        st.n_knots = len(knots)
        st.n_coefs = len(coefs)
        self.struct = st


_tables = {}


def device_profile_tables():
    dev = render.device()
    if dev.index not in _tables:
        _tables[dev.index] = DeviceProfileTables(dev)
    return _tables[dev.index]


class FourierGalaxyRenderer(object):
    """Galaxies on one image with a constant pixelized PSF.

    psf_img: odd-sized PSF image (PixelizedPSF); normalized: divide each
    spectrum by |P[0,0]| (NormalizedPixelizedPsf); cd_inv / pixscale: the
    image's constant WCS (NullWCS: cd_inv = I * 3600 / pixscale)."""

    def __init__(self, psf_img, pixscale=1., cd_inv=None, normalized=False):
        psf_img = np.asarray(psf_img, np.float32)
        ph, pw = psf_img.shape
        if cd_inv is None:
            cd_inv = np.eye(2) / (pixscale / 3600.)
        specs = []
        img = _lib.FftImage()
        img.cd_inv[:] = list(np.asarray(cd_inv, np.float64).ravel())
        img.pixscale = float(pixscale)
        img.psf_w, img.psf_h = pw, ph
        off = 0
        sp = render.psf_spectra()
        for i, sz in enumerate(FFT_SIZES):
            spec, cx, cy = sp.get(('renderer', id(self), psf_img.tobytes().__hash__()), psf_img, sz,
                                  normalize=normalized)
            specs.append(spec)
            img.psf_cx[i] = cx
            img.psf_cy[i] = cy
            img.spec_off[i] = off
            off += spec.numel()
        self.spec = torch.cat(specs)
        self.image = img
        self.tables = device_profile_tables()
        self._scratch = {}

    def _work(self, n):
        """Device scratch for n sources: items, components, flags, counter,
        status (reused between calls of the same size)."""
        if n not in self._scratch:
            dev = render.device()
            nb = n * _lib.FFT_ITEM.itemsize
            items = torch.empty(nb, dtype=torch.uint8, device=dev)
            camp = torch.empty(n * COMP_STRIDE, dtype=torch.float64, device=dev)
            cvar = torch.empty(n * COMP_STRIDE * 4, dtype=torch.float64, device=dev)
            flags = torch.empty(n, dtype=torch.int32, device=dev)
            misc = torch.zeros(8, dtype=torch.int32, device=dev)   # counter + status
            self._scratch[n] = (items, camp, cvar, flags, misc)
        return self._scratch[n]

    METHODS = ('fused', 'persistent', 'split')

    def render_device(self, srcs, n, out, stream=None, method=None):
        """Renders n sources whose GALAXY_SRC records are in device tensor
        `srcs` (uint8 view) into float32 device tensor `out`; nothing is
        copied to or from the host.  method: 'fused' (tb_galaxy_fft_render:
        preparation and render in one persistent launch), 'persistent' or
        'split' (tb_galaxy_fft_prep, then tb_fourier_render /
        tb_fourier_render_split); None: the method autotune chose, else
        'fused'.  Returns the flags tensor (see tb_galaxy_fft_prep)."""
        lib = _lib.load()
        items, camp, cvar, flags, misc = self._work(n)
        s = _lib.stream_ptr(stream)
        method = method or getattr(self, 'method', None) or 'fused'
        if method == 'fused':
            rc = lib.tb_galaxy_fft_render(srcs.data_ptr(), n, ctypes.addressof(self.image),
                                          ctypes.addressof(self.tables.struct),
                                          self.spec.data_ptr(), out.data_ptr(), items.data_ptr(),
                                          flags.data_ptr(), misc.data_ptr(), misc.data_ptr() + 16,
                                          s)
            _lib.check(rc, 'tb_galaxy_fft_render')
            return flags
        rc = lib.tb_galaxy_fft_prep(srcs.data_ptr(), n, ctypes.addressof(self.image),
                                    ctypes.addressof(self.tables.struct), items.data_ptr(),
                                    camp.data_ptr(), cvar.data_ptr(), COMP_STRIDE,
                                    flags.data_ptr(), s)
        _lib.check(rc, 'tb_galaxy_fft_prep')
        render.fourier_render(items.data_ptr(), n, camp.data_ptr(), cvar.data_ptr(),
                              self.spec.data_ptr(), out.data_ptr(), misc.data_ptr() + 16,
                              stream=stream, method=method)
        return flags

    def autotune(self, srcs, n, out):
        """Times the three methods on these device records (CUDA events,
        after a warm-up each) and keeps the fastest as this renderer's
        method; returns {method: ms}."""
        times = {}
        for m in self.METHODS:
            self.render_device(srcs, n, out, method=m)
            ts = []
            for _ in range(5):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                self.render_device(srcs, n, out, method=m)
                e1.record()
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
            times[m] = float(np.median(ts))
        self.method = min(times, key=times.get)
        return times

    def status(self, n):
        return self._work(n)[4][4:8]

    def render(self, srcs_host, out_host=None, stream=None, method=None):
        """End-to-end call with host buffers: copies the GALAXY_SRC records
        to the device, renders (render_device's `method`), and copies the
        patches back into `out_host` (pinned float32, allocated if None).
        Returns (out_host, flags)."""
        srcs_host = np.ascontiguousarray(srcs_host, dtype=GALAXY_SRC)
        n = len(srcs_host)
        nout = int((srcs_host['out_off'] + srcs_host['mw'].astype(np.int64) * srcs_host['mh']).max())
        dev = render.device()
        if out_host is None:
            out_host = torch.empty(nout, dtype=torch.float32).pin_memory()
        src_pinned = torch.from_numpy(srcs_host.view(np.uint8)).pin_memory()
        d_src = src_pinned.to(dev, non_blocking=True)
        out = torch.empty(nout, dtype=torch.float32, device=dev)
        flags = self.render_device(d_src, n, out, stream, method=method)
        out_host.copy_(out, non_blocking=True)
        flags_host = flags.to('cpu', non_blocking=True)
        torch.cuda.current_stream().synchronize()
        render.check_status(self.status(n).clone(), 'tb_fourier_render')
        return out_host, flags_host.numpy()


def sersic_sources(n, rng, mask=128, pos_jitter=0.5, flux=1000.):
    """Seeded synthetic Sersic galaxies each on its own mask x mask patch
    (`mask` a size, or one size per source; patches packed back to back):
    n ~ U[0.7, 6], r_e log-uniform in [0.5, 8] px, axis ratio U[0.2, 1],
    phi U[0, 180) deg, centre offset U[-0.5, 0.5] px (EllipseE shapes,
    pixel scale 1)."""
    mask = np.broadcast_to(np.asarray(mask, np.int64), (n,))
    srcs = np.zeros(n, GALAXY_SRC)
    ns = rng.uniform(0.7, 6.0, n)
    re = np.exp(rng.uniform(np.log(0.5), np.log(8.0), n))
    q = rng.uniform(0.2, 1.0, n)
    phi = rng.uniform(0., 180., n)
    d = rng.uniform(-pos_jitter, pos_jitter, (n, 2))
    ab = 1. / q
    e = (ab - 1) / (ab + 1)
    ang = np.radians(-2. * phi)
    srcs['px'] = mask / 2 + d[:, 0]
    srcs['py'] = mask / 2 + d[:, 1]
    srcs['counts'] = flux
    srcs['s0'] = re
    srcs['s1'] = e * np.cos(ang)
    srcs['s2'] = e * np.sin(ang)
    srcs['sersic_n'] = ns
    srcs['profile'] = _lib.PROFILE_SERSIC
    srcs['shape_type'] = _lib.SHAPE_ELLIPSE_E
    srcs['mx0'] = 0
    srcs['my0'] = 0
    srcs['mw'] = mask
    srcs['mh'] = mask
    srcs['out_off'] = np.concatenate([[0], np.cumsum(mask * mask)[:-1]])
    return srcs


def moffat_psf(size=63, fwhm=4.0, beta=3.0):
    """Normalised Moffat PSF image (sum 1)."""
    alpha = fwhm / (2 * np.sqrt(2 ** (1 / beta) - 1))
    y, x = np.mgrid[:size, :size] - size // 2
    img = (1 + (x ** 2 + y ** 2) / alpha ** 2) ** (-beta)
    return (img / img.sum()).astype(np.float32)


SCENE_SRC = _lib.SCENE_SRC
SCENE_TILE_HEIGHTS = (16, 32, 64)


def _circ_psf(sigmas, weights):
    K = len(weights)
    var = np.zeros((K, 2, 2))
    var[:, 0, 0] = var[:, 1, 1] = np.asarray(sigmas, np.float64) ** 2
    return np.asarray(weights, np.float64), np.zeros((K, 2)), var


class SceneImage(object):
    """One image of a scene: size, PSF mixture (amp (K,), mean (K, 2), var
    (K, 2, 2)) and the WCS's cdInverse (NullWCS by default)."""

    def __init__(self, W, H, psf_amp, psf_mean, psf_var, pixscale=1., cd_inv=None):
        self.W, self.H = int(W), int(H)
        self.psf_amp = np.asarray(psf_amp, np.float64).ravel()
        K = len(self.psf_amp)
        self.psf_mean = np.asarray(psf_mean, np.float64).reshape(K, 2)
        self.psf_var = np.asarray(psf_var, np.float64).reshape(K, 2, 2)
        self.pixscale = float(pixscale)
        self.cd_inv = (np.eye(2) / (pixscale / 3600.) if cd_inv is None
                       else np.asarray(cd_inv, np.float64).reshape(2, 2))

    @staticmethod
    def circular(W, H, sigmas, weights, pixscale=1.):
        return SceneImage(W, H, *_circ_psf(sigmas, weights), pixscale=pixscale)


class SceneRenderer(object):
    """Many sources into whole float32 images through mixture-of-Gaussians
    PSFs: the batched Tractor.getModelImage (tractor/engine.py:424-445).

    One record (SCENE_SRC) per (source, image).  tb_scene_prep builds every
    record's convolved mixture on the device and tb_scene_render bins the
    records by image tile and renders each tile once.  The images are packed
    back to back in one float32 buffer (image i at `offsets[i]`, row stride
    W).  `tile_h` is the tile height (16, 32 or 64 rows); autotune() picks it
    by timing all three on the caller's workload."""

    def __init__(self, images, comp_stride=None, tile_h=32):
        self.images = list(images)
        if not self.images:
            raise ValueError('a scene needs at least one image')
        self.n_images = len(self.images)
        sizes = np.array([im.W * im.H for im in self.images], np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        self.npix = int(sizes.sum())
        kpsf = max(len(im.psf_amp) for im in self.images)
        if kpsf > 32:
            raise ValueError('at most 32 PSF components')
        # galaxy components: composite exp + deV = 15, Sersic <= 9
        self.comp_stride = comp_stride or 16 * kpsf
        pamp, pmean, pvar, c0 = [], [], [], []
        n = 0
        for im in self.images:
            c0.append(n)
            n += len(im.psf_amp)
            pamp.append(im.psf_amp)
            pmean.append(im.psf_mean)
            pvar.append(im.psf_var)
        pk = render._Packer()
        self._o_pamp = pk.add(np.concatenate(pamp))
        self._o_pmean = pk.add(np.concatenate(pmean))
        self._o_pvar = pk.add(np.concatenate(pvar))
        self._psf = pk.to_device(render.device())
        self._psf_c0 = np.array(c0, np.int32)
        self.tables = device_profile_tables()
        self._img_tables = {}
        self._work = {}
        self.tile_h = tile_h
        self.last_tile_h = None

    # -- tables ------------------------------------------------------------
    def image_table(self, tile_h):
        """Device SCENE_IMAGE table for a tile height, and the tile count."""
        if tile_h not in self._img_tables:
            t = np.zeros(self.n_images, _lib.SCENE_IMAGE)
            tiles = np.array([((im.W + 31) // 32) * ((im.H + tile_h - 1) // tile_h)
                              for im in self.images], np.int64)
            t['W'] = [im.W for im in self.images]
            t['H'] = [im.H for im in self.images]
            t['ldo'] = 0
            t['psf_c0'] = self._psf_c0
            t['psf_K'] = [len(im.psf_amp) for im in self.images]
            t['out_off'] = self.offsets
            t['tile0'] = np.concatenate([[0], np.cumsum(tiles)[:-1]])
            t['cd_inv'] = np.stack([im.cd_inv.ravel() for im in self.images])
            t['pixscale'] = [im.pixscale for im in self.images]
            d = torch.from_numpy(t.view(np.uint8)).to(render.device())
            self._img_tables[tile_h] = (d, int(tiles.sum()))
        return self._img_tables[tile_h]

    def max_pairs(self, srcs_host, tile_h):
        """Upper bound of the (record, tile) overlaps: every record's mask
        clipped to its image, in tiles of 32 x tile_h."""
        s = np.asarray(srcs_host)
        W = np.array([im.W for im in self.images])[s['image']]
        H = np.array([im.H for im in self.images])[s['image']]
        x0 = np.maximum(s['mx0'], 0)
        y0 = np.maximum(s['my0'], 0)
        x1 = np.minimum(s['mx0'] + s['mw'], W)
        y1 = np.minimum(s['my0'] + s['mh'], H)
        ok = (x1 > x0) & (y1 > y0)
        nx = np.where(ok, (x1 - 1) // 32 - x0 // 32 + 1, 0)
        ny = np.where(ok, (y1 - 1) // tile_h - y0 // tile_h + 1, 0)
        return int((nx.astype(np.int64) * ny).sum())

    def workspace(self, n, max_pairs, tile_h):
        """Device scratch (reused while the sizes allow)."""
        lib = _lib.load()
        _, n_tiles = self.image_table(tile_h)
        nb = ctypes.c_int64()
        _lib.check(lib.tb_scene_workspace(n_tiles, max_pairs, ctypes.byref(nb)),
                   'tb_scene_workspace')
        w = self._work.get('buf')
        if (w is None or w[0] < n or w[1].numel() < nb.value):
            dev = render.device()
            items = torch.empty(max(n, 1) * _lib.SCENE_ITEM.itemsize, dtype=torch.uint8, device=dev)
            comps = torch.empty(max(n, 1) * self.comp_stride * 7, dtype=torch.float64, device=dev)
            ws = torch.empty(nb.value, dtype=torch.uint8, device=dev)
            status = torch.zeros(4, dtype=torch.int32, device=dev)
            w = (n, ws, items, comps, status)
            self._work['buf'] = w
        return w

    # -- rendering ---------------------------------------------------------
    def render_device(self, d_srcs, n, out, max_pairs, tile_h=None, mode=_lib.MOG_STORE,
                      stream=None):
        """Renders n records whose SCENE_SRC rows are in device tensor
        `d_srcs` (uint8 view) into the float32 device tensor `out` (npix
        elements).  Two launches for the prep and five for binning and
        rendering; nothing is copied to or from the host."""
        lib = _lib.load()
        tile_h = tile_h or self.tile_h
        d_img, n_tiles = self.image_table(tile_h)
        _, ws, items, comps, status = self.workspace(n, max_pairs, tile_h)
        stride = self.comp_stride
        base = comps.data_ptr()
        camp, cmean, cvar = base, base + 8 * n * stride, base + 24 * n * stride
        s = _lib.stream_ptr(stream)
        pb = self._psf.data_ptr()
        rc = lib.tb_scene_prep(d_srcs.data_ptr(), n, d_img.data_ptr(), self.n_images,
                               pb + self._o_pamp, pb + self._o_pmean, pb + self._o_pvar,
                               ctypes.addressof(self.tables.struct), items.data_ptr(), camp, cmean,
                               cvar, stride, s)
        _lib.check(rc, 'tb_scene_prep')
        rc = lib.tb_scene_render(items.data_ptr(), n, d_img.data_ptr(), self.n_images, n_tiles,
                                 tile_h, camp, cmean, cvar, out.data_ptr(), mode, ws.data_ptr(),
                                 ws.numel(), max_pairs, status.data_ptr(), s)
        _lib.check(rc, 'tb_scene_render')
        self.last_tile_h = tile_h
        return status

    def items(self, n):
        """The prepared SCENE_ITEM records of the last render (host copy)."""
        return self._work['buf'][2][:n * _lib.SCENE_ITEM.itemsize].cpu().numpy().view(
            _lib.SCENE_ITEM)

    def render(self, srcs_host, out_host=None, tile_h=None, stream=None):
        """End-to-end call with host buffers: copies the records to the
        device, renders, copies the images back (pinned float32, allocated if
        None) and checks the device status.  Returns the packed images."""
        srcs_host = np.ascontiguousarray(srcs_host, dtype=SCENE_SRC)
        n = len(srcs_host)
        tile_h = tile_h or self.tile_h
        dev = render.device()
        if out_host is None:
            out_host = torch.empty(self.npix, dtype=torch.float32).pin_memory()
        mp = self.max_pairs(srcs_host, tile_h)
        d_src = torch.from_numpy(srcs_host.view(np.uint8)).pin_memory().to(dev, non_blocking=True)
        out = torch.empty(self.npix, dtype=torch.float32, device=dev)
        status = self.render_device(d_src, n, out, mp, tile_h, stream=stream)
        out_host.copy_(out, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        render.check_status(status.clone(), 'tb_scene_render')
        return out_host

    def image(self, packed, i):
        """View of image i (H, W) in a packed buffer."""
        im = self.images[i]
        o = int(self.offsets[i])
        return packed[o:o + im.W * im.H].reshape(im.H, im.W)

    def autotune(self, d_srcs, n, max_pairs_by_h, reps=3):
        """Times every tile height on this workload (CUDA events, after one
        warm-up each), keeps the fastest as self.tile_h and returns
        {tile_h: ms}."""
        dev = render.device()
        out = torch.empty(self.npix, dtype=torch.float32, device=dev)
        times = {}
        for th in SCENE_TILE_HEIGHTS:
            mp = max_pairs_by_h[th]
            self.render_device(d_srcs, n, out, mp, th)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                self.render_device(d_srcs, n, out, mp, th)
            e1.record()
            e1.synchronize()
            times[th] = e0.elapsed_time(e1) / reps
        self.tile_h = min(times, key=times.get)
        return times


def scene_sources(n, rng, W=4096, H=4096, image=0, hw_range=(7, 127), flux_range=(10., 1e5),
                  mix=(0.4, 0.3, 0.2, 0.1)):
    """Seeded synthetic scene: n sources uniformly placed on a W x H image,
    kinds point / exp / deV / composite with probabilities `mix`, fluxes
    log-uniform in flux_range, square ModelMasks of half-width log-uniform
    in hw_range centred on the nearest pixel, EllipseE shapes with r_e
    log-uniform in [0.5, 8] px, axis ratio U[0.2, 1], phi U[0, 180)."""
    s = np.zeros(n, SCENE_SRC)
    kind = rng.choice(4, size=n, p=list(mix))
    profile = np.array([_lib.PROFILE_POINT, _lib.PROFILE_EXP, _lib.PROFILE_DEV,
                        _lib.PROFILE_COMPOSITE])[kind]
    px = rng.uniform(0, W, n)
    py = rng.uniform(0, H, n)
    flux = np.exp(rng.uniform(np.log(flux_range[0]), np.log(flux_range[1]), n))
    hw = np.round(np.exp(rng.uniform(np.log(hw_range[0]), np.log(hw_range[1]), n))).astype(int)

    def ellipse():
        re = np.exp(rng.uniform(np.log(0.5), np.log(8.), n))
        q = rng.uniform(0.2, 1., n)
        phi = rng.uniform(0., 180., n)
        ab = 1. / q
        e = (ab - 1) / (ab + 1)
        ang = np.radians(-2. * phi)
        return re, e * np.cos(ang), e * np.sin(ang)

    s['sa0'], s['sa1'], s['sa2'] = ellipse()
    s['sb0'], s['sb1'], s['sb2'] = ellipse()
    s['fdev'] = rng.uniform(0., 1., n)
    s['px'], s['py'], s['counts'] = px, py, flux
    s['profile'] = profile
    s['shape_type'] = _lib.SHAPE_ELLIPSE_E
    s['image'] = image
    cx, cy = np.round(px).astype(int), np.round(py).astype(int)
    s['mx0'], s['my0'] = cx - hw, cy - hw
    s['mw'] = s['mh'] = 2 * hw + 1
    return s
