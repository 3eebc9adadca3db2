"""Batched GPU rendering of many sources at once.

FourierGalaxyRenderer renders thousands of galaxies through the
pixelized-PSF Fourier path of ProfileGalaxy._realGetUnitFluxModelPatch
(tractor/galaxy.py:336-519) in two launches: tb_galaxy_fft_prep turns source
parameters into work items and component tables on the device, and
tb_fourier_render renders every item in one persistent launch.
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
            rinfo.append([r['K'], a0, v0, 0])
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

    def render_device(self, srcs, n, out, stream=None):
        """Renders n sources whose GALAXY_SRC records are in device tensor
        `srcs` (uint8 view) into float32 device tensor `out`.  Two kernel
        launches; nothing is copied to or from the host.  Returns the flags
        tensor (see tb_galaxy_fft_prep)."""
        lib = _lib.load()
        items, camp, cvar, flags, misc = self._work(n)
        s = _lib.stream_ptr(stream)
        rc = lib.tb_galaxy_fft_prep(srcs.data_ptr(), n, ctypes.addressof(self.image),
                                    ctypes.addressof(self.tables.struct), items.data_ptr(),
                                    camp.data_ptr(), cvar.data_ptr(), COMP_STRIDE,
                                    flags.data_ptr(), s)
        _lib.check(rc, 'tb_galaxy_fft_prep')
        rc = lib.tb_fourier_render(items.data_ptr(), n, camp.data_ptr(), cvar.data_ptr(),
                                   self.spec.data_ptr(), out.data_ptr(), misc.data_ptr(),
                                   misc.data_ptr() + 16, s)
        _lib.check(rc, 'tb_fourier_render')
        return flags

    def status(self, n):
        return self._work(n)[4][4:8]

    def render(self, srcs_host, out_host=None, stream=None):
        """End-to-end call with host buffers: copies the GALAXY_SRC records
        to the device, renders, and copies the patches back into `out_host`
        (pinned float32, allocated if None).  Returns (out_host, flags)."""
        srcs_host = np.ascontiguousarray(srcs_host, dtype=GALAXY_SRC)
        n = len(srcs_host)
        nout = int((srcs_host['out_off'] + srcs_host['mw'].astype(np.int64) * srcs_host['mh']).max())
        dev = render.device()
        if out_host is None:
            out_host = torch.empty(nout, dtype=torch.float32).pin_memory()
        src_pinned = torch.from_numpy(srcs_host.view(np.uint8)).pin_memory()
        d_src = src_pinned.to(dev, non_blocking=True)
        out = torch.empty(nout, dtype=torch.float32, device=dev)
        flags = self.render_device(d_src, n, out, stream)
        out_host.copy_(out, non_blocking=True)
        flags_host = flags.to('cpu', non_blocking=True)
        torch.cuda.current_stream().synchronize()
        render.check_status(self.status(n).clone(), 'tb_fourier_render')
        return out_host, flags_host.numpy()


def sersic_sources(n, rng, mask=128, pos_jitter=0.5, flux=1000.):
    """Seeded synthetic Sersic galaxies each on its own mask x mask patch:
    n ~ U[0.7, 6], r_e log-uniform in [0.5, 8] px, axis ratio U[0.2, 1],
    phi U[0, 180) deg, centre offset U[-0.5, 0.5] px (EllipseE shapes,
    pixel scale 1)."""
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
    srcs['out_off'] = np.arange(n, dtype=np.int64) * mask * mask
    return srcs


def moffat_psf(size=63, fwhm=4.0, beta=3.0):
    """Normalised Moffat PSF image (sum 1)."""
    alpha = fwhm / (2 * np.sqrt(2 ** (1 / beta) - 1))
    y, x = np.mgrid[:size, :size] - size // 2
    img = (1 + (x ** 2 + y ** 2) / alpha ** 2) ** (-beta)
    return (img / img.sum()).astype(np.float32)
