"""Batched blob fitting on the device: Levenberg-Marquardt over many
independent blobs at once (tb_fit_prep / tb_fit_pass / tb_fit_step).

A blob is a few sources (SersicGalaxy, ExpGalaxy, DevGalaxy or PointSource)
seen in up to three aligned band images with mixture-of-Gaussians PSFs.  The
fitter is the batched form of Tractor.optimize_loop with LsqrOptimizer
(tractor/lsqr_optimizer.py:280-326): every iteration renders every blob's
model and analytic derivatives, forms the normal equations per blob, and
takes one damped Gauss-Newton step with ConstrainedOptimizer's step limits;
a blob stops when the predicted log-likelihood gain of its next step is below
`tol` (optimize_loop's dchisq, tested on the prediction, which FP32 noise in
chi^2 does not disturb).  Only the 32 x 8 tiles that some source's mask
reaches are visited per iteration; the chi^2 of the others is computed once.
Iterations run as CUDA graphs of `check_every` steps; the host only counts
the running blobs between graphs.

Parameters per source (TB_FIT_NPAR = 9 slots): x, y, flux[3] (counts),
log r_e, ee1, ee2 (EllipseESoft), Sersic n.
"""
import ctypes

import numpy as np
import torch

from . import _lib, batch, render

NPAR = _lib.FIT_NPAR
UNIT_TILES = 64      # active 32 x 8 tiles per pass unit (larger images are split)
SERSIC_MIN, SERSIC_MAX = 0.29, 6.3


class BlobFitter(object):
    """Device state for fitting a set of blobs.

    blob_src:   (n_blobs + 1,) source offsets (sources of blob b are
                blob_src[b] .. blob_src[b+1]);
    sides:      (n_blobs, 2) image (W, H) of every blob (all bands alike);
    psf:        (n_blobs, n_bands) tuples (amp (K,), mean (K, 2), var (K, 2, 2));
    sources:    FIT_SOURCE records (profile, mask rectangle in blob pixels);
    params0:    (n_src, 9) starting parameters;
    data, inverr: float32 device tensors, unit (blob, band) images packed in
                blob-major, band-minor order (see `pix_offsets`);
    unit_tiles: active 32 x 8 tiles per pass unit at most (a (blob, band)
                image with more is split into that many units, each with its
                own partial normal-equation slice)."""

    def __init__(self, blob_src, sides, psf, sources, params0, data, inverr, n_bands=3,
                 cd_inv=None, unit_tiles=UNIT_TILES):
        lib = _lib.load()
        self.dev = render.device()
        self.n_bands = int(n_bands)
        if not 1 <= self.n_bands <= _lib.FIT_MAX_BANDS:
            raise ValueError('1 to 3 bands')
        blob_src = np.asarray(blob_src, np.int64)
        self.n_blobs = len(blob_src) - 1
        nsrc = np.diff(blob_src)
        if nsrc.min() < 1 or nsrc.max() > _lib.FIT_MAX_SRC:
            raise ValueError('every blob needs 1 to %d sources' % _lib.FIT_MAX_SRC)
        self.n_src = int(blob_src[-1])
        sides = np.asarray(sides, np.int64).reshape(self.n_blobs, 2)
        P = nsrc * NPAR
        blobs = np.zeros(self.n_blobs, _lib.FIT_BLOB)
        blobs['n_src'] = nsrc
        blobs['src0'] = blob_src[:-1]
        blobs['P'] = P
        tiles, n_active, n_tiles = blob_tiles(sides, sources, blob_src)
        blobs['n_active'] = n_active
        blobs['n_tiles'] = n_tiles
        blobs['tile_off'] = np.concatenate([[0], np.cumsum(n_tiles)[:-1]])
        # a band's active tiles go to ceil(n_active / UNIT_TILES) pass units,
        # each with its own partial blocks (slices), so that no unit holds
        # one CTA for long while few blobs are still running
        unit_tiles = int(unit_tiles)
        if unit_tiles < 1:
            raise ValueError('unit_tiles must be positive')
        parts = np.maximum(1, -(-n_active // unit_tiles)).astype(np.int64)
        n_slices = self.n_bands * parts
        blobs['n_slices'] = n_slices
        blobs['unit0'] = np.concatenate([[0], np.cumsum(n_slices)[:-1]])
        hsz = (n_slices + 2) * P * P
        gsz = (n_slices + 1) * P
        blobs['h_off'] = np.concatenate([[0], np.cumsum(hsz)[:-1]])
        blobs['g_off'] = np.concatenate([[0], np.cumsum(gsz)[:-1]])
        self.pix_offsets = pix_offsets(sides, self.n_bands)
        units = np.zeros(self.n_blobs * self.n_bands, _lib.FIT_UNIT)
        for b in range(self.n_blobs):
            for k in range(self.n_bands):
                u = units[b * self.n_bands + k]
                u['blob'], u['band'] = b, k
                u['W'], u['H'] = sides[b]
                u['pix_off'] = self.pix_offsets[b * self.n_bands + k]
                amp, mean, var = psf[b][k]
                K = len(amp)
                if K > _lib.FIT_MAX_PSF:
                    raise ValueError('at most %d PSF components' % _lib.FIT_MAX_PSF)
                u['psf_K'] = K
                u['psf_amp'][:K] = amp
                u['psf_mean'][:2 * K] = np.asarray(mean, np.float64).ravel()
                u['psf_var'][:4 * K] = np.asarray(var, np.float64).ravel()
        units['t1'] = n_active[units['blob']]
        units['slice'] = units['band']
        # pass units: the (blob, band) images split into tile ranges
        pu = []
        for b in range(self.n_blobs):
            q = int(parts[b])
            cut = (np.arange(q + 1) * int(n_active[b])) // q
            for k in range(self.n_bands):
                for j in range(q):
                    u = units[b * self.n_bands + k].copy()
                    u['slice'] = k * q + j
                    u['t0'], u['t1'] = cut[j], cut[j + 1]
                    pu.append(u)
        pass_units = np.array(pu, _lib.FIT_UNIT)
        # the pass takes units largest first
        cost = (pass_units['t1'] - pass_units['t0']).astype(np.float64) * \
            (1 + nsrc[pass_units['blob']])
        order = np.argsort(-cost, kind='stable').astype(np.int32)
        npix = int(self.pix_offsets[-1])
        if data.numel() < npix or inverr.numel() < npix:
            raise ValueError('data / inverr hold %d pixels, the blobs need %d' %
                             (min(data.numel(), inverr.numel()), npix))
        self.data, self.inverr = data, inverr
        to = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(self.dev)
        self.blobs_np, self.units_np, self.pass_units_np = blobs, units, pass_units
        self.d_blobs, self.d_units = to(blobs), to(units)
        self.d_pass_units = to(pass_units)
        self.d_order = torch.from_numpy(order).to(self.dev)
        self.sources_np = np.ascontiguousarray(sources, _lib.FIT_SOURCE).copy()
        self.sources_np['blob'] = np.repeat(np.arange(self.n_blobs), nsrc)
        self.d_sources = to(self.sources_np)
        self.params = torch.from_numpy(np.ascontiguousarray(params0, np.float64).reshape(-1)).to(
            self.dev)
        self.trial = self.params.clone()
        self.hbuf = torch.zeros(int(hsz.sum()), dtype=torch.float64, device=self.dev)
        self.gbuf = torch.zeros(int(gsz.sum()), dtype=torch.float64, device=self.dev)
        self.d_tiles = torch.from_numpy(tiles).to(self.dev)
        self.chi2_part = torch.zeros(int(n_slices.sum()), dtype=torch.float64,
                                     device=self.dev)
        self.chi2_const = torch.zeros_like(self.chi2_part)
        self._const_done = False
        self.state = torch.zeros(self.n_blobs * _lib.FIT_STATE.itemsize, dtype=torch.uint8,
                                 device=self.dev)
        nb = ctypes.c_int64()
        _lib.check(lib.tb_fit_workspace(self.n_src, self.n_bands, ctypes.byref(nb)),
                   'tb_fit_workspace')
        self.workspace = torch.empty(max(nb.value, 256), dtype=torch.uint8, device=self.dev)
        self.misc = torch.zeros(8, dtype=torch.int32, device=self.dev)   # counter + status
        cd = np.eye(2) * 3600. if cd_inv is None else np.asarray(cd_inv, np.float64)
        self.cd_inv = np.ascontiguousarray(cd, np.float64).ravel()
        self.tables = batch.device_profile_tables()
        self.iterations = 0
        self._graph = None

    # -- one iteration -----------------------------------------------------
    def _prep(self, all_blobs=False):
        lib = _lib.load()
        _lib.check(lib.tb_fit_prep(self.d_sources.data_ptr(), self.n_src, self.trial.data_ptr(),
                                   self.n_bands, self.d_units.data_ptr(), len(self.units_np),
                                   self.cd_inv.ctypes.data, ctypes.addressof(self.tables.struct),
                                   self.workspace.data_ptr(),
                                   None if all_blobs else self.state.data_ptr(),
                                   _lib.stream_ptr()), 'tb_fit_prep')

    def _pass(self, mode):
        lib = _lib.load()
        _lib.check(lib.tb_fit_pass(self.d_pass_units.data_ptr(), self.d_order.data_ptr(),
                                   len(self.pass_units_np), self.d_blobs.data_ptr(),
                                   self.d_sources.data_ptr(), self.n_src,
                                   self.workspace.data_ptr(), self.data.data_ptr(),
                                   self.inverr.data_ptr(), self.d_tiles.data_ptr(),
                                   self.hbuf.data_ptr(), self.gbuf.data_ptr(),
                                   self.chi2_part.data_ptr(), self.chi2_const.data_ptr(),
                                   self.state.data_ptr(), self.n_bands, mode,
                                   self.misc.data_ptr(), self.misc.data_ptr() + 16,
                                   _lib.stream_ptr()), 'tb_fit_pass')

    def _refine_pass(self):
        """A^T A, A^T r and chi^2 of the running blobs in FP64
        (tb_fit_refine), into the slices the FP32 pass writes."""
        lib = _lib.load()
        _lib.check(lib.tb_fit_refine(self.d_pass_units.data_ptr(), self.d_order.data_ptr(),
                                     len(self.pass_units_np), self.d_blobs.data_ptr(),
                                     self.d_sources.data_ptr(), self.n_src,
                                     self.workspace.data_ptr(), self.data.data_ptr(),
                                     self.inverr.data_ptr(), self.d_tiles.data_ptr(),
                                     self.hbuf.data_ptr(), self.gbuf.data_ptr(),
                                     self.chi2_part.data_ptr(),
                                     self.chi2_const.data_ptr(), self.state.data_ptr(),
                                     self.n_bands, self.misc.data_ptr(),
                                     self.misc.data_ptr() + 16, _lib.stream_ptr()),
                   'tb_fit_refine')

    def _iteration(self, tol, max_iter, precise=False):
        lib = _lib.load()
        s = _lib.stream_ptr()
        self._prep()
        if precise:
            self._refine_pass()
        else:
            self._pass(0)
        _lib.check(lib.tb_fit_step(self.d_blobs.data_ptr(), self.n_blobs, self.n_bands,
                                   self.d_sources.data_ptr(), self.params.data_ptr(),
                                   self.trial.data_ptr(), self.hbuf.data_ptr(),
                                   self.gbuf.data_ptr(), self.chi2_part.data_ptr(),
                                   self.state.data_ptr(), float(tol), int(max_iter), s),
                   'tb_fit_step')

    def reset(self, params0=None, lambda0=1e-3):
        lib = _lib.load()
        if params0 is not None:
            self.params.copy_(torch.as_tensor(np.asarray(params0, np.float64).reshape(-1)))
        self.trial.copy_(self.params)
        _lib.check(lib.tb_fit_reset(self.state.data_ptr(), self.n_blobs, float(lambda0),
                                    _lib.stream_ptr()), 'tb_fit_reset')
        self.iterations = 0
        if not self._const_done:
            # chi^2 of the tiles no source reaches: fixed for the data set
            self._prep()
            self._pass(1)
            self._const_done = True

    def running(self):
        st = self.state.view(torch.int32).view(self.n_blobs, _lib.FIT_STATE.itemsize // 4)
        return int((st[:, -1] == 0).sum().item())

    def fit(self, tol=1e-3, max_iter=200, check_every=4, graph=True, params0=None,
            lambda0=1e-3, refine=True, refine_tol=1e-9, refine_iter=100, handoff=0.005):
        """Runs FP32 iterations until every blob stops (or max_iter); then,
        with `refine`, continues every blob from where it stopped with the
        normal equations in FP64 (tb_fit_refine in place of the pass) until
        the predicted gain is below refine_tol (or refine_iter): the FP32
        objective cannot resolve the last ~1e-4 of log-likelihood, which
        leaves the flat directions of a blob a few 1e-3 sigma from the
        optimum, and an FP32 A^T A is too inexact for an ill-conditioned
        blob's steps to converge.  With `refine`, the FP32 phase also ends
        once at most a fraction `handoff` of the blobs still runs: those
        continue in the FP64 phase from where they are.  The slowest blobs
        of a 2,000-blob fit of 192-512 px blobs need about 60 FP64
        iterations (Gauss-Newton steps rejected and re-damped along an
        ill-conditioned direction); 40 left some of them several sigma from
        the optimum.  Returns the number of iterations launched (both
        phases)."""
        self.reset(params0, lambda0)
        g = None
        if graph:
            g = self._capture(check_every, tol, max_iter)
        while self.iterations < max_iter:
            if g is not None:
                g.replay()
            else:
                for _ in range(check_every):
                    self._iteration(tol, max_iter)
            self.iterations += check_every
            r = self.running()
            if r == 0 or (refine and r <= handoff * self.n_blobs):
                break
        if refine:
            # the FP64 phase starts every blob again from its parameters
            # (the first pass is accepted: the FP64 chi^2 is not comparable
            # with the FP32 one)
            # near the optimum: Gauss-Newton steps (a Marquardt damping of
            # 1e-9; a damped start would crawl along the flat directions)
            n = self.iterations
            self.reset(None, 1e-9)
            self.iterations = n
            for it in range(int(refine_iter)):
                self._iteration(refine_tol, refine_iter, precise=True)
                self.iterations += 1
                if it % 2 == 1 and self.running() == 0:
                    break
        return self.iterations

    def _capture(self, k, tol, max_iter):
        key = (k, float(tol), int(max_iter))
        if self._graph is not None and self._graph[0] == key:
            return self._graph[1]
        # warm-up launch outside capture (function attributes, lazy loading),
        # then restore the starting state
        p0 = self.params.clone()
        s0 = self.state.clone()
        self._iteration(tol, max_iter)
        torch.cuda.synchronize()
        self.params.copy_(p0)
        self.trial.copy_(p0)
        self.state.copy_(s0)
        g = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            with torch.cuda.graph(g, stream=side):
                for _ in range(k):
                    self._iteration(tol, max_iter)
        torch.cuda.current_stream().wait_stream(side)
        self._graph = (key, g)
        return g

    # -- results -------------------------------------------------------------
    def states(self):
        return self.state.cpu().numpy().view(_lib.FIT_STATE)

    def result(self):
        return self.params.cpu().numpy().reshape(self.n_src, NPAR)

    def normal_equations(self, b):
        """(H, g) of blob b at the last accepted parameters (FP64, host)."""
        bl = self.blobs_np[b]
        P = int(bl['P'])
        h0 = int(bl['h_off']) + int(bl['n_slices']) * P * P
        g0 = int(bl['g_off']) + int(bl['n_slices']) * P
        H = self.hbuf[h0:h0 + P * P].cpu().numpy().reshape(P, P)
        g = self.gbuf[g0:g0 + P].cpu().numpy()
        return H, g

    def status(self):
        return self.misc[4:8]


def blob_tiles(sides, sources, blob_src):
    """Per blob, its 32 x 8 tiles, encoded tx | ty << 10 | (s + 1) << 20:
    first the tiles exactly one source mask reaches (s, grouped by source:
    the fitting pass accumulates such runs in registers), then the tiles
    several masks reach (s + 1 = 0), then the others.  Returns (tiles,
    n_active, n_tiles)."""
    sides = np.asarray(sides, np.int64).reshape(-1, 2)
    out, n_act, n_all = [], [], []
    for b in range(len(sides)):
        W, H = sides[b]
        tx_n, ty_n = (W + 31) // 32, (H + 7) // 8
        count = np.zeros((ty_n, tx_n), np.int32)
        last = np.full((ty_n, tx_n), -1, np.int32)
        for k, r in enumerate(sources[blob_src[b]:blob_src[b + 1]]):
            x0, x1 = max(r['x0'], 0), min(r['x0'] + r['w'], W)
            y0, y1 = max(r['y0'], 0), min(r['y0'] + r['h'], H)
            if x1 > x0 and y1 > y0:
                sl = (slice(y0 // 8, (y1 - 1) // 8 + 1), slice(x0 // 32, (x1 - 1) // 32 + 1))
                count[sl] += 1
                last[sl] = k
        ty, tx = np.nonzero(count == 1)
        src = last[ty, tx]
        order = np.lexsort((tx, ty, src))
        single = tx[order] | (ty[order] << 10) | ((src[order] + 1) << 20)
        my, mx = np.nonzero(count > 1)
        multi = mx | (my << 10)
        py_, px_ = np.nonzero(count == 0)
        passive = px_ | (py_ << 10)
        out.append(np.concatenate([single, multi, passive]).astype(np.int32))
        n_act.append(len(single) + len(multi))
        n_all.append(tx_n * ty_n)
    return np.concatenate(out), np.array(n_act, np.int32), np.array(n_all, np.int32)


def pix_offsets(sides, n_bands):
    """Element offsets of the (blob, band) images packed blob-major (and the
    total at the end)."""
    sides = np.asarray(sides, np.int64).reshape(-1, 2)
    sz = np.repeat(sides[:, 0] * sides[:, 1], n_bands)
    return np.concatenate([[0], np.cumsum(sz)]).astype(np.int64)


def esoft_from_rabphi(re, q, phi):
    """EllipseESoft (log r_e, ee1, ee2) of radius, axis ratio, angle (deg)."""
    ab = 1. / np.asarray(q, np.float64)
    e = np.minimum((ab - 1) / (ab + 1), 0.999999)
    ee = -np.log(1. - e)
    ang = np.radians(-2. * np.asarray(phi, np.float64))
    return np.log(re), ee * np.cos(ang), ee * np.sin(ang)


def blob_workload(n_blobs, rng, side_range=(192, 512), n_bands=3, mean_src=6, max_src=30,
                  flux_range=(500., 5e4), noise_range=(1., 3.)):
    """Seeded synthetic blobs: sides U[side_range], Poisson(mean_src) Sersic
    sources clipped to [1, max_src] placed uniformly, n U[0.7, 6], r_e
    log-U[0.5, 8] px, axis ratio U[0.2, 1], phi U[0, 180), per-band fluxes
    log-uniform in flux_range, per (blob, band) 3-component MoG PSF
    (sigma1 U[1, 2], x2, x4; weights 0.7 / 0.2 / 0.1) and Gaussian noise
    sigma U[noise_range].  Square masks of half-width
    clip(round(6 r_e + 12 sigma1), 8, 64).  Returns a dict of host arrays
    (truth, a perturbed start, geometry)."""
    side = rng.integers(side_range[0], side_range[1] + 1, n_blobs)
    nsrc = np.clip(rng.poisson(mean_src, n_blobs), 1, max_src)
    blob_src = np.concatenate([[0], np.cumsum(nsrc)]).astype(np.int64)
    n = int(blob_src[-1])
    blob_of = np.repeat(np.arange(n_blobs), nsrc)
    s1 = rng.uniform(1., 2., (n_blobs, n_bands))
    noise = rng.uniform(noise_range[0], noise_range[1], (n_blobs, n_bands))
    truth = np.zeros((n, NPAR))
    S = side[blob_of]
    truth[:, 0] = rng.uniform(8, S - 8)
    truth[:, 1] = rng.uniform(8, S - 8)
    for k in range(n_bands):
        truth[:, 2 + k] = np.exp(rng.uniform(np.log(flux_range[0]), np.log(flux_range[1]), n))
    re = np.exp(rng.uniform(np.log(0.5), np.log(8.), n))
    q = rng.uniform(0.2, 1., n)
    phi = rng.uniform(0., 180., n)
    truth[:, 5], truth[:, 6], truth[:, 7] = esoft_from_rabphi(re, q, phi)
    truth[:, 8] = rng.uniform(0.7, 6., n)
    start = truth.copy()
    start[:, 0:2] += rng.uniform(-0.5, 0.5, (n, 2))
    start[:, 2:2 + n_bands] *= rng.uniform(0.8, 1.25, (n, n_bands))
    start[:, 5] += rng.uniform(-0.2, 0.2, n)
    start[:, 6:8] += rng.uniform(-0.05, 0.05, (n, 2))
    start[:, 8] = np.clip(start[:, 8] + rng.uniform(-0.5, 0.5, n), 0.5, 6.)
    hw = np.clip(np.round(6 * re + 12 * s1.max(axis=1)[blob_of]), 8, 64).astype(np.int64)
    cx = np.round(truth[:, 0]).astype(np.int64)
    cy = np.round(truth[:, 1]).astype(np.int64)
    sources = np.zeros(n, _lib.FIT_SOURCE)
    sources['profile'] = _lib.PROFILE_SERSIC
    sources['x0'], sources['y0'] = cx - hw, cy - hw
    sources['w'] = sources['h'] = 2 * hw + 1
    psf = []
    for b in range(n_blobs):
        row = []
        for k in range(n_bands):
            sig = np.array([1., 2., 4.]) * s1[b, k]
            var = np.zeros((3, 2, 2))
            var[:, 0, 0] = var[:, 1, 1] = sig ** 2
            row.append((np.array([0.7, 0.2, 0.1]), np.zeros((3, 2)), var))
        psf.append(row)
    return dict(blob_src=blob_src, sides=np.stack([side, side], 1), psf=psf, sources=sources,
                truth=truth, start=start, noise=noise, n_bands=n_bands)


def subset_workload(w, blobs):
    """The workload dict of blob_workload restricted to `blobs` (indices,
    kept in their order): a rank's share of a partitioned fit."""
    blobs = np.asarray(blobs, np.int64)
    bs = w['blob_src']
    src = np.concatenate([np.arange(bs[b], bs[b + 1]) for b in blobs]) if len(blobs) else \
        np.zeros(0, np.int64)
    nsrc = np.diff(bs)[blobs]
    out = dict(w)
    out['blob_src'] = np.concatenate([[0], np.cumsum(nsrc)]).astype(np.int64)
    out['sides'] = w['sides'][blobs]
    out['psf'] = [w['psf'][b] for b in blobs]
    out['sources'] = w['sources'][src]
    out['truth'] = w['truth'][src]
    out['start'] = w['start'][src]
    out['noise'] = w['noise'][blobs]
    return out


def render_blobs(w, params, seed=None):
    """Device images of the blobs' model at `params` through the scene
    renderer (an independent path), plus Gaussian noise of each unit's sigma
    when `seed` is given.  Returns (data, inverr) float32 device tensors."""
    n_bands = w['n_bands']
    sides = w['sides']
    nb = len(sides)
    imgs = []
    for b in range(nb):
        for k in range(n_bands):
            amp, mean, var = w['psf'][b][k]
            imgs.append(batch.SceneImage(sides[b, 0], sides[b, 1], amp, mean, var))
    r = batch.SceneRenderer(imgs, comp_stride=64)
    src = w['sources']
    blob_of = np.repeat(np.arange(nb), np.diff(w['blob_src']))
    n = len(src)
    recs = np.zeros(n * n_bands, _lib.SCENE_SRC)
    for k in range(n_bands):
        rk = recs[k::n_bands]
        rk['px'], rk['py'] = params[:, 0], params[:, 1]
        rk['counts'] = params[:, 2 + k]
        rk['sa0'], rk['sa1'], rk['sa2'] = params[:, 5], params[:, 6], params[:, 7]
        rk['sersic_n'] = params[:, 8]
        rk['profile'] = src['profile']
        rk['shape_type'] = _lib.SHAPE_ELLIPSE_ESOFT
        rk['image'] = blob_of * n_bands + k
        rk['mx0'], rk['my0'], rk['mw'], rk['mh'] = src['x0'], src['y0'], src['w'], src['h']
        recs[k::n_bands] = rk
    dev = render.device()
    out = torch.zeros(r.npix, dtype=torch.float32, device=dev)
    d = torch.from_numpy(recs.view(np.uint8).copy()).to(dev)
    st = r.render_device(d, len(recs), out, r.max_pairs(recs, 32), 32)
    render.check_status(st.clone(), 'tb_scene_render')
    sig = np.repeat(np.asarray(w['noise'], np.float64).reshape(-1), 1)
    npx = np.diff(pix_offsets(sides, n_bands))
    sig_px = torch.from_numpy(np.repeat(sig, npx).astype(np.float32)).to(dev)
    if seed is not None:
        gen = torch.Generator(device=dev)
        gen.manual_seed(int(seed))
        out += sig_px * torch.randn(out.shape, generator=gen, device=dev, dtype=torch.float32)
    return out, 1. / sig_px


def _esoft_params(ell, maxe=0.999999):
    """(log r_e, ee1, ee2) of the EllipseESoft equal to EllipseE `ell`
    (EllipseESoft.fromEllipseE, a round ellipse included)."""
    e = min(ell.e, maxe)
    if e == 0.:
        return np.log(ell.re), 0., 0.
    soft = -np.log(1. - e)
    return np.log(ell.re), ell.e1 / e * soft, ell.e2 / e * soft


def fit_tractors(tractors, tol=1e-3, max_iter=60, check_every=4):
    """Fits many independent blobs, each given as a reference-style Tractor,
    in one batched device fit, and writes the fitted parameters back.

    Each Tractor holds 1 to 3 images of one size with NullWCS, a
    LinearPhotoCal with a band (or no band for a single image) and a
    mixture-of-Gaussians PSF of at most 4 components, and at most 32
    sources: SersicGalaxy, ExpGalaxy or DevGalaxy with an EllipseESoft or
    EllipseE shape, or PointSource, at a PixPos, with a brightness holding
    one value per image band (Flux for a single image, NanoMaggies / Fluxes
    otherwise).  An EllipseE shape is fitted as the EllipseESoft of the same
    ellipse (the same models, so the same optimum) and written back as an
    EllipseE; its three parameters are then fitted or frozen together.  Model masks set with Tractor.setModelMasks are used (the
    same rectangle in every image); without them a source's mask is the
    whole image.  Frozen parameters (freezeParam / freezeAllBut) keep their
    values; every thawed one is fitted.  Returns the per-blob FIT_STATE
    records."""
    from . import sources as S, ellipses as E
    from .basics import NullWCS, LinearPhotoCal
    from .patch import ModelMask
    if not tractors:
        raise ValueError('no blobs')
    n_bands = max(len(tr.getImages()) for tr in tractors)
    blob_src, sides, psf, recs, params, datas, inverrs, layout = [0], [], [], [], [], [], [], []
    cd_inv = None
    for tr in tractors:
        imgs = list(tr.getImages())
        if not 1 <= len(imgs) <= _lib.FIT_MAX_BANDS:
            raise ValueError('a blob needs 1 to %d images' % _lib.FIT_MAX_BANDS)
        H, W = imgs[0].shape
        for img in imgs:
            if img.shape != (H, W) or not isinstance(img.getWcs(), NullWCS):
                raise ValueError('blob images must share one shape and a NullWCS')
            if not isinstance(img.getPhotoCal(), LinearPhotoCal):
                raise ValueError('blob images need a LinearPhotoCal')
            if len(imgs) > 1 and img.getPhotoCal().band is None:
                raise ValueError('several images of a blob need LinearPhotoCal bands')
            if not hasattr(img.getPsf(), 'getMixtureOfGaussians'):
                raise ValueError('blob images need a mixture-of-Gaussians PSF')
            cdi = np.asarray(img.getWcs().cdInverseAtPixel(0, 0), np.float64)
            if cd_inv is None:
                cd_inv = cdi
            elif not np.array_equal(cdi, cd_inv):
                raise ValueError('all blobs need the same pixel scale')
        row = []
        for b in range(n_bands):
            img = imgs[min(b, len(imgs) - 1)]
            mog = img.getPsf().getMixtureOfGaussians()
            row.append((np.asarray(mog.amp, np.float64), np.asarray(mog.mean, np.float64),
                        np.asarray(mog.var, np.float64)))
        psf.append(row)
        sides.append((W, H))
        for b in range(n_bands):
            img = imgs[min(b, len(imgs) - 1)]
            datas.append(np.asarray(img.getImage(), np.float32).ravel())
            # a missing band: zero weight
            ie = img.getInvError() if b < len(imgs) else np.zeros((H, W))
            inverrs.append(np.asarray(ie, np.float32).ravel())
        srcs = list(tr.catalog)
        if not 1 <= len(srcs) <= _lib.FIT_MAX_SRC:
            raise ValueError('a blob needs 1 to %d sources' % _lib.FIT_MAX_SRC)
        for src in srcs:
            r = np.zeros(1, _lib.FIT_SOURCE)[0]
            th = np.zeros(NPAR)
            if isinstance(src, S.PointSource):
                r['profile'] = _lib.PROFILE_POINT
            elif isinstance(src, (S.SersicGalaxy, S.ExpGalaxy, S.DevGalaxy)):
                if isinstance(src.shape, E.EllipseESoft):
                    th[5:8] = src.shape.getAllParams()
                elif isinstance(src.shape, E.EllipseE):
                    th[5:8] = _esoft_params(src.shape)
                else:
                    raise ValueError('galaxies need an EllipseESoft or EllipseE shape')
                if isinstance(src, S.SersicGalaxy):
                    r['profile'] = _lib.PROFILE_SERSIC
                    th[8] = src.sersicindex.val
                else:
                    r['profile'] = (_lib.PROFILE_EXP if isinstance(src, S.ExpGalaxy)
                                    else _lib.PROFILE_DEV)
            else:
                raise ValueError('unsupported source %s' % type(src).__name__)
            px, py = imgs[0].getWcs().positionToPixel(src.getPosition(), src)
            th[0], th[1] = px, py
            for b, img in enumerate(imgs):
                th[2 + b] = img.getPhotoCal().brightnessToCounts(src.getBrightness())
            # parameter slots held fixed: those whose name is not thawed
            thawed = set(src.getParamNames())
            ball = src.getBrightness().copy()
            if hasattr(ball, 'thawAllParams'):
                ball.thawAllParams()
            bnames = ball.getParamNames()      # every brightness value's name
            bslots = [('brightness.' + (img.getPhotoCal().band
                                        if img.getPhotoCal().band in bnames else bnames[0]))
                      for img in imgs]
            shape_names = ['shape.logre', 'shape.ee1', 'shape.ee2']
            if not isinstance(src, S.PointSource) and not isinstance(src.shape, E.EllipseESoft):
                # an EllipseE is fitted through its EllipseESoft: all or none
                ethawed = [n in thawed for n in ('shape.re', 'shape.e1', 'shape.e2')]
                if any(ethawed) and not all(ethawed):
                    raise ValueError('an EllipseE shape is fitted whole or frozen whole')
                if all(ethawed):
                    thawed = thawed | set(shape_names)
            names = ['pos.x', 'pos.y'] + bslots + [None] * (3 - len(imgs)) + \
                shape_names + ['sersicindex.SersicIndex']
            r['frozen'] = sum(1 << k for k, nm in enumerate(names)
                              if nm is not None and nm not in thawed)
            mask = tr._getModelMaskFor(imgs[0], src)
            if mask is None:
                r['x0'], r['y0'], r['w'], r['h'] = 0, 0, W, H
            else:
                if not isinstance(mask, ModelMask) or mask.mask is not None:
                    raise ValueError('model masks must be rectangles')
                r['x0'], r['y0'], r['w'], r['h'] = mask.x0, mask.y0, mask.w, mask.h
            recs.append(r)
            params.append(th)
        blob_src.append(blob_src[-1] + len(srcs))
        layout.append((tr, imgs, srcs))
    import torch
    dev = render.device()
    data = torch.from_numpy(np.concatenate(datas)).to(dev)
    inv = torch.from_numpy(np.concatenate(inverrs)).to(dev)
    f = BlobFitter(blob_src, sides, psf, np.array(recs, _lib.FIT_SOURCE), np.array(params),
                   data, inv, n_bands=n_bands, cd_inv=cd_inv)
    f.fit(tol=tol, max_iter=max_iter, check_every=check_every)
    out = f.result()
    k = 0
    for tr, imgs, srcs in layout:
        for src in srcs:
            th = out[k]
            fz = int(recs[k]['frozen'])
            k += 1
            thawed = lambda slot: not (fz >> slot) & 1   # noqa: E731
            wcs = imgs[0].getWcs()
            pos = src.getPosition()
            xy = pos.getAllParams()
            pos.setAllParams([th[0] - wcs.dx if thawed(0) else xy[0],
                              th[1] - wcs.dy if thawed(1) else xy[1]])
            br = src.getBrightness()
            for b, img in enumerate(imgs):
                if not thawed(2 + b):
                    continue
                pc = img.getPhotoCal()
                val = th[2 + b] / pc.getScale()
                if pc.band is None:
                    br.setAllParams([val])
                else:
                    br.setFlux(pc.band, val)
            if not isinstance(src, S.PointSource):
                if isinstance(src.shape, E.EllipseESoft):
                    sh = src.shape.getAllParams()
                    src.shape.setAllParams([th[5 + j] if thawed(5 + j) else sh[j]
                                            for j in range(3)])
                elif thawed(5):
                    src.shape.setAllParams(
                        E.EllipseESoft(*th[5:8]).toEllipseE().getAllParams())
                if isinstance(src, S.SersicGalaxy) and thawed(8):
                    src.sersicindex.setAllParams([th[8]])
    return f.states()
