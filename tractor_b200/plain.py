"""The plain FP64 GPU path the batched FP32 kernels are measured against.

One source (or one blob) at a time, every array FP64 on the device, library
operations only (torch elementwise ops, cuFFT through torch.fft, cuSOLVER
Cholesky) -- the way a straightforward port of the reference's GPU optimizer
(tractor/gpu_optimizer.py:184-1102, CuPy) would run on this machine.  It is a
measurement baseline for bench.py, not a product path: the product renders
and fits through the hand-written kernels of libtractor_b200.so.

  fourier_render_fp64   one galaxy through the pixelized-PSF Fourier path
                        (galaxy.py:336-519): mixture spectrum, times the PSF
                        spectrum, irfft2, Lanczos-3 shift, crop;
  BlobFitFP64           one blob: model and analytic Jacobian on the device,
                        Levenberg-Marquardt with the batched fitter's rules
                        (Marquardt scaling, FP64 Cholesky, maximum steps,
                        projected Sersic bounds, predicted-gain stopping).
"""
import math

import numpy as np
import torch

from . import profiles

_LOG2 = math.log(2.)


def _ellipse_esoft_factor(logre, ee1, ee2):
    """T T^T of an EllipseESoft under NullWCS (pixel scale 1)."""
    re = math.exp(logre)
    ee = math.hypot(ee1, ee2)
    e = min(0.999999, 1. - math.exp(-ee))
    th2 = math.atan2(ee2, ee1)
    e1, e2 = e * math.cos(th2), e * math.sin(th2)
    th = math.atan2(e2, e1) / 2.
    ct, st = math.cos(th), math.sin(th)
    ab = 1000. if e >= 1 else min(1000., (1. + e) / (1. - e))
    r = re / 3600.
    G = np.array([[r * ct / ab, r * st], [-r * st / ab, r * ct]])
    T = np.eye(2) * 3600. @ G
    return T @ T.T


def _sersic(n):
    return profiles.sersic_mixture().profile(float(min(max(n, 0.29), 6.3)))


# ---------------------------------------------------------------------------
# Fourier path, one galaxy
# ---------------------------------------------------------------------------

def _lanczos_taps(dx):
    if dx == 0.:
        t = np.zeros(7)
        t[3] = 1.
        return t
    i = np.arange(7)
    lo, hi = (0, 6) if dx > 0 else (1, 7)
    t = np.zeros(7)
    p = np.pi * (i[lo:hi] - 3. + dx)
    t[lo:hi] = 3. * np.sin(p) * np.sin(p / 3.) / (p * p)
    return t / t.sum()


def fourier_render_fp64(amp, var2, psf_spec, cx, cy, sz, px, py, mx0, my0, mw, mh, counts=1.):
    """(mh, mw) FP64 device patch of one galaxy: amp (K,), var2 (K, 2, 2)
    pixel covariances, psf_spec the FP64 rfft2 of the padded PSF (sz, sz/2+1)
    on the device, (cx, cy) its centre in the padded image."""
    dev = psf_spec.device
    v = torch.fft.rfftfreq(sz, device=dev, dtype=torch.float64)
    w = torch.fft.fftfreq(sz, device=dev, dtype=torch.float64)
    W2, V2 = torch.meshgrid(w, v, indexing='ij')
    a = torch.as_tensor(amp, dtype=torch.float64, device=dev)
    C = torch.as_tensor(np.asarray(var2).reshape(-1, 4), dtype=torch.float64, device=dev)
    e = (C[:, 0, None, None] * V2 * V2 + 2 * C[:, 1, None, None] * V2 * W2 +
         C[:, 3, None, None] * W2 * W2)
    F = (a[:, None, None] * torch.exp(-2. * np.pi ** 2 * e)).sum(0)
    G = torch.fft.irfft2(F * psf_spec, s=(sz, sz))
    mux, muy = px - cx - mx0, py - cy - my0
    sx, sy = int(np.round(mux)), int(np.round(muy))
    mux -= sx
    muy -= sy
    if mux != 0. or muy != 0.:
        fx = torch.as_tensor(_lanczos_taps(mux), device=dev)
        fy = torch.as_tensor(_lanczos_taps(muy), device=dev)
        G = torch.nn.functional.conv1d(G[:, None, :], fx[None, None, :], padding=3)[:, 0]
        G = torch.nn.functional.conv1d(G.T[:, None, :], fy[None, None, :], padding=3)[:, 0].T
    out = torch.zeros((mh, mw), dtype=torch.float64, device=dev)
    y0, y1 = max(0, -sy), min(sz, mh - sy)
    x0, x1 = max(0, -sx), min(sz, mw - sx)
    if y1 > y0 and x1 > x0:
        out[y0 + sy:y1 + sy, x0 + sx:x1 + sx] = G[y0:y1, x0:x1]
    return out * counts


def psf_spectrum_fp64(psf_img, sz, device):
    """FP64 rfft2 of the PSF padded to sz x sz (PixelizedPSF._padInImage)
    and its centre."""
    ph, pw = psf_img.shape
    pad = np.zeros((sz, sz))
    y0, x0 = (sz - ph) // 2, (sz - pw) // 2
    pad[y0:y0 + ph, x0:x0 + pw] = psf_img
    spec = torch.fft.rfft2(torch.as_tensor(pad, device=device))
    return spec, x0 + pw // 2, y0 + ph // 2


# ---------------------------------------------------------------------------
# Blob fitting, one blob
# ---------------------------------------------------------------------------

MAXSTEP = np.array([1., 1., 0., 0., 0., 1., 0.1, 0.1, 0.1])


class BlobFitFP64(object):
    """Levenberg-Marquardt fit of one blob in FP64 on the device.  data,
    inverr: (n_bands, H, W) arrays; psf: per band (amp, mean, var); rects:
    per source (x0, y0, w, h)."""

    def __init__(self, data, inverr, psf, rects, device):
        self.dev = device
        self.data = torch.as_tensor(np.asarray(data, np.float64), device=device)
        self.w = torch.as_tensor(np.asarray(inverr, np.float64), device=device)
        self.nb, self.H, self.W = self.data.shape
        self.psf = psf
        self.rects = rects
        ys, xs = torch.meshgrid(torch.arange(self.H, dtype=torch.float64, device=device),
                                torch.arange(self.W, dtype=torch.float64, device=device),
                                indexing='ij')
        self.xs, self.ys = xs, ys

    def _source_tables(self, th):
        """Host FP64: galaxy components, d/dn, T T^T and its shape derivatives."""
        n = th[8]
        a, v = _sersic(n)
        h = 1e-5
        ap, vp = _sersic(n + h)
        am, vm = _sersic(n - h)
        if len(ap) != len(a) or len(am) != len(a):
            da, dv = np.zeros_like(a), np.zeros_like(v)
        else:
            da, dv = (ap - am) / (2 * h), (vp - vm) / (2 * h)
        M = _ellipse_esoft_factor(*th[5:8])
        dM = []
        for j in range(3):
            p, m = list(th[5:8]), list(th[5:8])
            p[j] += 1e-6
            m[j] -= 1e-6
            dM.append((_ellipse_esoft_factor(*p) - _ellipse_esoft_factor(*m)) / 2e-6)
        return a, v, da, dv, M, dM

    def model_jacobian(self, theta):
        """(model (nb, H, W), columns (P, nb, H, W)) at theta (n, 9)."""
        n = len(theta)
        P = 9 * n
        model = torch.zeros((self.nb, self.H, self.W), dtype=torch.float64, device=self.dev)
        J = torch.zeros((P, self.nb, self.H, self.W), dtype=torch.float64, device=self.dev)
        for s in range(n):
            th = theta[s]
            a, v, da, dv, M, dM = self._source_tables(th)
            x0, y0, w, h = self.rects[s]
            X0, Y0 = max(x0, 0), max(y0, 0)
            X1, Y1 = min(x0 + w, self.W), min(y0 + h, self.H)
            if X1 <= X0 or Y1 <= Y0:
                continue
            xs = self.xs[Y0:Y1, X0:X1]
            ys = self.ys[Y0:Y1, X0:X1]
            for b in range(self.nb):
                pamp, pmean, pvar = self.psf[b]
                K = len(a) * len(pamp)
                C = np.zeros((K, 2, 2))
                amp = np.zeros(K)
                damp = np.zeros(K)
                mu = np.zeros((K, 2))
                dC = np.zeros((4, K, 2, 2))
                for p in range(len(pamp)):
                    for i in range(len(a)):
                        k = p * len(a) + i
                        C[k] = v[i] * M + pvar[p]
                        amp[k] = a[i] * pamp[p]
                        damp[k] = da[i] * pamp[p]
                        mu[k] = [th[0] + pmean[p][0], th[1] + pmean[p][1]]
                        for j in range(3):
                            dC[j, k] = v[i] * dM[j]
                        dC[3, k] = dv[i] * M
                T = lambda z: torch.as_tensor(z, dtype=torch.float64, device=self.dev)
                Ci = T(np.linalg.inv(C))
                det = T(np.linalg.det(C))
                dx = xs[None] - T(mu[:, 0])[:, None, None]
                dy = ys[None] - T(mu[:, 1])[:, None, None]
                ux = Ci[:, 0, 0, None, None] * dx + Ci[:, 0, 1, None, None] * dy
                uy = Ci[:, 1, 0, None, None] * dx + Ci[:, 1, 1, None, None] * dy
                q = dx * ux + dy * uy
                E = torch.where(-0.5 * q >= -50., torch.exp(-0.5 * q), torch.zeros_like(q))
                E = E / (2 * np.pi * torch.sqrt(det))[:, None, None]
                val = T(amp)[:, None, None] * E
                c = th[2 + b]
                model[b, Y0:Y1, X0:X1] += c * val.sum(0)
                base = 9 * s
                J[base + 0, b, Y0:Y1, X0:X1] += c * (val * ux).sum(0)
                J[base + 1, b, Y0:Y1, X0:X1] += c * (val * uy).sum(0)
                J[base + 2 + b, b, Y0:Y1, X0:X1] += val.sum(0)
                for j in range(4):
                    D = T(dC[j])
                    tr = (Ci * D).sum((1, 2))
                    quad = (D[:, 0, 0, None, None] * ux * ux + 2 * D[:, 0, 1, None, None] * ux * uy +
                            D[:, 1, 1, None, None] * uy * uy)
                    g = 0.5 * (quad - tr[:, None, None]) * val
                    if j == 3:
                        g = g + T(damp)[:, None, None] * E
                    J[base + 5 + j, b, Y0:Y1, X0:X1] += c * g.sum(0)
        return model, J

    def fisher(self, theta):
        """A^T A (FP64, host) at theta: the inverse gives the parameter
        covariance used to state errors in sigma."""
        _, J = self.model_jacobian(np.asarray(theta, np.float64))
        A = (J * self.w[None]).reshape(J.shape[0], -1)
        return (A @ A.T).cpu().numpy()

    def fit(self, theta0, tol=1e-3, max_iter=60, lam=1e-3):
        theta = np.array(theta0, np.float64)
        n = len(theta)

        def normal_eq(th):
            model, J = self.model_jacobian(th)
            r = ((self.data - model) * self.w).reshape(-1)
            A = (J * self.w[None]).reshape(J.shape[0], -1)
            return A @ A.T, A @ r, float(r @ r)

        H, g, c2 = normal_eq(theta)
        it = 0
        for it in range(1, max_iter + 1):
            d = torch.sqrt(torch.clamp(torch.diagonal(H), min=0.))
            nidx = np.arange(n) * 9 + 8
            gh = g.cpu().numpy()
            held = ((theta[:, 8] >= 6.3) & (gh[nidx] > 0)) | ((theta[:, 8] <= 0.29) & (gh[nidx] < 0))
            live = (d > 0).cpu().numpy()
            live[nidx[held]] = False
            L = torch.as_tensor(live, device=self.dev)
            dl = d[L]
            Hs = H[L][:, L] / torch.outer(dl, dl) + lam * torch.eye(int(L.sum()), dtype=torch.float64,
                                                                      device=self.dev)
            y0 = g[L] / dl
            xs = torch.cholesky_solve(y0[:, None], torch.linalg.cholesky(Hs))[:, 0]
            pred = 0.5 * float(xs @ y0 + lam * xs @ xs)
            if pred < tol and lam <= 1.:
                break
            step = np.zeros(9 * n)
            step[live] = (xs / dl).cpu().numpy()
            step = step.reshape(n, 9)
            ms = np.tile(MAXSTEP, (n, 1))
            lim = 1.
            big = (ms > 0) & (np.abs(step) > ms)
            if big.any():
                lim = min(lim, float((ms[big] / np.abs(step[big])).min()))
            nn = theta[:, 8] + lim * step[:, 8]
            for s in range(n):
                if nn[s] > 6.3 and step[s, 8] > 0:
                    lim = min(lim, (6.3 - theta[s, 8]) / step[s, 8])
                if nn[s] < 0.29 and step[s, 8] < 0:
                    lim = min(lim, (0.29 - theta[s, 8]) / step[s, 8])
            sc = max(lim, 0.)
            trial = theta + sc * step
            trial[:, 8] = np.clip(trial[:, 8], 0.29, 6.3)
            H2, g2, c22 = normal_eq(trial)
            if c22 < c2:
                # damping from the gain ratio (Nielsen's rule), the prediction
                # for the step as scaled
                a, b = float(xs @ y0), float(xs @ xs)
                pred_s = sc * a - 0.5 * sc * sc * (a - lam * b)
                t = 2. * (0.5 * (c2 - c22) / pred_s) - 1. if pred_s > 0 else -1.
                theta, H, g, c2 = trial, H2, g2, c22
                lam = max(lam * max(1. / 3., 1. - t ** 3), 1e-9)
            else:
                lam *= 10.
                if lam > 1e12:
                    break
        return theta, it


def sersic_edges():
    """Sersic indices where the mixture tables change: the inner edges of
    the index ranges (each range is a separate fit, with its own component
    count) and n = 1, above which the core component is added.  The model
    is not smooth across them."""
    R = profiles.tables()['sersic']['ranges']
    return np.array(sorted({r['lo'] for r in R[1:]} | {1.0}))


def optimum_distance(w, data, inv, fitted, status, blobs, device, tol=1e-10, max_iter=100,
                     edge=1e-3):
    """Distance of batched-fit results from the FP64 optimum, per blob of
    `blobs` (a blob workload of tractor_b200.fit): the FP64 fitter continued
    from the batched result to a predicted gain of `tol`, then
    max_i |fitted_i - opt_i| / sigma_i with sigma from its FP64 Fisher
    matrix (a Sersic index held at a bound, and directions the Fisher
    matrix leaves unconstrained, count as sigma = inf).  Returns one record
    per blob: (sigma, blob, status, on_edge, converged), on_edge when a
    Sersic index (batched or FP64) lies within `edge` of sersic_edges(),
    converged when the FP64 fitter reached `tol` within `max_iter`."""
    from . import fit as _fit
    po = _fit.pix_offsets(w['sides'], 3)
    hd, hi = data.cpu().numpy(), inv.cpu().numpy()
    edges = sersic_edges()
    out = []
    for b in blobs:
        s0, s1 = int(w['blob_src'][b]), int(w['blob_src'][b + 1])
        W, H = (int(v) for v in w['sides'][b])
        d3 = np.stack([hd[po[3 * b + k]:po[3 * b + k + 1]].reshape(H, W) for k in range(3)])
        i3 = np.stack([hi[po[3 * b + k]:po[3 * b + k + 1]].reshape(H, W) for k in range(3)])
        rects = [tuple(int(v) for v in (r['x0'], r['y0'], r['w'], r['h']))
                 for r in w['sources'][s0:s1]]
        pf = BlobFitFP64(d3, i3, w['psf'][b], rects, device)
        opt, nit = pf.fit(fitted[s0:s1], tol=tol, max_iter=max_iter)
        Hf = pf.fisher(opt)
        o = opt.ravel()
        n_idx = np.arange(8, o.size, 9)
        held = np.zeros(o.size, bool)
        held[n_idx] = (o[n_idx] >= _fit.SERSIC_MAX) | (o[n_idx] <= _fit.SERSIC_MIN)
        free = ~held & (np.diag(Hf) > 0)
        sig = np.full(o.size, np.inf)
        with np.errstate(invalid='ignore'):
            sig[free] = np.sqrt(np.diag(np.linalg.inv(Hf[np.ix_(free, free)])))
        sig[~(np.isfinite(sig) & (sig > 0))] = np.inf
        err = float(np.max(np.abs(np.asarray(fitted[s0:s1]).ravel() - o) / sig))
        nn = np.concatenate([np.asarray(fitted[s0:s1])[:, 8], opt[:, 8]])
        on_edge = bool(np.min(np.abs(nn[:, None] - edges[None])) < edge)
        out.append((err, int(b), int(status[b]), on_edge, nit < max_iter))
    return out
