"""EM fits of 2-D Gaussian mixtures to images on the GPU (tractor/emfit.i and
tractor/fitpsf.py).

`em_fit_2d_reg` keeps the reference's in-place signature
(tractor/emfit.i:274-557); `em_fit_2d_batch` fits many images of one size in
one launch of `tb_em_fit_2d` (one CTA per image, every iteration inside the
kernel, FP64).  There is no CPU path: without the library or a CUDA device
these raise.
"""
import numpy as np
import torch

from . import _lib, render


def em_init_params(K, w, mu, sig):
    """Initial mixture for the EM fit (tractor/fitpsf.py:72-86): equal
    weights, zero means, variances (k + 1) I."""
    if w is None:
        w = np.ones(K) / float(K)
    assert w.shape == (K,)
    w /= np.sum(w)
    if mu is None:
        mu = np.zeros((K, 2))
    assert mu.shape == (K, 2)
    if sig is None:
        sig = np.array([np.eye(2) * (i + 1) for i in range(K)])
    assert sig.shape == (K, 2, 2)
    return w, mu, sig


def em_fit_2d_batch(imgs, amp, mean, var, alpha=0., steps=1000, xy0=None):
    """EM fits of K-component mixtures to n images (n, ny, nx), starting from
    amp (n, K), mean (n, K, 2), var (n, K, 2, 2).  Pixel (ix, iy) of image s
    sits at xy0[s] + (ix, iy) (default (-(nx // 2), -(ny // 2))).  Returns
    (amp, mean, var, status) as float64 numpy arrays, status[s] = 0, or 1
    where a covariance determinant became non-positive (that fit stopped
    there, as the reference returns -1)."""
    imgs = np.ascontiguousarray(imgs, np.float64)
    if imgs.ndim != 3:
        raise ValueError('imgs must be (n, ny, nx)')
    n, ny, nx = imgs.shape
    amp = np.array(amp, np.float64).reshape(n, -1)
    K = amp.shape[1]
    if not 1 <= K <= _lib.EM_MAX_K:
        raise ValueError('1 <= K <= %d components' % _lib.EM_MAX_K)
    mean = np.array(mean, np.float64).reshape(n, K, 2)
    var = np.array(var, np.float64).reshape(n, K, 2, 2)
    if n == 0:
        return amp, mean, var, np.zeros(0, np.int32)
    xy = None
    if xy0 is not None:
        xy = np.ascontiguousarray(np.broadcast_to(np.asarray(xy0, np.int32), (n, 2)))
    return _run(imgs, amp, mean, var, float(alpha), int(steps), xy)


def _run(imgs, amp, mean, var, alpha, steps, xy):
    """One tb_em_fit_2d launch over the stacked images."""
    n, ny, nx = imgs.shape
    K = amp.shape[1]
    dev = render.device()
    d_img = torch.from_numpy(imgs).to(dev)
    d_amp = torch.from_numpy(amp.copy()).to(dev)
    d_mean = torch.from_numpy(mean.copy()).to(dev)
    d_var = torch.from_numpy(var.copy()).to(dev)
    d_st = torch.zeros(n, dtype=torch.int32, device=dev)
    d_xy = torch.from_numpy(xy.copy()).to(dev) if xy is not None else None
    lib = _lib.load()
    _lib.check(lib.tb_em_fit_2d(d_img.data_ptr(), n, ny, nx,
                                d_xy.data_ptr() if d_xy is not None else None,
                                d_amp.data_ptr(), d_mean.data_ptr(), d_var.data_ptr(), K,
                                alpha, steps, d_st.data_ptr(), _lib.stream_ptr()),
               'tb_em_fit_2d')
    return (d_amp.cpu().numpy(), d_mean.cpu().numpy(), d_var.cpu().numpy(),
            d_st.cpu().numpy())


def em_fit_2d_reg(img, x0, y0, amp, mean, var, alpha, steps):
    """em_fit_2d_reg (tractor/emfit.i:274-557): fits the mixture (amp, mean,
    var), updated in place, to img, pixel (ix, iy) at (x0 + ix, y0 + iy);
    returns 0, or -1 when a covariance determinant became non-positive."""
    img = np.asarray(img)
    a, m, v, st = em_fit_2d_batch(img[None], np.asarray(amp)[None], np.asarray(mean)[None],
                                  np.asarray(var)[None], alpha, steps, xy0=(x0, y0))
    amp[...] = a[0]
    mean[...] = m[0]
    var[...] = v[0]
    return -1 if st[0] else 0


def em_fit_2d_reg2_batch(imgs, amp, mean, var, alpha=0., steps=1000, approx=1e-30, xy0=None):
    """The EM fits with a flat sky term (em_fit_2d_reg2, tractor/emfit2.c) of
    n images in one tb_em_fit_2d_sky launch, in em_fit_2d_batch's layout.
    Returns (amp, mean, var, skyamp, status)."""
    imgs = np.ascontiguousarray(imgs, np.float64)
    if imgs.ndim != 3:
        raise ValueError('imgs must be (n, ny, nx)')
    n, ny, nx = imgs.shape
    amp = np.array(amp, np.float64).reshape(n, -1)
    K = amp.shape[1]
    if not 1 <= K <= _lib.EM_MAX_K:
        raise ValueError('1 <= K <= %d components' % _lib.EM_MAX_K)
    mean = np.array(mean, np.float64).reshape(n, K, 2)
    var = np.array(var, np.float64).reshape(n, K, 2, 2)
    if n == 0:
        return amp, mean, var, np.zeros(0), np.zeros(0, np.int32)
    dev = render.device()
    d_img = torch.from_numpy(imgs).to(dev)
    d_amp = torch.from_numpy(amp.copy()).to(dev)
    d_mean = torch.from_numpy(mean.copy()).to(dev)
    d_var = torch.from_numpy(var.copy()).to(dev)
    d_sky = torch.zeros(n, dtype=torch.float64, device=dev)
    d_st = torch.zeros(n, dtype=torch.int32, device=dev)
    d_xy = None
    if xy0 is not None:
        d_xy = torch.from_numpy(np.array(np.broadcast_to(np.asarray(xy0, np.int32), (n, 2)))
                                ).to(dev)
    lib = _lib.load()
    _lib.check(lib.tb_em_fit_2d_sky(d_img.data_ptr(), n, ny, nx,
                                    d_xy.data_ptr() if d_xy is not None else None,
                                    d_amp.data_ptr(), d_mean.data_ptr(), d_var.data_ptr(), K,
                                    float(alpha), int(steps), float(approx), d_sky.data_ptr(),
                                    d_st.data_ptr(), _lib.stream_ptr()),
               'tb_em_fit_2d_sky')
    return (d_amp.cpu().numpy(), d_mean.cpu().numpy(), d_var.cpu().numpy(),
            d_sky.cpu().numpy(), d_st.cpu().numpy())


def em_fit_2d_reg2(img, x0, y0, amp, mean, var, alpha, steps, approx):
    """em_fit_2d_reg2 (tractor/emfit2.c): fits the mixture (amp, mean, var),
    updated in place, and a flat sky to img, pixel (ix, iy) at (x0 + ix,
    y0 + iy); returns [status, skyamp] as the reference's wrapper does
    (status 0, or -1 when a covariance determinant became non-positive)."""
    img = np.asarray(img)
    a, m, v, sky, st = em_fit_2d_reg2_batch(img[None], np.asarray(amp)[None],
                                            np.asarray(mean)[None], np.asarray(var)[None],
                                            alpha, steps, approx, xy0=(x0, y0))
    amp[...] = a[0]
    mean[...] = m[0]
    var[...] = v[0]
    return [-1 if st[0] else 0, float(sky[0])]


def em_fit_2d(img, x0, y0, amp, mean, var):
    """em_fit_2d (tractor/emfit.i:570-576): no prior, 1000 iterations."""
    return em_fit_2d_reg(img, x0, y0, amp, mean, var, 0.0, 1000)
