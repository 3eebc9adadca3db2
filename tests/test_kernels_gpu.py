"""Kernel-level parity of the CUDA path (through the C ABI) against the oracle.

Tolerances: model pixels within 1e-5 of the peak (the parity bar for
rendering); Lanczos bit-exact with the reference's float arithmetic; FFT-based
spectra within 2e-6 relative to the largest element; least-squares solutions
within 1e-9 relative of numpy's FP64 lstsq on well-conditioned problems.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PEAK_TOL = 1e-5


def _rand_mix(rng, K, spread=3.0, vmin=0.2, vmax=6.0):
    amp = rng.uniform(0.1, 1.0, K)
    mean = rng.normal(scale=spread, size=(K, 2))
    var = np.zeros((K, 2, 2))
    for k in range(K):
        a = rng.normal(size=(2, 2))
        var[k] = a @ a.T * rng.uniform(vmin, vmax) / 2 + vmin * np.eye(2)
    return amp, mean, var


def _moffat(size=63, fwhm=4.0, beta=3.0):
    alpha = fwhm / (2 * np.sqrt(2 ** (1 / beta) - 1))
    y, x = np.mgrid[:size, :size] - size // 2
    img = (1 + (x ** 2 + y ** 2) / alpha ** 2) ** (-beta)
    return (img / img.sum()).astype(np.float32)


def test_mog_grid_matches_oracle(tb, oracle):
    import torch
    from tractor_b200 import render
    rng = np.random.default_rng(1)
    b = render.MogBatch()
    cases = []
    for (w, h, K) in [(33, 33, 12), (64, 64, 6), (45, 17, 3), (100, 130, 27), (1, 1, 2), (255, 255, 45)]:
        amp, mean, var = _rand_mix(rng, K, spread=w / 6)
        x0, y0 = int(rng.integers(-50, 50)), int(rng.integers(-50, 50))
        fx, fy = x0 + w / 2 + rng.normal(), y0 + h / 2 + rng.normal()
        off = b.add(x0, y0, w, h, amp, mean, var, fx=fx, fy=fy, scale=1.0)
        cases.append((off, x0, y0, w, h, amp, mean, var, fx, fy))
    out = b.run().cpu().numpy()
    for off, x0, y0, w, h, amp, mean, var, fx, fy in cases:
        ref = oracle.mog_grid(x0, x0 + w, y0, y0 + h, fx, fy, amp, mean, var)
        got = out[off:off + w * h].reshape(h, w)
        err = np.abs(got - ref).max() / ref.max()
        assert err < PEAK_TOL, (w, h, err)


def test_mog_masked_matches_oracle(tb, oracle):
    from tractor_b200 import render
    rng = np.random.default_rng(2)
    amp, mean, var = _rand_mix(rng, 9, spread=5)
    h, w = 40, 50
    mask = rng.uniform(size=(h, w)) > 0.3
    b = render.MogBatch()
    b.add(-3, 4, w, h, amp, mean, var, fx=20.5, fy=22.25, floor=render.FLOOR_MASKED, mask=mask)
    got = b.run().cpu().numpy()[:h * w].reshape(h, w)
    ref, _, _ = oracle.mog_masked(-3, 4, mask, 20.5, 22.25, amp, mean, var)
    assert np.all(got[~mask] == 0)
    assert np.abs(got - ref).max() / ref.max() < PEAK_TOL


def test_mog_atomic_image_matches_sum(tb, oracle):
    import torch
    from tractor_b200 import render
    rng = np.random.default_rng(3)
    H, W = 96, 80
    img = torch.zeros(H * W, dtype=torch.float32, device='cuda')
    ref = np.zeros((H, W))
    b = render.MogBatch()
    for i in range(20):
        amp, mean, var = _rand_mix(rng, 6, spread=1)
        cx, cy = rng.uniform(0, W), rng.uniform(0, H)
        hw = int(rng.integers(5, 30))
        x0, x1 = max(0, int(cx) - hw), min(W, int(cx) + hw + 1)
        y0, y1 = max(0, int(cy) - hw), min(H, int(cy) + hw + 1)
        counts = rng.uniform(10, 1000)
        b.add(x0, y0, x1 - x0, y1 - y0, amp, mean, var, fx=cx, fy=cy, scale=counts,
              out_off=y0 * W + x0, ldo=W, mode=render.MOG_ATOMIC)
        ref[y0:y1, x0:x1] += counts * oracle.mog_grid(x0, x1, y0, y1, cx, cy, amp, mean, var)
    b.run(out=img)
    got = img.cpu().numpy().reshape(H, W)
    assert np.abs(got - ref).max() / ref.max() < PEAK_TOL


def test_mog_host_entry_equals_device_path(tb):
    """tb_mog_render_host (host buffers in and out, staging inside) writes
    exactly what tb_mog_render writes into device memory: grid, masked,
    derivative-plane and difference items in one batch, and ATOMIC items
    into a shared image; items outside the given sizes and a short
    workspace are rejected before any copy."""
    import ctypes
    import torch
    from tractor_b200 import _lib, render
    rng = np.random.default_rng(11)
    b = render.MogBatch()
    for (w, h, K) in [(33, 33, 12), (64, 64, 6), (1, 1, 2), (100, 70, 27)]:
        amp, mean, var = _rand_mix(rng, K, spread=w / 6)
        b.add(int(rng.integers(-20, 20)), int(rng.integers(-20, 20)), w, h, amp, mean, var,
              fx=w / 2, fy=h / 2)
    amp, mean, var = _rand_mix(rng, 9, spread=5)
    b.add(-3, 4, 50, 40, amp, mean, var, fx=20.5, fy=22.25, floor=render.FLOOR_MASKED,
          mask=rng.uniform(size=(40, 50)) > 0.3)
    b.add(0, 0, 31, 29, amp, mean, var, fx=15., fy=14., derivs=True)
    amp2, _, var2 = _rand_mix(rng, 9, spread=5)
    b.add(2, 1, 40, 36, amp, mean, var, fx=20., fy=18., diff=(amp2, var2))
    dev = b.run().cpu().numpy()[:b.nout]
    host = b.run_host()
    assert host.dtype == np.float32 and host.shape == (b.nout,)
    assert np.array_equal(host, dev)
    # ATOMIC items into one image (outputs start at zero)
    H, W = 60, 70
    a = render.MogBatch()
    for i in range(8):
        amp, mean, var = _rand_mix(rng, 4, spread=1)
        x0, y0 = int(rng.integers(0, W - 20)), int(rng.integers(0, H - 20))
        a.add(x0, y0, 20, 20, amp, mean, var, fx=x0 + 10., fy=y0 + 10., scale=100.,
              out_off=y0 * W + x0, ldo=W, mode=render.MOG_ATOMIC)
    a.nout = H * W
    img = torch.zeros(H * W, dtype=torch.float32, device='cuda')
    a.run(out=img)
    got = a.run_host()
    assert np.abs(got - img.cpu().numpy()).max() <= 1e-5 * np.abs(got).max()
    # rejections: an output beyond n_out, a workspace one byte short
    lib = _lib.load()
    items = np.array(b.items[:1], dtype=_lib.MOG_ITEM)
    w0, h0 = int(items['w'][0]), int(items['h'][0])
    tiles = ((w0 + 31) // 32) * ((h0 + 31) // 32)
    K = int(items['K'][0])
    ca, cm, cv = b.amp[0], b.mean[0], b.var[0]
    nbytes = ctypes.c_int64()
    assert lib.tb_mog_render_host_bytes(1, K, 0, w0 * h0, ctypes.byref(nbytes)) == _lib.TB_OK
    pinned = torch.empty(nbytes.value, dtype=torch.uint8).pin_memory()
    ws = torch.empty(nbytes.value, dtype=torch.uint8, device='cuda')
    st = np.zeros(1, _lib.STATUS)

    def call(n_out, ws_bytes):
        out = np.full(max(n_out, 1), -7., np.float32)
        rc = lib.tb_mog_render_host(items.ctypes.data, 1, tiles, ca.ctypes.data, cm.ctypes.data,
                                    cv.ctypes.data, K, None, 0, out.ctypes.data, n_out,
                                    st.ctypes.data, pinned.data_ptr(), ws.data_ptr(), ws_bytes,
                                    _lib.stream_ptr())
        return rc, out
    rc, out = call(w0 * h0, nbytes.value)
    assert rc == _lib.TB_OK and np.array_equal(out, dev[:w0 * h0])
    rc, out = call(w0 * h0 - 1, nbytes.value)
    assert rc == _lib.TB_ERR_ARG and np.all(out == -7.)
    rc, out = call(w0 * h0, nbytes.value - 1)
    assert rc == _lib.TB_ERR_SIZE and np.all(out == -7.)


def test_lanczos_bit_exact(tb, oracle):
    import torch
    from tractor_b200 import render
    rng = np.random.default_rng(4)
    for (h, w) in [(37, 45), (128, 128), (9, 70)]:
        imgs = rng.normal(size=(3, h, w)).astype(np.float32)
        shifts = rng.uniform(-0.5, 0.5, size=(3, 2))
        shifts[1] = [0.0, 0.3]
        got = render.lanczos_shift(torch.from_numpy(imgs).cuda(), shifts).cpu().numpy()
        for i in range(3):
            ref = oracle.lanczos_shift(imgs[i], shifts[i, 0], shifts[i, 1])
            assert np.array_equal(got[i], ref), (h, w, i, np.abs(got[i] - ref).max())


@pytest.mark.parametrize('sz', [32, 64, 128, 256])
def test_psf_spectrum(tb, sz):
    from tractor_b200 import render
    psf = _moffat(min(63, sz - 1) if sz > 32 else 31)
    spec, cx, cy = render.PsfSpectra().get(('moffat', sz), psf, sz)
    got = spec.cpu().numpy().view(np.complex64).reshape(sz // 2 + 1, sz).T
    pad, cx2, cy2 = render.PsfSpectra.pad(psf, sz)
    ref = np.fft.rfft2(pad)
    assert (cx, cy) == (cx2, cy2)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 2e-6


def _fourier_path(N, mw, mh, sx, sy, mux, muy):
    """Which variant tb_fourier_render takes: the Lanczos-3 pass becomes a
    product in frequency space when no tap of a shifted direction reaches
    outside the N x N box (the reference's zero edges then never matter)."""
    gr0, gr1 = max(0, -sy), min(N, mh - sy)
    gc0, gc1 = max(0, -sx), min(N, mw - sx)
    xin = mux == 0 or (gc0 >= 3 and gc1 <= N - 3)
    yin = muy == 0 or (gr0 >= 3 and gr1 <= N - 3)
    return 'spectral' if xin and yin else 'spatial'


@pytest.mark.parametrize('sz,mw,mh', [(256, 128, 128), (128, 64, 64), (64, 40, 33),
                                      (32, 20, 20), (256, 200, 180)])
def test_fourier_render_matches_oracle(tb, oracle, sz, mw, mh):
    from tractor_b200 import render
    rng = np.random.default_rng(5 + sz + mw)
    psf = _moffat(63 if sz >= 128 else (31 if sz == 64 else 15))
    spec, cx, cy = render.psf_spectra().get(('moffat-test', sz), psf, sz)
    b = render.FftBatch()
    cases, paths = [], set()
    for i in range(6):
        amp, var_s = oracle.exp_profile() if i % 2 else oracle.dev_profile()
        T = rng.normal(size=(2, 2)) * rng.uniform(0.5, 4)
        amp2, var2 = oracle.sheared(amp, var_s, T)
        mx0, my0 = int(rng.integers(-20, 20)), int(rng.integers(-20, 20))
        px = mx0 + mw / 2 + rng.uniform(-8, 8)
        py = my0 + mh / 2 + rng.uniform(-8, 8)
        if i == 5:
            px = mx0 - 10.3   # source outside the mask: rows / columns clip
        ref, (mux, muy, sx, sy, rsz) = oracle.galaxy_fft_masked(
            amp2, var2, px, py, psf, mx0, my0, mw, mh, force_halfsize=sz / 2)
        assert rsz == sz
        off = b.add(amp2, var2, sz, ('moffat-test', sz), spec, mw, mh, sx, sy, mux, muy)
        cases.append((off, ref))
        paths.add(_fourier_path(sz, mw, mh, sx, sy, mux, muy))
    # both kernel variants (spectral Lanczos, spatial Lanczos at the box edge)
    assert paths == {'spectral', 'spatial'}, paths
    out = b.run().cpu().numpy()
    for off, ref in cases:
        got = out[off:off + mw * mh].reshape(mh, mw)
        peak = max(np.abs(ref).max(), 1e-30)
        assert np.abs(got - ref).max() / peak < PEAK_TOL, np.abs(got - ref).max() / peak


def test_split_path_matches_persistent_kernel(tb, oracle):
    """tb_fourier_render_split (column and row kernels through the scratch,
    the box-edge items by the persistent kernel) against tb_fourier_render
    (the persistent kernel alone) on the same items, within the rendering
    parity bar (1e-5 of the peak; the two order their FP32 arithmetic
    differently): 300 galaxies of every FFT size (more than one column / row
    launch pair), windows inside and at the edge of the box, and difference
    items."""
    import torch
    from tractor_b200 import render, _lib
    rng = np.random.default_rng(31)
    b = render.FftBatch()
    spec_keys = {}
    for i in range(300):
        sz = [32, 64, 128, 256][i % 4]
        mw = int(rng.integers(8, sz // 2 + 8))
        mh = int(rng.integers(8, sz // 2 + 8))
        psf = _moffat(63 if sz >= 128 else (31 if sz == 64 else 15))
        if sz not in spec_keys:
            spec_keys[sz] = render.psf_spectra().get(('split-test', sz), psf, sz)
        spec, cx, cy = spec_keys[sz]
        amp, var_s = oracle.exp_profile() if i % 3 else oracle.dev_profile()
        T = rng.normal(size=(2, 2)) * rng.uniform(0.3, 2.5)
        amp2, var2 = oracle.sheared(amp, var_s, T)
        sx, sy = int(rng.integers(-6, 4)), int(rng.integers(-6, 4))
        mux, muy = rng.uniform(-0.5, 0.5, 2)
        diff = None
        if i % 17 == 0:
            diff = (amp2 * 1.01, var2 * 1.02)
        b.add(amp2, var2, sz, ('split-test', sz), spec, mw, mh, sx, sy, mux, muy,
              scale=float(rng.uniform(0.5, 2)), diff=diff)
    items = np.array(b.items, dtype=_lib.FFT_ITEM)
    dev = torch.device('cuda')
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    d_items = t(items.view(np.uint8))
    amp, var = t(np.concatenate(b.amp)), t(np.concatenate(b.var))
    dcoef = t(np.concatenate(b.dcoef))
    specs = torch.cat(b.spec_list)
    lib = _lib.load()
    out0 = torch.full((b.nout,), 7.0, dtype=torch.float32, device=dev)
    misc = torch.zeros(8, dtype=torch.int32, device=dev)
    rc = lib.tb_fourier_render_deriv(d_items.data_ptr(), len(items), amp.data_ptr(),
                                     var.data_ptr(), dcoef.data_ptr(), specs.data_ptr(),
                                     out0.data_ptr(), None, misc.data_ptr(), misc.data_ptr() + 16,
                                     None)
    assert rc == 0
    out1 = torch.full((b.nout,), 7.0, dtype=torch.float32, device=dev)
    render.fourier_render(d_items.data_ptr(), len(items), amp.data_ptr(), var.data_ptr(),
                          specs.data_ptr(), out1.data_ptr(), misc.data_ptr() + 16,
                          dcoef_ptr=dcoef.data_ptr(), method='split')
    torch.cuda.synchronize()
    render.check_status(misc[4:8].clone(), 'tb_fourier_render_split')
    a, c = out0.cpu().numpy(), out1.cpu().numpy()
    amps = np.concatenate(b.amp)
    for it in items:
        o, n = int(it['out_off']), int(it['mw'] * it['mh'])
        pa, pc = a[o:o + n], c[o:o + n]
        # the window's peak, or for a window that sees only the far wings a
        # thousandth of the galaxy's total (its rounding floor is set by it)
        tot = abs(float(it['scale'])) * np.abs(amps[it['c0']:it['c0'] + it['K']]).sum()
        peak = max(np.abs(pa).max(), 1e-3 * tot, 1e-30)
        assert np.abs(pa - pc).max() <= PEAK_TOL * peak, (it, np.abs(pa - pc).max() / peak)
    # a second call over the scratch the first left behind gives the same pixels
    out2 = torch.zeros_like(out1)
    render.fourier_render(d_items.data_ptr(), len(items), amp.data_ptr(), var.data_ptr(),
                          specs.data_ptr(), out2.data_ptr(), misc.data_ptr() + 16,
                          dcoef_ptr=dcoef.data_ptr(), method='split')
    assert torch.equal(out1, out2)


@pytest.mark.parametrize('derivs', [False, True])
def test_approx3_region_on_device_matches_oracle(tb, oracle, derivs):
    """approx3 (tb_mog_render with the minval floors, then tb_approx3_region
    walking the rings on the device) against the oracle's c_gauss_2d_approx3
    (pinned to the reference's C): the sliced patch, its extent and, with
    derivs, the d/dx and d/dy planes, for start pixels inside the box and
    beyond each of its edges and corners; all walks in one plan."""
    from tractor_b200 import approx
    from tractor_b200.plan import RenderPlan
    from tractor_b200.profiles import MixtureOfGaussians
    rng = np.random.default_rng(41 + derivs)
    plan = RenderPlan()
    cases = []
    starts = ['in', 'left', 'right', 'below', 'above', 'corner']
    for i in range(18):
        K = int(rng.integers(2, 8))
        amp, mean, var = _rand_mix(rng, K, spread=2.0, vmin=0.5, vmax=9.0)
        W, H = int(rng.integers(20, 90)), int(rng.integers(20, 90))
        x0, y0 = int(rng.integers(-30, 30)), int(rng.integers(-30, 30))
        fx, fy = x0 + W * rng.uniform(0.2, 0.8), y0 + H * rng.uniform(0.2, 0.8)
        minval = float(10 ** rng.uniform(-5, -2))
        where = starts[i % len(starts)]
        xc, yc = int(fx), int(fy)
        if where == 'left':
            xc = x0 - 5
        elif where == 'right':
            xc = x0 + W + 3
        elif where == 'below':
            yc = y0 - 4
        elif where == 'above':
            yc = y0 + H
        elif where == 'corner':
            xc, yc = x0 - 2, y0 + H + 7
        mix = MixtureOfGaussians(amp, mean, var)
        pend = approx.plan_approx3(plan, mix, x0, x0 + W, y0, y0 + H, fx, fy, minval, xc, yc,
                                   derivs=derivs)
        cases.append((pend, (x0, W, y0, H, fx, fy, minval, amp, mean, var, xc, yc)))
    # the same boxes rendered without the walk, for the CPU walk over the
    # device's own values
    raw = [plan.mog.add(a[0], a[2], a[1], a[3], a[7], a[8], a[9], fx=a[4], fy=a[5],
                        minval=a[6]) for _, a in cases]
    flips = 0
    from oracle.host_kernels import ring_region
    for (pend, (x0, W, y0, H, fx, fy, minval, amp, mean, var, xc, yc)), ro in zip(cases, raw):
        got = pend.result()
        planes = got if derivs else (got,)
        vals = plan._mog_host[ro:ro + W * H].reshape(H, W).astype(np.float64)
        # start pixel as approx3.c chooses it, from the oracle's plain edges
        out, dxo, dyo, (sx0, sx1, sy0, sy1) = oracle.mog_approx3(
            x0, x0 + W, y0, y0 + H, fx, fy, minval, amp, mean, var, xc, yc, derivs=derivs)
        # (1) the device walk is exactly the CPU walk over the same values
        inside = x0 <= xc < x0 + W and y0 <= yc < y0 + H
        cx, cy = xc - x0, yc - y0
        if not inside:
            # approx3.c: the brightest pixel of the nearest edge column, then row
            best, cx, cy = 0., int((2 * x0 + W) / 2) - x0, int((2 * y0 + H) / 2) - y0
            def plain(xs, ys):   # eval_all (mix.i:19-42): exponents below -100 are 0
                v = np.zeros(len(xs))
                for k in range(len(amp)):
                    iv = np.linalg.inv(var[k])
                    dx, dy = xs - fx - mean[k, 0], ys - fy - mean[k, 1]
                    e = -0.5 * (iv[0, 0] * dx * dx + 2 * iv[0, 1] * dx * dy + iv[1, 1] * dy * dy)
                    v += np.where(e < -100, 0., amp[k] / (2 * np.pi * np.sqrt(np.linalg.det(var[k])))
                                  * np.exp(e))
                return v
            if xc < x0 or xc >= x0 + W:
                ex = 0 if xc < x0 else W - 1
                col = plain(np.full(H, x0 + ex, float), np.arange(y0, y0 + H, dtype=float))
                for yy, v in enumerate(col):
                    if v > best:
                        best, cx, cy = v, ex, yy
            if yc < y0 or yc >= y0 + H:
                ey = 0 if yc < y0 else H - 1
                row = plain(np.arange(x0, x0 + W, dtype=float), np.full(W, y0 + ey, float))
                for xx, v in enumerate(row):
                    if v > best:
                        best, cx, cy = v, xx, ey
        if True:
            ev, ext = ring_region(vals, cx, cy, minval, 3)
            assert (planes[0].x0 - x0, planes[0].y0 - y0) == (ext[0], ext[2])
            assert planes[0].patch.shape == (ext[3] - ext[2], ext[1] - ext[0])
            sub = np.where(ev, vals, 0.)[ext[2]:ext[3], ext[0]:ext[1]]
            assert np.array_equal(planes[0].patch, sub)
        # (2) against the oracle's approx3 (FP64 values): the same region and
        # values within 1e-5 of the peak, unless a pixel whose value lies
        # within 1e-5 of minval decided the walk differently in FP32
        same = (planes[0].x0, planes[0].y0) == (x0 + sx0, y0 + sy0) and \
            planes[0].patch.shape == (sy1 - sy0, sx1 - sx0)
        if not same:
            near = np.abs(vals / minval - 1) < 1e-5
            assert near.any(), ((planes[0].x0, planes[0].y0), (x0 + sx0, y0 + sy0))
            flips += 1
            continue
        refs = [out, dxo, dyo] if derivs else [out]
        for p, ref in zip(planes, refs):
            sub = ref[sy0:sy1, sx0:sx1]
            peak = max(np.abs(sub).max(), 1e-300)
            assert np.abs(p.patch - sub).max() <= 1e-5 * peak
            assert np.array_equal(p.patch == 0, sub == 0)
    assert flips <= 2, flips


def test_normal_equations_and_solve(tb):
    import torch
    from tractor_b200 import render
    rng = np.random.default_rng(6)
    Ps, Rs = [6, 11, 54], [4096, 900, 3000]
    A_list, r_list = [], []
    for P, R in zip(Ps, Rs):
        A = rng.normal(size=(R, P)).astype(np.float32) * rng.uniform(0.1, 100, P).astype(np.float32)
        r = rng.normal(size=R).astype(np.float32)
        A_list.append(A)
        r_list.append(r)
    A_flat = np.concatenate([a.T.ravel() for a in A_list])
    r_flat = np.concatenate(r_list)
    a_off = np.concatenate([[0], np.cumsum([a.size for a in A_list])[:-1]])
    r_off = np.concatenate([[0], np.cumsum(Rs)[:-1]])
    AtA, Atr, ao, ro = render.normal_equations(torch.from_numpy(A_flat).cuda(),
                                               torch.from_numpy(r_flat).cuda(),
                                               a_off, r_off, Rs, Ps, Rs)
    X, info, x_off = render.solve_update(AtA, Atr, ao, ro, Ps)
    AtA, Atr, X = AtA.cpu().numpy(), Atr.cpu().numpy(), X.cpu().numpy()
    assert np.all(info.cpu().numpy() == 0)
    o = 0
    for i, (P, A, r) in enumerate(zip(Ps, A_list, r_list)):
        M = AtA[o:o + P * P].reshape(P, P)
        A64 = A.astype(np.float64)
        refM = A64.T @ A64
        assert np.abs(M - refM).max() / np.abs(refM).max() < 1e-6
        xs, *_ = np.linalg.lstsq(A64, r.astype(np.float64), rcond=None)
        got = X[x_off[i]:x_off[i] + P]
        assert np.abs(got - xs).max() / np.abs(xs).max() < 1e-5
        o += P * P


def test_chi2(tb):
    import torch
    from tractor_b200 import render
    rng = np.random.default_rng(7)
    n = [4096, 100000, 17]
    d = rng.normal(size=sum(n)).astype(np.float32)
    m = rng.normal(size=sum(n)).astype(np.float32)
    ie = rng.uniform(0.5, 2, size=sum(n)).astype(np.float32)
    off = np.concatenate([[0], np.cumsum(n)[:-1]])
    got = render.chi2(*(torch.from_numpy(a).cuda() for a in (d, m, ie)), off, n).cpu().numpy()
    for i in range(3):
        s = slice(off[i], off[i] + n[i])
        chi = (d[s] - m[s]) * ie[s]
        ref = np.sum(chi.astype(np.float64) ** 2)
        assert abs(got[i] - ref) / ref < 1e-6
