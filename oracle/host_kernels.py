"""Test infrastructure: CPU stand-ins for the device kernels, so the host-side
logic of tractor_b200 (geometry rules, plan bookkeeping, finite-difference
arithmetic, least-squares assembly) can be tested without a GPU.

Installed by the `host_only` fixture and the host backend of the API tests
(tests/fake_device.py re-exports this module), and by the CPU-baseline leg of
bench.py for the small plain fit: the same object-API fit with every kernel
computed by the oracle's C / numpy code on the host, the shape of the
reference's own CPU path (Python driving C kernels).  The stand-ins compute
each kernel's documented result; they never ship and the product path never
reaches them (it raises without a CUDA device).
"""
import numpy as np
import torch

from oracle import oracle as O


def mog_items(items, amp, mean, var, masks, out):
    """tb_mog_render's result, item by item, in FP64 (a difference item as
    the difference of its two mixtures' values, both with the first one's
    means)."""
    for it in items:
        x0, y0, w, h, c0, K = (int(it[k]) for k in ('x0', 'y0', 'w', 'h', 'c0', 'K'))
        m = mean[c0:c0 + K]
        yy, xx = np.mgrid[y0:y0 + h, x0:x0 + w].astype(np.float64)
        val = np.zeros((h, w))
        gx = np.zeros((h, w))
        gy = np.zeros((h, w))
        sets = [(c0, 1.)]
        if it['diff_c0'] >= 0:
            sets = [(int(it['diff_c0']), 1.), (c0, -1.)]
        for cs, sign in sets:
            a = amp[cs:cs + K]
            V = var[cs:cs + K]
            asum = a.sum()
            v, g1, g2 = _mog_values(it, a, m, V, asum, xx, yy)
            val += sign * v
            gx += sign * g1
            gy += sign * g2
        _mog_store(it, val, gx, gy, masks, out)


def _mog_values(it, a, m, V, asum, xx, yy):
    """Values and d/dmean planes of one mixture on the pixel grid (xx, yy)."""
    val = np.zeros(xx.shape)
    gx = np.zeros(xx.shape)
    gy = np.zeros(xx.shape)
    for k in range(len(a)):
        vxx, vyy = V[k, 0, 0], V[k, 1, 1]
        vxy = 0.5 * (V[k, 0, 1] + V[k, 1, 0])
        det = vxx * vyy - vxy * vxy
        q0, q1, q2 = -0.5 * vyy / det, vxy / det, -0.5 * vxx / det
        s = a[k] / (2 * np.pi * np.sqrt(det))
        fl = it['floor']
        if it['floor_mode'] == 1:
            fl = -100.
            if it['floor'] > 0:
                fl = max(-100., np.log(it['floor'] * 2 * np.pi * np.sqrt(det) / asum))
        dx = xx - it['fx'] - m[k, 0]
        dy = yy - it['fy'] - m[k, 1]
        e = q0 * dx * dx + q1 * dx * dy + q2 * dy * dy
        G = np.where(e >= fl, s * np.exp(e), 0.)
        val += G
        gx += -G * (2 * q0 * dx + q1 * dy)
        gy += -G * (2 * q2 * dy + q1 * dx)
    return val, gx, gy


def _mog_store(it, val, gx, gy, masks, out):
    """Writes one item's planes as the kernel does (mask, scale, mode)."""
    w, h = int(it['w']), int(it['h'])
    on = np.ones((h, w), bool)
    if it['mask_off'] >= 0:
        on = masks[it['mask_off']:it['mask_off'] + w * h].reshape(h, w).astype(bool)
    sc = float(np.float32(it['scale']))
    val = np.where(on, val * sc, 0.).astype(np.float32)
    ldo = int(it['ldo']) if it['ldo'] > 0 else w
    base = int(it['out_off'])
    for r in range(h):
        dst = out[base + r * ldo: base + r * ldo + w]
        if it['mode'] == 0:
            dst[:] = val[r]
        else:
            dst[:] += val[r]
    if it['deriv_off'] >= 0:
        d = int(it['deriv_off'])
        out[d:d + w * h] = np.where(on, gx * sc, 0.).astype(np.float32).ravel()
        out[d + w * h:d + 2 * w * h] = np.where(on, gy * sc, 0.).astype(np.float32).ravel()


def fft_items(items, amp, var, specs, out, dcoef=None):
    """tb_fourier_render's result, item by item (a TB_FFT_DIFF item as the
    FP64 difference of its two mixtures' spectra)."""
    for it in items:
        c0, K, N = int(it['c0']), int(it['K']), int(it['sz'])
        NH = N // 2 + 1
        so = int(it['spec_off'])
        P = specs[so:so + 2 * N * NH].view(np.complex64).reshape(NH, N).T
        fv, fw = np.fft.rfftfreq(N), np.fft.fftfreq(N)
        F = O.fourier_mog(amp[c0:c0 + K], var[c0:c0 + K], fv, fw)
        if it['dmode'] == 4:
            dc = dcoef[int(it['dc0']):int(it['dc0']) + K]
            V2 = var[c0:c0 + K].copy()
            V2[:, 0, 0] += dc[:, 1]
            V2[:, 0, 1] += dc[:, 2]
            V2[:, 1, 0] += dc[:, 2]
            V2[:, 1, 1] += dc[:, 3]
            F = O.fourier_mog(amp[c0:c0 + K] + dc[:, 0], V2, fv, fw) - F
        G = np.fft.irfftn(F * P).astype(np.float32)
        if it['mux'] != 0 or it['muy'] != 0:
            G = O.lanczos_shift(G, it['mux'], it['muy'])
        mw, mh, sx, sy = int(it['mw']), int(it['mh']), int(it['sx']), int(it['sy'])
        res = np.zeros((mh, mw), np.float32)
        for i in range(mh):
            r = i - sy
            if not (0 <= r < N):
                continue
            for j0 in range(mw):
                pass
            cols = np.arange(mw) - sx
            ok = (cols >= 0) & (cols < N)
            res[i, ok] = G[r, cols[ok]]
        res *= np.float32(it['scale'])
        ldo = int(it['ldo']) if it['ldo'] > 0 else mw
        base = int(it['out_off'])
        for r in range(mh):
            dst = out[base + r * ldo: base + r * ldo + mw]
            if it['mode'] == 0:
                dst[:] = res[r]
            else:
                dst[:] += res[r]


def ring_region(vals, cx, cy, minval, minradius):
    """c_gauss_2d_approx3's ring walk (tractor/approx3.c:126-442) over the
    box's values: boolean mask of evaluated pixels and (sx0, sx1, sy0, sy1)
    (exclusive upper bounds), for box-relative start pixel (cx, cy)."""
    H, W = vals.shape
    ev = np.zeros((H, W), bool)

    def mark(arr, i, n):
        if 0 <= i < n:
            arr[i] = True

    nT, nB = np.zeros(W, bool), np.zeros(W, bool)
    nL, nR = np.zeros(H, bool), np.zeros(H, bool)
    if cy > 0:
        for d in (-1, 0, 1):
            mark(nB, cx + d, W)
    if cy < H - 1:
        for d in (-1, 0, 1):
            mark(nT, cx + d, W)
    if cx > 0:
        mark(nL, cy, H)
    if cx < W - 1:
        mark(nR, cy, H)
    ev[cy, cx] = True
    sx0 = sx1 = cx
    sy0 = sy1 = cy

    def spread(marks, n):
        """Union of i-1, i, i+1 over marked i, clipped to [0, n)."""
        out = marks.copy()
        out[1:] |= marks[:-1]
        out[:-1] |= marks[1:]
        return out

    R = 1
    while True:
        cT, cB, cL, cR = nT, nB, nL, nR
        nT, nB = np.zeros(W, bool), np.zeros(W, bool)
        nL, nR = np.zeros(H, bool), np.zeros(H, bool)
        anyev = False
        # top (y = cy + R), bottom (y = cy - R)
        for side in (0, 1):
            y = cy + R if side == 0 else cy - R
            if not (0 <= y < H):
                continue
            cur = cT if side == 0 else cB
            idx = np.flatnonzero(cur)
            if len(idx) == 0:
                continue
            anyev = True
            ev[y, idx] = True
            if side == 0:
                sy1 = y
            else:
                sy0 = y
            ok = np.zeros(W, bool)
            ok[idx] = (R <= minradius) | (vals[y, idx] >= minval)
            inward = -1 if side == 0 else 1
            if cx - R > 0 and 0 <= cx - R < W and ok[cx - R]:
                mark(nL, y, H)
                mark(nL, y + inward, H)
            if cx + R < W - 1 and 0 <= cx + R < W and ok[cx + R]:
                mark(nR, y, H)
                mark(nR, y + inward, H)
            if (side == 0 and y < H - 1) or (side == 1 and y > 0):
                nxt = spread(ok, W)
                if side == 0:
                    nT |= nxt
                else:
                    nB |= nxt
        # left (x = cx - R), right (x = cx + R)
        for side in (0, 1):
            x = cx - R if side == 0 else cx + R
            if not (0 <= x < W):
                continue
            cur = cL if side == 0 else cR
            idx = np.flatnonzero(cur)
            if len(idx) == 0:
                continue
            anyev = True
            ev[idx, x] = True
            if side == 0:
                sx0 = x
            else:
                sx1 = x
            ok = np.zeros(H, bool)
            ok[idx] = (R <= minradius) | (vals[idx, x] >= minval)
            if (side == 0 and x > 0) or (side == 1 and x < W - 1):
                nxt = spread(ok, H)
                if side == 0:
                    nL |= nxt
                else:
                    nR |= nxt
        if not anyev:
            break
        R += 1
    return ev, (sx0, sx1 + 1, sy0, sy1 + 1)


def ring_items(rings, out):
    """tb_approx3_region's result: each walk's start, region and extent, the
    other pixels of the box (and of its derivative planes) set to zero."""
    ext = np.zeros((len(rings), 4), np.int32)
    for i, r in enumerate(rings):
        W, H = int(r['w']), int(r['h'])
        vo = int(r['val_off'])
        vals = out[vo:vo + W * H].reshape(H, W).astype(np.float64)
        if r['start_inside']:
            cx, cy = int(r['xc']), int(r['yc'])
        else:
            best, cx, cy = 0., int(r['dcx']), int(r['dcy'])
            if r['edge_col_off'] >= 0:
                col = out[int(r['edge_col_off']):int(r['edge_col_off']) + H]
                for y, v in enumerate(col):
                    if v > best:
                        best, cx, cy = v, int(r['edge_x']), y
            if r['edge_row_off'] >= 0:
                row = out[int(r['edge_row_off']):int(r['edge_row_off']) + W]
                for x, v in enumerate(row):
                    if v > best:
                        best, cx, cy = v, x, int(r['edge_y'])
        ev, e = ring_region(vals, cx, cy, float(r['minval']), int(r['minradius']))
        ext[i] = e
        offs = [vo] + ([int(r['deriv_off']), int(r['deriv_off']) + W * H]
                       if r['deriv_off'] >= 0 else [])
        for o in offs:
            plane = out[o:o + W * H].reshape(H, W)
            plane[~ev] = 0.
    return ext


def install(monkeypatch):
    from tractor_b200 import render, _lib

    monkeypatch.setattr(render, 'device', lambda: torch.device('cpu'))

    def mog_run(self, out=None, stream=None, check=True):
        if out is None:
            # packed outputs carry the (zero) status word at their end, as the
            # device batches do
            out = torch.zeros(max(self.nout, 1) + 4, dtype=torch.float32)
        if self.items:
            items = np.array(self.items, dtype=_lib.MOG_ITEM)
            masks = np.concatenate(self.masks) if self.masks else None
            o = out.numpy()
            mog_items(items, np.concatenate(self.amp), np.concatenate(self.mean),
                      np.concatenate(self.var), masks, o)
        self.extents = None
        self.ring_status = None
        if self.rings:
            self.extents = torch.from_numpy(ring_items(self.rings, out.numpy()).ravel())
            self.ring_status = torch.zeros(16, dtype=torch.uint8)
        self.status = torch.zeros(16, dtype=torch.uint8)
        return out

    def fft_run(self, out=None, stream=None, check=True):
        if out is None:
            # packed outputs carry the (zero) status word at their end, as the
            # device batches do
            out = torch.zeros(max(self.nout, 1) + 4, dtype=torch.float32)
        if self.items:
            items = np.array(self.items, dtype=_lib.FFT_ITEM)
            specs = torch.cat(self.spec_list).numpy()
            fft_items(items, np.concatenate(self.amp), np.concatenate(self.var), specs, out.numpy(),
                      np.concatenate(self.dcoef) if self.dcoef else None)
        self.status = torch.zeros(16, dtype=torch.uint8)
        return out

    def spectra_compute(self, img, sz, normalize=False):
        pad, cx, cy = render.PsfSpectra.pad(img, sz)
        P = np.fft.rfft2(pad).astype(np.complex64)
        if normalize:
            n = np.abs(P[0][0])
            if n != 0:
                P /= n
        flat = np.ascontiguousarray(P.T).view(np.float32).ravel()
        return (torch.from_numpy(flat.copy()), cx, cy)

    def spectra_get(self, key, img, sz, normalize=False):
        k = (key, sz, bool(normalize))
        if k not in self.cache:
            self.cache[k] = spectra_compute(self, img, sz, normalize)
        return self.cache[k]

    def lanczos(imgs, shifts, stream=None):
        a = imgs.numpy()
        sh = np.asarray(shifts, np.float64).reshape(len(a), 2)
        return torch.from_numpy(np.stack([O.lanczos_shift(a[i], sh[i, 0], sh[i, 1])
                                          for i in range(len(a))]))

    def normal_equations(A, rhs, a_off, r_off, lda, P, R, stream=None):
        A = A.numpy()
        rhs = rhs.numpy()
        AtA, Atr, ao, ro = [], [], [], []
        oa = orr = 0
        for b in range(len(P)):
            M = A[a_off[b]:a_off[b] + P[b] * lda[b]].reshape(P[b], lda[b])[:, :R[b]].astype(np.float64)
            r = rhs[r_off[b]:r_off[b] + R[b]].astype(np.float64)
            AtA.append((M @ M.T).ravel())
            Atr.append(M @ r)
            ao.append(oa)
            ro.append(orr)
            oa += P[b] * P[b]
            orr += P[b]
        return (torch.from_numpy(np.concatenate(AtA)), torch.from_numpy(np.concatenate(Atr)),
                torch.tensor(ao), torch.tensor(ro))

    def solve_update(AtA, Atr, ata_off, atr_off, P, damp=0., stream=None):
        AtA, Atr = AtA.numpy(), Atr.numpy()
        X, info, xo = [], [], []
        o = 0
        for b, p in enumerate(P):
            M = AtA[int(ata_off[b]):int(ata_off[b]) + p * p].reshape(p, p)
            g = Atr[int(atr_off[b]):int(atr_off[b]) + p]
            d = np.sqrt(np.where(np.diag(M) > 0, np.diag(M), 0.))
            ds = np.where(d > 0, d, 1.)
            Ms = M / ds[:, None] / ds[None, :] + damp ** 2 * np.eye(p)
            for i in np.flatnonzero(d == 0):
                Ms[i, :] = 0
                Ms[:, i] = 0
                Ms[i, i] = 1
            gs = np.where(d > 0, g / ds, 0.)
            try:
                x = np.linalg.solve(Ms, gs)
                info.append(0)
            except np.linalg.LinAlgError:
                x = np.zeros(p)
                info.append(1)
            X.append(np.where(d > 0, x / ds, 0.))
            xo.append(o)
            o += p
        return torch.from_numpy(np.concatenate(X)), torch.tensor(info, dtype=torch.int32), \
            np.array(xo)

    def em_run(imgs, amp, mean, var, alpha, steps, xy):
        n, ny, nx = imgs.shape
        amp, mean, var = amp.copy(), mean.copy(), var.copy()
        st = np.zeros(n, np.int32)
        for i in range(n):
            x0, y0 = (int(xy[i, 0]), int(xy[i, 1])) if xy is not None else (-(nx // 2),
                                                                           -(ny // 2))
            st[i] = O.em_fit_2d_reg(imgs[i], x0, y0, amp[i], mean[i], var[i], alpha, steps) != 0
        return amp, mean, var, st

    def label_run(mask, conn8):
        import scipy.ndimage as ndi
        st = np.ones((3, 3), bool) if conn8 else None
        lab, n = ndi.label(np.asarray(mask) != 0, structure=st)
        return lab.astype(np.int32), int(n)

    def boxes_run(labels, n):
        import scipy.ndimage as ndi
        out = np.tile(np.array([labels.shape[0], labels.shape[1], 0, 0], np.int32), (n, 1))
        for l, sl in enumerate(ndi.find_objects(labels, n)):
            if sl is not None:
                out[l] = (sl[0].start, sl[1].start, sl[0].stop, sl[1].stop)
        return out

    from tractor_b200 import emfit, blobs
    monkeypatch.setattr(emfit, '_run', em_run)
    monkeypatch.setattr(blobs, '_run_label', label_run)
    monkeypatch.setattr(blobs, '_run_boxes', boxes_run)

    def segment_run(mask, conn8):
        lab, n = label_run(mask, conn8)
        return lab, n, boxes_run(lab, n)
    monkeypatch.setattr(blobs, '_run_segment', segment_run)
    monkeypatch.setattr(render.MogBatch, 'run', mog_run)
    monkeypatch.setattr(render.FftBatch, 'run', fft_run)
    monkeypatch.setattr(render.PsfSpectra, 'get', spectra_get)
    monkeypatch.setattr(render.PsfSpectra, 'compute', spectra_compute)
    monkeypatch.setattr(render, 'lanczos_shift', lanczos)
    monkeypatch.setattr(render, 'normal_equations', normal_equations)
    monkeypatch.setattr(render, 'solve_update', solve_update)

    def solve_dense(A_colmajor, b, damp=0., stream=None):
        A = torch.from_numpy(np.ascontiguousarray(A_colmajor, np.float32).ravel())
        P, R = A_colmajor.shape
        AtA, Atr, ao, ro = normal_equations(A, torch.from_numpy(np.asarray(b, np.float32)),
                                            [0], [0], [R], [P], [R])
        X, info, _ = solve_update(AtA, Atr, ao, ro, [P], damp=damp)
        return X.numpy(), int(info[0])
    monkeypatch.setattr(render, 'solve_dense', solve_dense)
    render._spectra.cache.clear()
