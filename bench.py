"""Benchmark: the pixelized-PSF Fourier rendering workload.

Workload (per GPU): 256 SersicGalaxy sources (n ~ U[0.7, 6], r_e log-uniform
in [0.5, 8] px, axis ratio U[0.2, 1], phi U[0, 180)), each on its own 128x128
ModelMask, PSF a 63x63 normalised Moffat image (beta 3, FWHM 4 px) used as a
PixelizedPSF, sub-pixel offsets U[-0.5, 0.5] applied by Lanczos-3.  The FFT
size is 256 (the reference's next power of two of twice the patch
half-size).  Synthetic, seeded.

One step = render every source's model patch from its parameters already in
device memory, by the fastest of three methods timed first on the workload:
tb_galaxy_fft_render (each source's profile, shape and geometry prepared by
one warp into shared memory, then spectrum, FFTs, Lanczos and crop by its
block: one persistent launch), or tb_galaxy_fft_prep followed by the
persistent tb_fourier_render or by tb_fourier_render_split (column and row
kernels through an L2-resident scratch).  The metric
is Mpix x components per second with Npix = sz^2 per source and the
source's Gaussian component count (SersicGalaxy mixtures have 5-9), summed
over sources.  L2 is flushed (a 256 MB write) before every timed step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

The JSON line ends with a summary, under "secondary", of the other
workloads (the full record of each goes to stderr as its own JSON line):
C3 the batched scene (20,000 point / exp / deV / composite sources on one
4096x4096 image through a 3-component MoG PSF; prep + binning + one
persistent tile render, the tile height autotuned), C5 batched blob fitting
(2,000 blobs x 3 bands; with N GPUs the blobs are cost-balanced over the
ranks: strong scaling), C4 the seven analytic derivative columns of the
Fourier path, K5 the dense normal equations on the tensor cores (512
problems x 63 parameters x 16,384 rows), C1 the small plain fit through the
object API (latency-bound: us per render, ms per fit), EM fits of 4,096 PSF
stamps (GaussianMixturePSF.fromStamp's em_fit_2d_reg, FP64) and SEG blob
segmentation of a 4096x4096 detection map, each with its own end-to-end
number, roofline and CPU baseline (--no-secondary skips them, --only picks
some).

With N GPUs the headline workload is one set of 256 x N sources,
cost-balanced over the ranks (about 256 each: weak scaling), and the ranks'
patches are all-gathered once after the timed steps.

--impl reference times the reference's CPU implementation of the same
workload on the host cores (its own compiled C for the spectrum and the
Lanczos shift, numpy's irfftn, galaxy.py's geometry), one source per task
over all cores, each step a bounded sample of the 256 sources.
"""
import argparse
import json
import multiprocessing as mp
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_SOURCES = 256
MASK = 128
SFU_EX2_PER_CLK_PER_SM = 16      # MUFU.EX2 issue rate of an SM (sm_100)
WORKLOAD = ('256 SersicGalaxy sources, each on a 128x128 ModelMask, 63x63 Moffat '
            'PixelizedPSF (FFT 256, Lanczos-3)')
METRIC = 'Mpix*components/s (pixelized-PSF Fourier render)'


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=50)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--cpu-seconds', type=float, default=12.0)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-secondary', action='store_true',
                    help='skip the batched-scene, blob-fitting and normal-equation '
                         'measurements')
    ap.add_argument('--fit-blobs', type=int, default=2000,
                    help='blobs in the blob-fitting measurement (2000 = the full workload)')
    ap.add_argument('--fourier-method', default='auto',
                    choices=['auto', 'fused', 'persistent', 'split'],
                    help='Fourier render method of the headline (auto: the fastest on this '
                         'workload, timed first)')
    ap.add_argument('--ne-problems', type=int, default=0,
                    help='problems in the normal-equation measurement (0: the full workload)')
    ap.add_argument('--secondary-only', action='store_true',
                    help='run only the secondary measurements (with --only: one kernel, for '
                         'profiling); the line then carries no headline figures')
    ap.add_argument('--only', default='',
                    help='comma-separated secondary measurements to run (C3, C5, C4, K5, C1, '
                         'EM, SEG); default all')
    return ap.parse_args()


def config_keys():
    """The workload's config, the same in both arms."""
    return {'workload': WORKLOAD, 'n_sources': N_SOURCES, 'mask': MASK, 'fft_size': 256,
            'l2': 'flushed before every timed step (256 MB write)'}


def _sig(x, d=4):
    if isinstance(x, float) and np.isfinite(x) and x != 0.:
        return float('%.*g' % (d, x))
    return x


def compact(sec):
    """A secondary measurement's key numbers (value, end to end, roofline
    fraction, CPU baseline, parity) for the main JSON line."""
    if 'error' in sec:
        return {'error': sec['error']}
    c = {'v': _sig(sec.get('value')), 'u': sec.get('unit'), 'ms': _sig(sec.get('ms_per_step'))}
    if isinstance(sec.get('e2e'), dict):
        c['e2e'] = _sig(sec['e2e']['value'])
    rf = sec.get('roofline')
    if isinstance(rf, dict):
        c['frac'] = _sig(rf.get('frac'), 3)
        c['bound'] = rf.get('bound')
    cb = sec.get('cpu_baseline')
    if isinstance(cb, dict):
        c['cpu'] = _sig(cb.get('value'))
        c['cpu_kind'] = cb.get('kind')
        c['cores'] = cb.get('cores')
    for k, v in (sec.get('summary') or {}).items():
        c[k] = _sig(v, 3) if isinstance(v, float) else v
    return c


# ---------------------------------------------------------------------------
# CPU side (oracle port / reference C), one source per task
# ---------------------------------------------------------------------------

def _cpu_worker(args):
    """Renders sources [i0, i1) of the workload on the CPU; returns
    (pix*components, seconds)."""
    i0, i1, seed, use_ref, budget = args
    sys.path.insert(0, ROOT)
    os.environ.setdefault('OMP_NUM_THREADS', '1')
    from oracle import oracle as O
    from tractor_b200 import batch
    rng = np.random.default_rng(seed)
    srcs = batch.sersic_sources(N_SOURCES, rng, mask=MASK)
    psf = batch.moffat_psf()
    kern = O.reference_kernels() if use_ref else None
    cdinv = O.nullwcs_cdinv()
    work = 0.
    t0 = time.perf_counter()
    i = i0
    while i < i1:
        s = srcs[i]
        amp, var = O.sersic_profile(float(s['sersic_n']))
        T = cdinv @ O.ellipseE_basis(s['s0'], s['s1'], s['s2'])
        a2, v2 = O.sheared(amp, var, T)
        _, (_, _, _, _, sz) = O.galaxy_fft_masked(a2, v2, s['px'], s['py'], psf, 0, 0, MASK, MASK,
                                                  kernels=kern)
        work += sz * sz * len(amp)
        i += 1
        if time.perf_counter() - t0 > budget:
            break
    return work, time.perf_counter() - t0, i - i0


def fourier_plain_fp64(srcs, out, dev, budget):
    """The plain FP64 GPU renderer (tractor_b200.plain.fourier_render_fp64:
    one galaxy at a time, FP64 torch ops and cuFFT) over the workload's
    sources for about `budget` seconds: Mpix x components / s, and the
    batched FP32 patches' largest deviation from it (of each patch's peak)."""
    import torch
    from tractor_b200 import plain, profiles
    psf = batch_moffat()
    cdinv = np.eye(2) * 3600.
    specs = {}
    got = out.view(len(srcs), MASK, MASK)
    err, work, n = 0., 0., 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i, s in enumerate(srcs):
        amp, var = profiles.sersic_mixture().profile(float(s['sersic_n']))
        from tractor_b200 import ellipses
        G = ellipses.EllipseE(s['s0'], s['s1'], s['s2']).getRaDecBasis()
        T = cdinv @ G
        v2 = np.array([v * (T @ T.T) for v in var])
        hs = max(MASK / 2., 1 + s['px'], 1 + MASK - s['px'], 1 + s['py'], 1 + MASK - s['py'], 31.5)
        sz = 1
        while sz < 2 * np.ceil(hs):
            sz *= 2
        if sz not in specs:
            specs[sz] = plain.psf_spectrum_fp64(psf.astype(np.float64), sz, dev)
        spec, cx, cy = specs[sz]
        p = plain.fourier_render_fp64(amp, v2, spec, cx, cy, sz, float(s['px']), float(s['py']),
                                      0, 0, MASK, MASK, counts=float(s['counts']))
        g = got[i].double()
        err = max(err, float((g - p).abs().max() / p.abs().max()))
        work += sz * sz * len(amp)
        n += 1
        if time.perf_counter() - t0 > budget:
            break
    e1.record()
    e1.synchronize()
    secs = e0.elapsed_time(e1) / 1e3
    return {'value': work / secs / 1e6, 'unit': 'Mpix*components/s', 'sources': n,
            'seconds': secs, 'batched_fp32_max_err_of_peak': err,
            'how': 'tractor_b200.plain.fourier_render_fp64, one galaxy at a time, FP64 torch '
                   'ops and cuFFT on the same GPU'}


def batch_moffat():
    from tractor_b200 import batch
    return batch.moffat_psf()


def cpu_rate(seconds, use_ref, seed=1000):
    """Mpix*components/s of the CPU path on all host cores (spawned worker
    processes), over a bounded sample of the workload."""
    ncores = os.cpu_count() or 1
    ctx = mp.get_context('spawn')
    per = max(1, N_SOURCES // ncores)
    tasks = []
    for c in range(ncores):
        i0 = (c * per) % N_SOURCES
        tasks.append((i0, min(N_SOURCES, i0 + per), seed, use_ref, seconds))
    t0 = time.perf_counter()
    with ctx.Pool(ncores) as pool:
        res = pool.map(_cpu_worker, tasks)
    wall = time.perf_counter() - t0
    work = sum(r[0] for r in res)
    nsrc = sum(r[2] for r in res)
    busy = max(r[1] for r in res)
    return work / busy / 1e6, ncores, nsrc, wall


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------

class ClockSampler(object):
    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.gpu), '--query-gpu=' + self.QUERY,
                 '--format=csv,noheader,nounits', '-lms', '100'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in self.lines:
            f = [x.strip() for x in ln.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() in ('active', '1', 'yes'):
                    reasons.add(nm)
        if not sm:
            return None
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': mx, 'reasons': sorted(reasons),
                'samples': len(sm)}


# ---------------------------------------------------------------------------
# secondary workload: the batched scene (20,000 sources on one 4096^2 image)
# ---------------------------------------------------------------------------

SCENE_N = 20000
SCENE_WH = 4096
SCENE_WORKLOAD = ('20,000 sources (40% point, 30% exp, 20% deV, 10% exp+deV composite) on one '
                  '4096x4096 float32 image, square ModelMasks of half-width log-U[7, 127], '
                  'fluxes log-U[10, 1e5], 3-component MoG PSF')


def _scene_inputs(seed):
    from tractor_b200 import batch
    rng = np.random.default_rng(seed)
    s1 = rng.uniform(1., 2.)
    sig, wts = [s1, 2 * s1, 4 * s1], [0.7, 0.2, 0.1]
    recs = batch.scene_sources(SCENE_N, rng, W=SCENE_WH, H=SCENE_WH)
    return recs, sig, wts


def _scene_cpu_worker(args):
    """Oracle scene render of records [i0, i1) (each source's grid over its
    mask clipped to the image); returns (pix*components, seconds, count)."""
    i0, i1, seed, budget = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    recs, sig, wts = _scene_inputs(seed)
    pa = np.asarray(wts, np.float64)
    pm = np.zeros((3, 2))
    pv = np.zeros((3, 2, 2))
    pv[:, 0, 0] = pv[:, 1, 1] = np.asarray(sig) ** 2
    kind = {4: 0, 0: 1, 1: 2, 5: 3}
    work, t0, i = 0., time.perf_counter(), i0
    while i < i1 and time.perf_counter() - t0 < budget:
        q = recs[i]
        x0, y0 = max(q['mx0'], 0), max(q['my0'], 0)
        x1, y1 = min(q['mx0'] + q['mw'], SCENE_WH), min(q['my0'] + q['mh'], SCENE_WH)
        if x1 > x0 and y1 > y0:
            ca, cm, cv, fx, fy = O.scene_source_mixture(
                kind[int(q['profile'])], q['px'], q['py'], q['fdev'],
                [q['sa0'], q['sa1'], q['sa2']], [q['sb0'], q['sb1'], q['sb2']], pa, pm, pv)
            O.mog_grid(x0, x1, y0, y1, fx, fy, ca, cm, cv)
            work += (x1 - x0) * (y1 - y0) * len(ca)
        i += 1
    return work, time.perf_counter() - t0, i - i0


def scene_cpu_rate(seconds, seed):
    ncores = os.cpu_count() or 1
    per = SCENE_N // ncores
    tasks = [(c * per, (c + 1) * per, seed, seconds) for c in range(ncores)]
    with mp.get_context('spawn').Pool(ncores) as pool:
        res = pool.map(_scene_cpu_worker, tasks)
    work = sum(r[0] for r in res)
    busy = max(r[1] for r in res)
    return work / busy / 1e6, ncores, sum(r[2] for r in res)


def bench_scene(args, dev, flush, clk, cpu_seconds):
    """The batched-scene workload: autotuned tile height, device-timed steps
    (prep + bin + render from records resident in HBM, L2 flushed), the
    host-buffer call end to end, roofline against the SFU ex2 rate."""
    import ctypes
    import torch
    from tractor_b200 import batch, _lib, render as R
    recs, sig, wts = _scene_inputs(2000)
    img = batch.SceneImage.circular(SCENE_WH, SCENE_WH, sig, wts)
    r = batch.SceneRenderer([img])
    n = len(recs)
    pinned = torch.from_numpy(recs.view(np.uint8).copy()).pin_memory()
    d_src = pinned.to(dev)
    mp_by_h = dict((th, r.max_pairs(recs, th)) for th in batch.SCENE_TILE_HEIGHTS)
    tune = r.autotune(d_src, n, mp_by_h)
    th = r.tile_h
    out = torch.empty(r.npix, dtype=torch.float32, device=dev)
    out_pinned = torch.empty(r.npix, dtype=torch.float32).pin_memory()
    for _ in range(max(3, args.warmup)):
        r.render_device(d_src, n, out, mp_by_h[th], th)
    torch.cuda.synchronize()
    items = r.items(n)
    assert np.all(items['flag'] == 0)
    pixcomp = float(np.sum(items['w'].astype(np.float64) * items['h'] * items['K']))
    lib = _lib.load()
    d_img, n_tiles = r.image_table(th)
    _, ws, it_t, comps, status = r.workspace(n, mp_by_h[th], th)
    stride = r.comp_stride
    base = comps.data_ptr()
    camp, cmean, cvar = base, base + 8 * n * stride, base + 24 * n * stride
    pb = r._psf.data_ptr()
    steps = max(3, min(args.steps, 20))
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
    stream = _lib.stream_ptr()
    for k in range(steps):
        flush.zero_()
        ev[k][0].record()
        _lib.check(lib.tb_scene_prep(d_src.data_ptr(), n, d_img.data_ptr(), 1, pb + r._o_pamp,
                                     pb + r._o_pmean, pb + r._o_pvar,
                                     ctypes.addressof(r.tables.struct), it_t.data_ptr(), camp,
                                     cmean, cvar, stride, stream), 'tb_scene_prep')
        ev[k][1].record()
        _lib.check(lib.tb_scene_render(it_t.data_ptr(), n, d_img.data_ptr(), 1, n_tiles, th,
                                       camp, cmean, cvar, out.data_ptr(), _lib.MOG_STORE,
                                       ws.data_ptr(), ws.numel(), mp_by_h[th],
                                       status.data_ptr(), stream), 'tb_scene_render')
        ev[k][2].record()
    torch.cuda.synchronize()
    step_s = sum(e[0].elapsed_time(e[2]) for e in ev) / 1e3 / steps
    render_s = sum(e[1].elapsed_time(e[2]) for e in ev) / 1e3 / steps
    R.check_status(status.clone(), 'tb_scene_render')
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    for k in range(steps):
        flush.zero_()
        ev2[k][0].record()
        d_src.copy_(pinned, non_blocking=True)
        r.render_device(d_src, n, out, mp_by_h[th], th)
        out_pinned.copy_(out, non_blocking=True)
        ev2[k][1].record()
    torch.cuda.synchronize()
    e2e_s = sum(a.elapsed_time(b) for a, b in ev2) / 1e3 / steps
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    peak_clk = clk['sm_mhz'] if clk else 1965.0
    peak = SFU_EX2_PER_CLK_PER_SM * nsm * peak_clk * 1e6 / 1e9
    achieved = pixcomp / render_s / 1e9
    line = {
        'workload': SCENE_WORKLOAD,
        'metric': 'Mpix*components/s (batched scene render)',
        'value': pixcomp / step_s / 1e6, 'unit': 'Mpix*components/s',
        'ms_per_step': step_s * 1e3, 'steps': steps,
        'pix_components_per_step': pixcomp,
        'autotuned_tile': {'tile_w': 32, 'tile_h': th,
                           'ms_by_tile_h': dict((str(k), v) for k, v in tune.items())},
        'e2e': {'value': pixcomp / e2e_s / 1e6, 'unit': 'Mpix*components/s',
                'h2d_bytes_per_step': int(pinned.numel()),
                'd2h_bytes_per_step': int(out_pinned.numel() * 4)},
        'gpu_launches_per_step': 7,
        'roofline': {'bound': 'sfu', 'kernel': 'tb_scene_render (bin + render)',
                     'achieved': achieved, 'peak': peak, 'unit': 'Gex2/s',
                     'frac': achieved / peak,
                     'algorithmic': 'sum over sources of rectangle pixels x components = '
                                    '%.0f ex2 per launch' % pixcomp,
                     'kernel_ms': render_s * 1e3,
                     'traffic': ncu_traffic('scene_render_c3.json')},
    }
    if cpu_seconds:
        rate, cores, nsrc = scene_cpu_rate(cpu_seconds, 2000)
        line['cpu_baseline'] = {'value': rate, 'unit': 'Mpix*components/s', 'cores': cores,
                                'kind': 'port',
                                'sample': '%d of the 20,000 sources rendered by the oracle '
                                          '(c_gauss_2d_grid restatement), one process per core'
                                          % nsrc}
    return line


# ---------------------------------------------------------------------------
# secondary workload: batched blob fitting (2,000 blobs x 3 bands)
# ---------------------------------------------------------------------------

FIT_FLOPS_PER_PIXCOMP = 58    # FP32 flops of one pixel x component in tb_fit_pass's inner loop


def fit_workload_text(n):
    return ('%d blobs, sides U[192, 512] px, Poisson(6) SersicGalaxy sources clipped to [1, 30] '
            '(n U[0.7, 6], r_e log-U[0.5, 8] px, q U[0.2, 1]), 3 bands (g, r, z) with per-band '
            '3-component MoG PSFs and Gaussian noise sigma U[1, 3]; 9 parameters per source; '
            'fit from a perturbed start until the predicted dlnp < 1e-3' % n)


def _fit_cpu_worker(args):
    """The oracle's FP64 blob fitter (central-difference Jacobian) on blobs
    [b0, b1) of the workload until the time budget; returns (sources fitted,
    seconds)."""
    b0, b1, n_blobs, seed, budget = args
    sys.path.insert(0, ROOT)
    os.environ.setdefault('OMP_NUM_THREADS', '1')
    from oracle import oracle as O
    from tractor_b200 import fit
    w = fit.blob_workload(n_blobs, np.random.default_rng(seed))
    rng = np.random.default_rng(seed + 1)
    done, t0 = 0, time.perf_counter()
    for b in range(b0, b1):
        if time.perf_counter() - t0 > budget:
            break
        s0, s1 = w['blob_src'][b], w['blob_src'][b + 1]
        W, H = (int(v) for v in w['sides'][b])
        rects = [tuple(int(v) for v in (r['x0'], r['y0'], r['w'], r['h']))
                 for r in w['sources'][s0:s1]]
        mod = O.blob_model(w['truth'][s0:s1], rects, W, H, w['psf'][b], 3)
        sig = w['noise'][b][:, None, None]
        data = mod + sig * rng.normal(size=mod.shape)
        inv = np.broadcast_to(1. / sig, mod.shape)
        O.blob_fit(w['start'][s0:s1], rects, W, H, w['psf'][b], 3, data, inv, tol=1e-3,
                   max_iter=60)
        done += s1 - s0
    return done, time.perf_counter() - t0


def fit_cpu_rate(seconds, n_blobs, seed):
    ncores = os.cpu_count() or 1
    per = max(1, n_blobs // ncores)
    tasks = [((c * per) % n_blobs, min(n_blobs, (c * per) % n_blobs + per), n_blobs, seed,
              seconds) for c in range(ncores)]
    with mp.get_context('spawn').Pool(ncores) as pool:
        res = pool.map(_fit_cpu_worker, tasks)
    done = sum(r[0] for r in res)
    busy = max(r[1] for r in res)
    return done / busy, ncores, done


def bench_fit(args, dev, flush, clk, cpu_seconds):
    """Batched blob fitting: fitted sources per second, device-timed from
    data resident in HBM (warm graph), and end to end with the pixels copied
    in from pinned host memory and the parameters copied out."""
    import torch
    from tractor_b200 import fit, shard
    world, rank, _ = init_dist()
    n_blobs_job = args.fit_blobs
    w_all = fit.blob_workload(n_blobs_job, np.random.default_rng(3000))
    # strong scaling: the one fixed set of blobs, cost-balanced over the ranks
    costs = shard.blob_costs(w_all['blob_src'], w_all['sides'], w_all['sources'],
                             w_all['start'])
    own = np.flatnonzero(shard.balance(costs, world) == rank)
    w = fit.subset_workload(w_all, own) if world > 1 else w_all
    n_blobs = len(w['sides'])
    data, inv = fit.render_blobs(w, w['truth'], seed=3001 + rank)
    f = fit.BlobFitter(w['blob_src'], w['sides'], w['psf'], w['sources'], w['start'], data, inv)
    n_src = int(w['blob_src'][-1])
    for _ in range(max(1, min(args.warmup, 2))):
        f.fit(params0=w['start'])
    torch.cuda.synchronize()
    steps = max(2, min(args.steps, 5))
    times, iters = [], []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        iters.append(f.fit(params0=w['start']))
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    st = f.states()
    fit_s = float(np.mean(times))
    n_src_job, n_blobs_job_done, gather_ms = n_src, n_blobs, None
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([fit_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        fit_s = float(t.item())
        t = torch.tensor([n_src, n_blobs], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        n_src_job, n_blobs_job_done = int(t[0].item()), int(t[1].item())
        # the fit's one collective: every blob's parameters gathered at the end
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record()
        bs = w_all['blob_src']
        own_src = np.concatenate([np.arange(bs[b], bs[b + 1]) for b in own]) if len(own) else \
            np.zeros(0, np.int64)
        shard.gather_units(f.params.view(n_src, fit.NPAR), own_src, int(bs[-1]))
        g1.record()
        g1.synchronize()
        gather_ms = g0.elapsed_time(g1)
    # the dominant kernel at full activity: one pass over every blob
    f.reset(w['start'])
    f._prep()
    pe = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    pe[0].record()
    f._pass(0)
    pe[1].record()
    pe[1].synchronize()
    pass_s = pe[0].elapsed_time(pe[1]) / 1e3
    # pixel x component evaluations of one pass: every source's mask pixels
    # inside its blob, Sersic mixtures of up to 9 components x 3 PSF components
    x0 = np.maximum(w['sources']['x0'], 0)
    y0 = np.maximum(w['sources']['y0'], 0)
    side = np.repeat(w['sides'][:, 0], np.diff(w['blob_src']))
    x1 = np.minimum(w['sources']['x0'] + w['sources']['w'], side)
    y1 = np.minimum(w['sources']['y0'] + w['sources']['h'], side)
    area = np.maximum(x1 - x0, 0).astype(np.float64) * np.maximum(y1 - y0, 0)
    kgal = np.array([fit_ncomp(n) for n in w['start'][:, 8]])
    pixcomp = float(np.sum(area * kgal * 3 * 3))   # 3 PSF components, 3 bands
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    peak_clk = clk['sm_mhz'] if clk else 1965.0
    peak = 128 * 2 * nsm * peak_clk * 1e6 / 1e12
    achieved = pixcomp * FIT_FLOPS_PER_PIXCOMP / pass_s / 1e12
    # end to end: pixels in from pinned host memory, fit, parameters out
    h_data = data.cpu().pin_memory()
    h_inv = inv.cpu().pin_memory()
    h_out = torch.empty(n_src * fit.NPAR, dtype=torch.float64).pin_memory()
    e2e = []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        data.copy_(h_data, non_blocking=True)
        inv.copy_(h_inv, non_blocking=True)
        f.fit(params0=w['start'])
        h_out.copy_(f.params, non_blocking=True)
        e1.record()
        e1.synchronize()
        e2e.append(e0.elapsed_time(e1) / 1e3)
    plain = fit_plain_fp64(w, data, inv, f.result(), st['status'], dev, budget=8.0)
    line = {
        'workload': fit_workload_text(n_blobs),
        'metric': 'fitted sources/s (batched LM blob fitting)',
        'value': n_src_job / fit_s, 'unit': 'sources/s', 'ms_per_step': fit_s * 1e3,
        'steps': steps, 'n_sources': n_src_job, 'n_blobs': n_blobs_job_done,
        'scaling': 'strong (one fixed set of blobs, cost-balanced over the ranks)',
        'gather_ms': gather_ms,
        'iterations_per_fit': float(np.mean(iters)),
        'status': {'converged': int(np.sum(st['status'] == 1)),
                   'stopped': int(np.sum(st['status'] == 2)),
                   'iteration_limit': int(np.sum(st['status'] == 3))},
        'mean_blob_iterations': float(st['iters'].mean()),
        'e2e': {'value': n_src / float(np.mean(e2e)), 'unit': 'sources/s',
                'h2d_bytes_per_step': int(h_data.numel() * 4 + h_inv.numel() * 4),
                'd2h_bytes_per_step': int(h_out.numel() * 8)},
        'plain_fp64': plain,
        'summary': {'max_sigma': plain['batched_vs_fp64_optimum_max_sigma'],
                    'parity_blobs': plain['parity_blobs'],
                    'edge': plain['edge_blobs'], 'edge_sigma': plain['edge_max_sigma'],
                    'flat': plain['flat_blobs'], 'flat_sigma': plain['flat_max_sigma'],
                    'limit': int(np.sum(st['status'] == 3)),
                    'limit_sigma': plain['limit_max_sigma'],
                    'limit_inner_sigma': plain['limit_inner_max_sigma'],
                    'stopped': int(np.sum(st['status'] == 2))},
        'roofline': {'bound': 'fp32', 'kernel': 'tb_fit_pass (all blobs running)',
                     'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s',
                     'frac': achieved / peak,
                     'peak_basis': '128 FP32 FMA/clk/SM x 2 x %d SMs x %s MHz' % (nsm, peak_clk),
                     'algorithmic': '%.4g pixel x component evaluations x %d FP32 flops per '
                                    'pass' % (pixcomp, FIT_FLOPS_PER_PIXCOMP),
                     'kernel_ms': pass_s * 1e3,
                     'traffic': ncu_traffic('fit_pass_c5.json')},
    }
    if cpu_seconds:
        rate, cores, done = fit_cpu_rate(cpu_seconds, n_blobs, 3000)
        line['cpu_baseline'] = {'value': rate, 'unit': 'sources/s', 'cores': cores,
                                'kind': 'port',
                                'sample': '%d sources in whole blobs fitted by the oracle\'s '
                                          'FP64 fitter (central-difference Jacobian), one '
                                          'process per core' % done}
    return line


# ---------------------------------------------------------------------------
# secondary workload: analytic derivatives of the Fourier path (C4)
# ---------------------------------------------------------------------------

DERIV_SEED = 1400


def deriv_sources():
    """The derivative workload: the Fourier-path source mix on masks of 32 to
    128 px (log-uniform; FFT sizes 64 to 256)."""
    from tractor_b200 import batch
    rng = np.random.default_rng(DERIV_SEED)
    masks = np.round(np.exp(rng.uniform(np.log(32), np.log(128), N_SOURCES))).astype(np.int64)
    return batch.sersic_sources(N_SOURCES, rng, mask=masks)


def _deriv_cpu_worker(args):
    """The reference's finite-difference derivatives of sources [i0, i1):
    patch0 plus one render per shape parameter and one for the Sersic index
    (galaxy.py:137-223, sersic.py:402-445; position and flux columns come from
    patch0), each through the reference's compiled Fourier-path C with
    galaxy.py's geometry.  Returns (7 x pix*components, seconds, sources)."""
    i0, i1, use_ref, budget = args
    sys.path.insert(0, ROOT)
    os.environ.setdefault('OMP_NUM_THREADS', '1')
    from oracle import oracle as O
    from tractor_b200 import batch
    srcs = deriv_sources()
    psf = batch.moffat_psf()
    kern = O.reference_kernels() if use_ref else None
    cdinv = O.nullwcs_cdinv()
    work, done = 0., 0
    t0 = time.perf_counter()
    for i in range(i0, i1):
        s = srcs[i]
        m = int(s['mw'])
        th = [float(s['s0']), float(s['s1']), float(s['s2']), float(s['sersic_n'])]
        for j in range(5):
            t = list(th)
            if j > 0:
                t[j - 1] += 0.01
            amp, var = O.sersic_profile(t[3])
            T = cdinv @ O.ellipseE_basis(t[0], t[1], t[2])
            a2, v2 = O.sheared(amp, var, T)
            _, (_, _, _, _, sz) = O.galaxy_fft_masked(a2, v2, s['px'], s['py'], psf, 0, 0, m, m,
                                                      kernels=kern)
            if j == 0:
                work += 7. * sz * sz * len(amp)
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    return work, time.perf_counter() - t0, done


def bench_derivs(args, dev, flush, clk, cpu_seconds):
    """All seven analytic derivative columns (x, y, counts, r_e, e1, e2, n)
    of 256 Sersic galaxies on 32-128 px masks (FFT 64-256): Jacobian through
    tb_galaxy_fft_jac_prep + tb_fourier_render_deriv (one launch of 7 x 256
    derivative items), and the fused vector-Jacobian product (TB_FFT_DOT).
    Metric: Mpix x components / s with every column counted as a render."""
    import ctypes
    import torch
    from tractor_b200 import batch, grad, _lib, render
    srcs = deriv_sources()
    n = len(srcs)
    npix = int((srcs['out_off'] + srcs['mw'].astype(np.int64) * srcs['mh']).max())
    r = batch.FourierGalaxyRenderer(batch.moffat_psf())
    jac = grad.FourierJacobian(r)
    h_src = torch.from_numpy(srcs.view(np.uint8).copy()).pin_memory()
    d_src = h_src.to(dev)
    out = torch.empty(7 * npix, dtype=torch.float32, device=dev)
    upstream = torch.randn(npix, generator=torch.Generator(device=dev).manual_seed(7),
                           device=dev, dtype=torch.float32)
    dots = torch.zeros(7 * n, dtype=torch.float64, device=dev)
    for _ in range(max(3, args.warmup)):
        jac._run(d_src, n, out, _lib.MOG_STORE, npix)
        jac._run(d_src, n, upstream, _lib.FFT_DOT, 0, dots=dots)
    torch.cuda.synchronize()
    flags = jac._work(n)[4].cpu().numpy()
    assert np.all(flags == 0), 'jac prep flagged sources: %s' % np.unique(flags)
    items = jac._work(n)[0].cpu().numpy().view(_lib.FFT_ITEM)
    pixcomp = float(np.sum(items['sz'].astype(np.float64) ** 2 * items['K']))   # 7 columns
    ex2 = float(np.sum(items['sz'].astype(np.float64) * (items['sz'] // 2 + 1) * items['K']))
    steps = max(5, min(args.steps, 20))
    lib = _lib.load()
    it_t, camp, cvar, dcoef, flg, misc = jac._work(n)

    def timed(mode, o, dts):
        tt, kt = [], []
        for _ in range(steps):
            flush.zero_()
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record()
            rc = lib.tb_galaxy_fft_jac_prep(d_src.data_ptr(), n, ctypes.addressof(r.image),
                                            ctypes.addressof(r.tables.struct), it_t.data_ptr(),
                                            camp.data_ptr(), cvar.data_ptr(), dcoef.data_ptr(),
                                            batch.COMP_STRIDE, mode,
                                            npix if mode == _lib.MOG_STORE else 0,
                                            flg.data_ptr(), _lib.stream_ptr())
            _lib.check(rc, 'tb_galaxy_fft_jac_prep')
            e[1].record()
            render.fourier_render(it_t.data_ptr(), 7 * n, camp.data_ptr(), cvar.data_ptr(),
                                  r.spec.data_ptr(), o.data_ptr(), misc.data_ptr() + 16,
                                  dcoef_ptr=dcoef.data_ptr(),
                                  dots_ptr=None if dts is None else dts.data_ptr())
            e[2].record()
            e[2].synchronize()
            tt.append(e[0].elapsed_time(e[2]) / 1e3)
            kt.append(e[1].elapsed_time(e[2]) / 1e3)
        return float(np.mean(tt)), float(np.mean(kt))

    jac_s, jac_k = timed(_lib.MOG_STORE, out, None)
    vjp_s, vjp_k = timed(_lib.FFT_DOT, upstream, dots)
    # end to end: records in from pinned memory, the Jacobian out
    h_out = torch.empty(7 * npix, dtype=torch.float32).pin_memory()
    e2e = []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        d_src.copy_(h_src, non_blocking=True)
        jac._run(d_src, n, out, _lib.MOG_STORE, npix)
        h_out.copy_(out, non_blocking=True)
        e1.record()
        e1.synchronize()
        e2e.append(e0.elapsed_time(e1) / 1e3)
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    peak_clk = clk['sm_mhz'] if clk else 1965.0
    peak = SFU_EX2_PER_CLK_PER_SM * nsm * peak_clk * 1e6 / 1e9
    line = {
        'name': 'C4 derivatives',
        'workload': 'C4: 7 analytic columns of 256 Sersic galaxies, masks 32-128 px, FFT 64-256',
        'metric': 'Mpix*components/s (7 derivative columns, each a render)',
        'value': pixcomp / jac_s / 1e6, 'unit': 'Mpix*components/s',
        'ms_per_step': jac_s * 1e3, 'steps': steps,
        'vjp_ms_per_step': vjp_s * 1e3, 'vjp_value': pixcomp / vjp_s / 1e6,
        'e2e': {'value': pixcomp / float(np.mean(e2e)) / 1e6, 'unit': 'Mpix*components/s',
                'h2d_bytes_per_step': int(h_src.numel()),
                'd2h_bytes_per_step': int(h_out.numel() * 4)},
        'gpu_launches_per_step': 2 + 2 * (-(-7 * n // 256)),
        'roofline': {'bound': 'sfu', 'kernel': 'tb_fourier_render_split (Jacobian items)',
                     'achieved': ex2 / jac_k / 1e9, 'peak': peak, 'unit': 'Gex2/s',
                     'frac': ex2 / jac_k / 1e9 / peak, 'kernel_ms': jac_k * 1e3,
                     'algorithmic': '%.0f ex2 per launch' % ex2,
                     'traffic': ncu_traffic('fourier_deriv_c4.json')},
    }
    if cpu_seconds:
        ncores = os.cpu_count() or 1
        from oracle import oracle as O
        use_ref = O.reference_kernels() is not None
        per = max(1, n // ncores)
        tasks = [((c * per) % n, min(n, (c * per) % n + per), use_ref, cpu_seconds)
                 for c in range(ncores)]
        with mp.get_context('spawn').Pool(ncores) as pool:
            res = pool.map(_deriv_cpu_worker, tasks)
        work = sum(x[0] for x in res)
        busy = max(x[1] for x in res)
        line['cpu_baseline'] = {'value': work / busy / 1e6, 'unit': 'Mpix*components/s',
                                'cores': ncores, 'kind': 'reference' if use_ref else 'port',
                                'sample': '%d sources, 5 finite-difference renders each' %
                                          sum(x[2] for x in res)}
    return line


# ---------------------------------------------------------------------------
# secondary workload: dense normal equations on the tensor cores
# ---------------------------------------------------------------------------

NE_PROBLEMS, NE_P, NE_R = 512, 63, 16384


def _ne_call(lib, A, r, meta, AtA, Atr, n, max_p, stream):
    from tractor_b200 import _lib
    return lib.tb_normal_equations(A.data_ptr(), r.data_ptr(), *[m.data_ptr() for m in meta],
                                   AtA.data_ptr(), Atr.data_ptr(), n, max_p,
                                   _lib.stream_ptr(stream))


def bench_normal_equations(args, dev, flush, clk, cpu_seconds):
    """tb_normal_equations (A^T A and A^T r of many independent least-squares
    problems, the LsqrOptimizer step) on NE_PROBLEMS problems of NE_P
    parameters x NE_R pixel rows, FP32 column-major in HBM (2.1 GB, above L2):
    problems per second, device-timed and end to end from pinned host memory,
    HBM roofline of the tensor-core kernel, the CUDA-core kernel the library
    keeps for P > 255 timed on the same problems, and numpy FP64 on the host."""
    import torch
    from tractor_b200 import _lib
    lib = _lib.load()
    n, P, R = (args.ne_problems or NE_PROBLEMS), NE_P, NE_R
    g = torch.Generator(device=dev).manual_seed(4000)
    A = torch.randn(n * P * R, device=dev, generator=g)
    r = torch.randn(n * R, device=dev, generator=g)
    t = lambda a, dt: torch.as_tensor(np.asarray(a, dt), device=dev)  # noqa: E731
    meta = [t(np.arange(n) * P * R, np.int64), t(np.arange(n) * R, np.int64), t([R] * n, np.int32),
            t([P] * n, np.int32), t([R] * n, np.int32), t(np.arange(n) * P * P, np.int64),
            t(np.arange(n) * P, np.int64)]
    AtA = torch.empty(n * P * P, dtype=torch.float64, device=dev)
    Atr = torch.empty(n * P, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()

    def timed(max_p, steps):
        for _ in range(3):
            _lib.check(_ne_call(lib, A, r, meta, AtA, Atr, n, max_p, stream), 'tb_normal_equations')
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _ne_call(lib, A, r, meta, AtA, Atr, n, max_p, stream)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        return float(np.mean(ts))

    steps = max(3, min(args.steps, 20))
    tc_s = timed(P, steps)
    # accuracy of the timed results against FP64 on a few problems
    err = 0.
    for q in (0, n // 2, n - 1):
        Aq = A[q * P * R:(q + 1) * P * R].view(P, R).double()
        ref = (Aq @ Aq.T).cpu().numpy()
        d = np.sqrt(np.diag(ref))
        got = AtA[q * P * P:(q + 1) * P * P].view(P, P).cpu().numpy()
        err = max(err, float((np.abs(got - ref) / np.outer(d, d)).max()))
    simt_s = timed(300, 3)   # max_p above 255 selects the CUDA-core kernel
    in_bytes = float(n * (P + 1) * R * 4)
    out_bytes = float(n * (P * P + P) * 8)
    achieved = (in_bytes + out_bytes) / tc_s / 1e9
    peak, peak_kind = measured_hbm_peak()
    # end to end: the problems copied in from pinned host memory, results out
    h_A = A.cpu().pin_memory()
    h_r = r.cpu().pin_memory()
    h_AtA = torch.empty(AtA.shape, dtype=AtA.dtype).pin_memory()
    h_Atr = torch.empty(Atr.shape, dtype=Atr.dtype).pin_memory()
    e2e = []
    for _ in range(max(2, min(steps, 3))):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        A.copy_(h_A, non_blocking=True)
        r.copy_(h_r, non_blocking=True)
        _ne_call(lib, A, r, meta, AtA, Atr, n, P, stream)
        h_AtA.copy_(AtA, non_blocking=True)
        h_Atr.copy_(Atr, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        e2e.append(e0.elapsed_time(e1) / 1e3)
    line = {
        'workload': '%d least-squares problems x %d parameters x %d pixel rows, FP32 '
                    'column-major (A^T A, A^T r in FP64)' % (n, P, R),
        'metric': 'normal-equation problems/s (tb_normal_equations)',
        'value': n / tc_s, 'unit': 'problems/s', 'ms_per_step': tc_s * 1e3, 'steps': steps,
        'max_scaled_error_vs_fp64': err,
        'cuda_core_kernel': {'ms_per_step': simt_s * 1e3, 'value': n / simt_s,
                             'speedup_tensor_cores': simt_s / tc_s},
        'e2e': {'value': n / float(np.mean(e2e)), 'unit': 'problems/s',
                'h2d_bytes_per_step': int(in_bytes), 'd2h_bytes_per_step': int(out_bytes)},
        'roofline': {'bound': 'hbm', 'kernel': 'normal_eq_tc64_kernel (tcgen05 kind::tf32, P <= 63)',
                     'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                     'frac': achieved / peak, 'peak_basis': peak_kind,
                     'algorithmic': '%d x (%d + 1) x %d x 4 bytes read + %d x (%d^2 + %d) x 8 '
                                    'bytes written per launch' % (n, P, R, n, P, P),
                     'kernel_ms': tc_s * 1e3,
                     'traffic': ncu_traffic('normal_eq_tc.json')},
    }
    if cpu_seconds:
        An = A[:P * R].view(P, R).cpu().numpy().astype(np.float64)
        rn = r[:R].cpu().numpy().astype(np.float64)
        t0 = time.time()
        done = 0
        while time.time() - t0 < cpu_seconds and done < n:
            _ = An @ An.T, An @ rn
            done += 1
        rate = done / (time.time() - t0)
        line['cpu_baseline'] = {'value': rate, 'unit': 'problems/s',
                                'cores': os.cpu_count() or 1, 'kind': 'port',
                                'sample': '%d problems, numpy FP64 A^T A and A^T r (BLAS, all '
                                          'host threads)' % done}
    return line


def _plain_small_setup(T):
    psf = T.NCircularGaussianPSF([1.5, 3.0], [0.8, 0.2])
    truth = T.ExpGalaxy(T.PixPos(32., 32.), T.Flux(1000.), T.EllipseE.fromRAbPhi(2.0, 0.6, 30.))
    tim = T.Image(data=np.zeros((64, 64)), invvar=np.ones((64, 64)), psf=psf,
                  photocal=T.LinearPhotoCal(1.))
    trc = T.Tractor([tim], [truth])
    trc.modtype = np.float64
    clean = trc.getModelImage(0)
    tim.data = clean + np.random.default_rng(300).normal(size=clean.shape)
    start = [32.5, 32.5, 800.] + list(T.EllipseE.fromRAbPhi(2.4, 0.6, 30.).getAllParams())
    src = T.ExpGalaxy(T.PixPos(32.5, 32.5), T.Flux(800.), T.EllipseE.fromRAbPhi(2.4, 0.6, 30.))
    tr = T.Tractor([tim], [src])
    tr.modtype = np.float64
    tr.freezeParam('images')
    return tr, start


def _plain_small_time(T, reps, fits):
    tr, start = _plain_small_setup(T)
    for _ in range(3):
        tr.getModelImage(0)
    t0 = time.perf_counter()
    for _ in range(reps):
        tr.getModelImage(0)
    render_us = (time.perf_counter() - t0) / reps * 1e6
    times, steps = [], 0
    for _ in range(fits):
        tr.setParams(start)
        t0 = time.perf_counter()
        R = tr.optimize_loop(dchisq=1e-3)
        times.append(time.perf_counter() - t0)
        steps = R['steps']
    return render_us, times, steps


class _SetAttr(object):
    """The one method of a monkeypatch that oracle.host_kernels.install uses."""

    @staticmethod
    def setattr(obj, name, value):
        setattr(obj, name, value)


def _plain_small_cpu_worker(_):
    """The small plain fit on the host: the same object API with every kernel
    computed by the oracle (C / numpy), one core."""
    sys.path.insert(0, ROOT)
    os.environ.setdefault('OMP_NUM_THREADS', '1')
    from oracle import host_kernels
    host_kernels.install(_SetAttr())
    import tractor_b200 as T
    render_us, times, steps = _plain_small_time(T, reps=20, fits=2)
    return render_us, float(np.median(times)), steps


def bench_plain_small(args, dev, cpu_seconds=None):
    """The small plain fit through the object API (an ExpGalaxy, r_e 2 px, b/a
    0.6, phi 30, flux 1000, at the centre of a 64 x 64 FP64 image, two-
    Gaussian PSF with sigma 1.5 / 3.0 and weights 0.8 / 0.2, noise sigma 1
    drawn from seed 300; start off by 0.5 px and 20 % in flux and r_e):
    microseconds per Tractor.getModelImage and milliseconds per
    optimize_loop(dchisq=1e-3) with B200Optimizer, host timed (each call
    returns host arrays: copies and launches included).  The case is
    latency-bound (49k pixel x components per render): no roofline.  CPU
    baseline: the same calls with the oracle's kernels on one host core."""
    import tractor_b200 as T
    render_us, times, steps = _plain_small_time(T, reps=50,
                                                fits=max(2, min(args.steps, 3)) + 1)
    fit_s = float(np.median(times[1:]))
    line = {'workload': 'C1: ExpGalaxy on 64x64, 2-Gaussian PSF, optimize_loop(dchisq=1e-3)',
            'metric': 'fitted sources/s (plain small fit, object API)',
            'value': 1.0 / fit_s, 'unit': 'sources/s', 'ms_per_step': fit_s * 1e3,
            'ms_per_fit': fit_s * 1e3, 'steps_per_fit': steps, 'us_per_render': render_us,
            'timing': 'host wall clock per call (launches, copies and host logic included)',
            'roofline': None,
            'summary': {'us_render': render_us, 'steps': steps}}
    if cpu_seconds:
        with mp.get_context('spawn').Pool(1) as pool:
            cr_us, cfit_s, csteps = pool.map(_plain_small_cpu_worker, [0])[0]
        line['cpu_baseline'] = {'value': 1.0 / cfit_s, 'unit': 'sources/s', 'cores': 1,
                                'kind': 'port',
                                'sample': 'the same fit (%d steps) and 20 renders with the '
                                          'oracle kernels on the host: %.1f ms per fit, %.0f us '
                                          'per render' % (csteps, cfit_s * 1e3, cr_us)}
        line['summary']['cpu_us_render'] = cr_us
    return line


# secondary workload: EM fits of PSF stamps (GaussianMixturePSF.fromStamp)
EM_STAMPS, EM_SIDE, EM_K, EM_STEPS = 4096, 25, 3, 1000
FP64_NOMINAL_TFLOPS = 40.0     # B200 FP64 (non-tensor), nominal: no measured figure


def em_stamps(n, seed=900):
    """Seeded 25 x 25 PSF stamps: two concentric Gaussians (sigma s and 2.5 s,
    s U[1, 2], weights 0.7 / 0.3, centre offset U[-0.5, 0.5] px) plus noise
    of 1e-5 of the total, normalised and clipped at 0 as fromStamp does."""
    rng = np.random.default_rng(seed)
    h = EM_SIDE // 2
    y, x = np.mgrid[:EM_SIDE, :EM_SIDE] - float(h)
    out = np.empty((n, EM_SIDE, EM_SIDE))
    for i in range(n):
        s = rng.uniform(1., 2.)
        cx, cy = rng.uniform(-0.5, 0.5, 2)
        r2 = (x - cx) ** 2 + (y - cy) ** 2
        im = 0.7 * np.exp(-r2 / (2 * s * s)) + 0.3 * np.exp(-r2 / (2 * (2.5 * s) ** 2))
        im = im / im.sum() + rng.normal(0., 1e-5, im.shape)
        out[i] = np.maximum(im / im.sum(), 0.)
    return out


def bench_emfit(args, dev, flush, clk, cpu_seconds):
    """EM fits of 3-Gaussian mixtures to 4,096 PSF stamps of 25 x 25 pixels,
    1,000 iterations each (GaussianMixturePSF.fromStamp's em_fit_2d_reg,
    FP64): device-resident launches of tb_em_fit_2d timed with CUDA events,
    and end to end through tractor_b200.emfit.em_fit_2d_batch from host
    arrays.  CPU baseline: the reference's own em_fit_2d_reg (compiled from
    tractor/emfit.i into oracle/_ref) on a bounded sample, one core."""
    import torch
    from tractor_b200 import _lib, emfit
    lib = _lib.load()
    n, K = EM_STAMPS, EM_K
    imgs = em_stamps(n)
    w, mu, var = emfit.em_init_params(K, None, None, None)
    A0 = np.ascontiguousarray(np.broadcast_to(w, (n, K)))
    M0 = np.ascontiguousarray(np.broadcast_to(mu, (n, K, 2)))
    V0 = np.ascontiguousarray(np.broadcast_to(var, (n, K, 2, 2)))
    d_img = torch.from_numpy(imgs).to(dev)
    init = [torch.from_numpy(a).to(dev) for a in (A0, M0, V0)]
    work = [t.clone() for t in init]
    d_st = torch.zeros(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()

    def launch():
        for t, t0 in zip(work, init):
            t.copy_(t0)
        rc = lib.tb_em_fit_2d(d_img.data_ptr(), n, EM_SIDE, EM_SIDE, None, work[0].data_ptr(),
                              work[1].data_ptr(), work[2].data_ptr(), K, 0., EM_STEPS,
                              d_st.data_ptr(), stream.cuda_stream)
        assert rc == 0
    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize()
    ts = []
    for _ in range(args.steps):
        flush.fill_(1.)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        launch()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) / 1e3)
    kern_s = float(np.median(ts))
    fails = int(d_st.sum().item())
    value = n / kern_s
    # end to end: host stamps and initial mixtures in, fitted mixtures out
    emfit.em_fit_2d_batch(imgs[:64], A0[:64], M0[:64], V0[:64], 0., EM_STEPS)
    e2e_t = []
    for _ in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        emfit.em_fit_2d_batch(imgs, A0, M0, V0, 0., EM_STEPS)
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = float(np.median(e2e_t))
    units = float(n) * EM_SIDE * EM_SIDE * K * EM_STEPS
    flops_per_unit = 30   # dx, dy, dsq (10), scale x exp, sum, z / zsum, w, 6 moments (11)
    achieved = units * flops_per_unit / kern_s / 1e12
    cpu = None
    if cpu_seconds:
        try:
            from oracle import refharness
            ref = refharness._emfit_module()
            kind, fit = 'reference', ref.em_fit_2d_reg
        except Exception:
            from oracle import oracle as O
            kind, fit = 'port', O.em_fit_2d_reg
        done, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < cpu_seconds and done < n:
            a, m_, v = A0[done].copy(), M0[done].copy(), V0[done].copy()
            fit(imgs[done], -(EM_SIDE // 2), -(EM_SIDE // 2), a, m_, v, 0., EM_STEPS)
            done += 1
        cpu = {'value': done / (time.perf_counter() - t0), 'unit': 'stamps/s', 'cores': 1,
               'kind': kind,
               'sample': '%d of the %d stamps, em_fit_2d_reg one after another, %.0f s budget'
                         % (done, n, cpu_seconds)}
    return {'workload': '%d PSF stamps of %dx%d px, %d-Gaussian EM fit, %d iterations '
                        '(GaussianMixturePSF.fromStamp / em_fit_2d_reg), FP64'
                        % (n, EM_SIDE, EM_SIDE, K, EM_STEPS),
            'metric': 'PSF stamps fitted/s', 'value': value, 'unit': 'stamps/s',
            'ms_per_step': kern_s * 1e3, 'failed_fits': fails,
            'e2e': {'value': n / e2e_s, 'unit': 'stamps/s',
                    'h2d_bytes_per_step': int(imgs.nbytes + A0.nbytes + M0.nbytes + V0.nbytes),
                    'd2h_bytes_per_step': int(A0.nbytes + M0.nbytes + V0.nbytes + 4 * n)},
            'gpu_launches_per_step': 1,
            'roofline': {'bound': 'fp64', 'kernel': 'tb_em_fit_2d',
                         'achieved': achieved, 'peak': FP64_NOMINAL_TFLOPS, 'unit': 'TFLOP/s',
                         'frac': achieved / FP64_NOMINAL_TFLOPS,
                         'peak_basis': 'nominal B200 FP64 (no measured FP64 peak on this pool)',
                         'algorithmic': '%.3g pixel x component x iterations x %d FP64 flops '
                                        '(exp not counted)' % (units, flops_per_unit),
                         'traffic': ncu_traffic('emfit_psf_stamps.json'),
                         'note': 'FP64-pipe and dependency-latency bound (FP64 exp per pixel x '
                                 'component); the stamps stay on chip'},
            'cpu_baseline': cpu}


# secondary workload: blob segmentation of a detection map
SEG_SIDE = 4096


def seg_map(seed=950):
    """A seeded 4096 x 4096 detection map: white noise smoothed by a
    Gaussian of sigma 4 px, thresholded at 0.02 (about 11k blobs, 40 % of
    the pixels set), and 20,000 source positions drawn on it."""
    import scipy.ndimage as ndi
    rng = np.random.default_rng(seed)
    f = ndi.gaussian_filter(rng.normal(size=(SEG_SIDE, SEG_SIDE)).astype(np.float32), 4)
    pos = rng.uniform(0, SEG_SIDE - 1, (20000, 2))
    return f > 0.02, pos


def bench_segment(args, dev, flush, clk, cpu_seconds):
    """Blob segmentation (tractor_b200.blobs): connected components of a
    4096 x 4096 detection map with scipy.ndimage.label's numbering and their
    boxes, device-resident launches timed with CUDA events; end to end
    through blobs.segment from the host map (plus 20,000 source positions
    assigned to blobs).  CPU baseline: scipy.ndimage.label + find_objects
    (the tool the reference's callers use) on the same map, one core."""
    import torch
    import scipy.ndimage as ndi
    from tractor_b200 import _lib, blobs
    lib = _lib.load()
    det, pos = seg_map()
    H = W = SEG_SIDE
    d_mask = torch.from_numpy(det.astype(np.uint8)).to(dev)
    labels, n = blobs._label_device(d_mask, H, W, 0)
    nbytes = int(lib.tb_label_workspace_bytes(H, W))
    ws = torch.empty((nbytes + 15) // 16 * 4, dtype=torch.int32, device=dev)
    scal = torch.zeros(2, dtype=torch.int32, device=dev)
    boxes = torch.empty((n, 4), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()

    def launch():
        assert lib.tb_label_components(d_mask.data_ptr(), H, W, 0, labels.data_ptr(),
                                       scal.data_ptr(), ws.data_ptr(), scal.data_ptr() + 4,
                                       stream.cuda_stream) == 0
        assert lib.tb_component_boxes(labels.data_ptr(), H, W, n, boxes.data_ptr(),
                                      stream.cuda_stream) == 0
    for _ in range(args.warmup):
        launch()
    torch.cuda.synchronize()
    ts = []
    for _ in range(args.steps):
        flush.fill_(1.)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        launch()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) / 1e3)
    kern_s = float(np.median(ts))
    assert int(scal[0].item()) == n and int(scal[1].item()) == 0
    blobs.segment(det[:256, :256])
    e2e_t = []
    for _ in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        seg = blobs.segment(det, pos)
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = float(np.median(e2e_t))
    assert seg.n == n
    cpu = None
    if cpu_seconds:
        t0 = time.perf_counter()
        reps = 0
        while reps == 0 or time.perf_counter() - t0 < min(cpu_seconds, 2.0):
            ref, nr = ndi.label(det)
            ndi.find_objects(ref)
            reps += 1
        cpu_s = (time.perf_counter() - t0) / reps
        assert nr == n
        cpu = {'value': H * W / cpu_s / 1e6, 'unit': 'Mpix/s', 'cores': 1, 'kind': 'port',
               'sample': 'the whole map, scipy.ndimage.label + find_objects (the checker of the '
                         'tests), %d runs' % reps}
    peak, basis = measured_hbm_peak()
    alg_bytes = H * W * (1 + 4)
    achieved = alg_bytes / kern_s / 1e9
    return {'workload': '4096x4096 detection map (smoothed noise > 0.02, %d blobs), 4-connected '
                        'components with scipy.ndimage.label numbering + bounding boxes' % n,
            'metric': 'Mpix/s segmented (blob labelling + boxes)',
            'value': H * W / kern_s / 1e6, 'unit': 'Mpix/s', 'ms_per_step': kern_s * 1e3,
            'n_blobs': n,
            'e2e': {'value': H * W / e2e_s / 1e6, 'unit': 'Mpix/s',
                    'h2d_bytes_per_step': int(H * W), 'd2h_bytes_per_step': int(H * W * 4 + n * 16)},
            'gpu_launches_per_step': 9,
            'roofline': {'bound': 'hbm', 'kernel': 'tb_label_components + tb_component_boxes',
                         'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                         'frac': achieved / peak, 'peak_basis': basis,
                         'algorithmic': '1 byte read + 4 bytes written per pixel',
                         'traffic': None,
                         'note': 'latency / atomics bound: union-find merges chase parent '
                                 'chains; 9 launches per step'},
            'cpu_baseline': cpu}


def measured_hbm_peak():
    """The pool's measured copy bandwidth (GB/s) and where it came from."""
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(p) as f:
            d = json.load(f)
        if 'hbm_gbs' in d:
            return float(d['hbm_gbs']), 'measured copy bandwidth (MEASURED_PEAKS.json hbm_gbs)'
    except (OSError, ValueError):
        pass
    return 6650.0, 'fallback 6.65 TB/s'


def fit_plain_fp64(w, data, inv, batched, status, dev, budget):
    """The plain FP64 GPU fitter (tractor_b200.plain.BlobFitFP64: one blob at
    a time, FP64 torch / cuSOLVER) on the workload's first blobs for about
    `budget` seconds: fitted sources / s from the perturbed start (same
    stopping rule, predicted dlnp < 1e-3).  Parity: for those blobs that the
    batched fitter converged, the FP64 optimum (the FP64 fitter continued
    from the batched result to a predicted gain of 1e-10) and the batched
    parameters' distance from it in units of the FP64 sigma."""
    import torch
    from tractor_b200 import fit, plain
    po = fit.pix_offsets(w['sides'], 3)
    hd, hi = data.cpu().numpy(), inv.cpu().numpy()
    done, blobs = 0, 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    fits = []
    for b in range(len(w['sides'])):
        s0, s1 = w['blob_src'][b], w['blob_src'][b + 1]
        W, H = (int(v) for v in w['sides'][b])
        d3 = np.stack([hd[po[3 * b + k]:po[3 * b + k + 1]].reshape(H, W) for k in range(3)])
        i3 = np.stack([hi[po[3 * b + k]:po[3 * b + k + 1]].reshape(H, W) for k in range(3)])
        rects = [tuple(int(v) for v in (r['x0'], r['y0'], r['w'], r['h']))
                 for r in w['sources'][s0:s1]]
        pf = plain.BlobFitFP64(d3, i3, w['psf'][b], rects, dev)
        pf.fit(w['start'][s0:s1], tol=1e-3)
        fits.append((b, pf, s0, s1))
        done += s1 - s0
        blobs += 1
        if time.perf_counter() - t0 > budget:
            break
    e1.record()
    e1.synchronize()
    secs = e0.elapsed_time(e1) / 1e3
    # parity: 120 blobs spread over the workload, and every blob that
    # stopped by rejections (status 2) or at the iteration limit (status 3)
    n_b = len(status)
    pick = np.linspace(0, n_b - 1, min(120, n_b)).astype(int)
    pick = np.union1d(pick, np.flatnonzero(status >= 2))
    res = plain.optimum_distance(w, data, inv, batched, status, pick, dev)
    inner = [r[0] for r in res if not r[3] and r[4]]
    edge = [r[0] for r in res if r[3]]
    flat = [r[0] for r in res if not r[3] and not r[4]]
    limit = [r for r in res if r[2] == 3]
    return {'value': done / secs, 'unit': 'sources/s', 'blobs': blobs, 'sources': int(done),
            'seconds': secs, 'parity_blobs': len(res),
            'batched_vs_fp64_optimum_max_sigma': float(np.max(inner)) if inner else None,
            'batched_vs_fp64_optimum_median_sigma': float(np.median(inner)) if inner else None,
            'edge_blobs': len(edge),
            'edge_max_sigma': float(np.max(edge)) if edge else None,
            'flat_blobs': len(flat),
            'flat_max_sigma': float(np.max(flat)) if flat else None,
            'limit_blobs': len(limit),
            'limit_max_sigma': float(np.max([r[0] for r in limit])) if limit else None,
            'limit_inner_max_sigma': (float(np.max([r[0] for r in limit if not r[3] and r[4]]))
                                      if any(not r[3] and r[4] for r in limit) else None),
            'how': 'tractor_b200.plain.BlobFitFP64 (FP64 torch ops + cuSOLVER, one blob at a '
                   'time, same GPU) from the start for the rate; continued from the batched '
                   'result to predicted dlnp 1e-10 for the FP64 optimum; sigma from its FP64 '
                   'Fisher matrix; edge blobs have a Sersic index within 1e-3 of a profile '
                   'range edge, where the mixture tables change and the model jumps; flat '
                   'blobs are those the FP64 fitter itself does not converge on within 100 '
                   'iterations; the parity set is 120 blobs spread over the workload plus '
                   'every blob that stopped by rejections near its optimum or at the iteration '
                   'limit (limit_*: those at the limit alone)'}


def fit_ncomp(n):
    """Galaxy components of a Sersic mixture at index n (the spline range's
    count, plus the core for n > 1)."""
    from tractor_b200 import profiles
    S = profiles.tables()['sersic']
    for r in S['ranges']:
        if r['lo'] <= n < r['hi']:
            return r['K'] + (1 if n > 1 else 0)
    return S['ranges'][-1]['K'] + 1


# ---------------------------------------------------------------------------

def init_dist():
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    return world, rank, local


def ncu_traffic(name='fourier_render_c2.json'):
    """DRAM bytes per launch of a workload's top kernel, from its committed
    ncu summary under profiles/, or None."""
    p = os.path.join(ROOT, 'profiles', name)
    try:
        with open(p) as f:
            return json.load(f).get('dram_bytes_per_launch')
    except (OSError, ValueError):
        return None


def run_reference(args, world, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    use_ref = O.reference_kernels() is not None
    kind = 'reference' if use_ref else 'port'
    ncores = os.cpu_count() or 1
    per_step = max(8.0, 60.0 / max(1, args.steps + args.warmup))
    for _ in range(args.warmup):
        cpu_rate(min(per_step, 2.0), use_ref)
    rates, nsrc = [], 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r, ncores, n, _ = cpu_rate(per_step, use_ref)
        rates.append(r)
        nsrc += n
    wall = time.perf_counter() - t0
    value = float(np.mean(rates))
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': 'Mpix*components/s',
        'n_gpus': 0, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': wall / max(1, args.steps) * 1e3, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64/f32 (reference CPU path)',
        'data': 'synthetic', 'config': config_keys(),   # the same keys as the GPU arm
        'cpu_baseline': {'value': value, 'unit': 'Mpix*components/s', 'cores': ncores,
                         'kind': kind,
                         'sample': '%d source renders over %d steps (%.0f s budget per step), '
                                   'one process per core' % (nsrc, args.steps, per_step)},
        'e2e': {'value': value, 'unit': 'Mpix*components/s', 'h2d_bytes_per_step': 0,
                'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


def run_secondaries(args, dev, flush, clk, cpu_s, rank):
    """Runs the secondary measurements (all, or those --only names); each
    full record goes to stderr, the returned dict holds their summaries."""
    runs = [('C3', lambda: bench_scene(args, dev, flush, clk, cpu_s)),
            ('C5', lambda: bench_fit(args, dev, flush, clk, cpu_s)),
            ('C4', lambda: bench_derivs(args, dev, flush, clk, cpu_s and min(cpu_s, 6.0))),
            ('K5', lambda: bench_normal_equations(
                args, dev, flush, clk, cpu_s and min(cpu_s, 4.0))),
            ('C1', lambda: bench_plain_small(args, dev, cpu_s and min(cpu_s, 6.0))),
            ('EM', lambda: bench_emfit(args, dev, flush, clk, cpu_s and min(cpu_s, 4.0))),
            ('SEG', lambda: bench_segment(args, dev, flush, clk, cpu_s))]
    if args.only:
        runs = [r for r in runs if r[0] in args.only.split(',')]
    secondary = {}
    for name, run in runs:
        # a secondary line that fails is reported in the line, not fatal
        try:
            full = run()
        except Exception as e:   # noqa: BLE001
            full = {'error': repr(e)[:300]}
        full['name'] = name
        if rank == 0:
            # the full record on stderr; the main line carries a summary
            print(json.dumps(full), file=sys.stderr, flush=True)
        secondary[name] = compact(full)
    return secondary


def main():
    args = parse()
    world, rank, local = init_dist()
    if args.impl == 'reference':
        if world > 1:
            import torch.distributed as dist  # noqa: F401
        run_reference(args, world, rank)
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group('nccl', init_method='env://',
                                timeout=__import__('datetime').timedelta(seconds=120))
    torch.cuda.set_device(local)
    from tractor_b200 import batch, _lib, build
    build.build()
    _lib.load()

    if args.secondary_only:
        dev = torch.device('cuda', local)
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
        cpu_s = None if (args.no_cpu_baseline or world > 1 or rank) else min(args.cpu_seconds, 8.0)
        secondary = run_secondaries(args, dev, flush, None, cpu_s, rank)
        if rank == 0:
            print(json.dumps({'metric': METRIC, 'secondary_only': True, 'secondary': secondary}),
                  flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    # one global workload of 256 sources per GPU, cost-balanced over the
    # ranks (tractor_b200.shard); each rank renders its share
    from tractor_b200 import shard
    all_srcs = batch.sersic_sources(N_SOURCES * world, np.random.default_rng(1000), mask=MASK)
    own = np.flatnonzero(shard.balance(shard.fourier_costs(all_srcs), world) == rank)
    srcs = all_srcs[own].copy()
    srcs['out_off'] = np.arange(len(srcs), dtype=np.int64) * MASK * MASK
    renderer = batch.FourierGalaxyRenderer(batch.moffat_psf())
    n = len(srcs)
    nout = n * MASK * MASK
    dev = torch.device('cuda', local)
    src_pinned = torch.from_numpy(srcs.view(np.uint8).copy()).pin_memory()
    d_src = src_pinned.to(dev)
    out = torch.empty(nout, dtype=torch.float32, device=dev)
    out_pinned = torch.empty(nout, dtype=torch.float32).pin_memory()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MB > L2
    stream = torch.cuda.current_stream()

    def step():
        renderer.render_device(d_src, n, out)

    # the fastest Fourier method on this workload (fused prep + render, or
    # prep then the persistent or split render), unless one is asked for
    from tractor_b200 import render as R
    if args.fourier_method == 'auto':
        tune = renderer.autotune(d_src, n, out)
    else:
        tune = {}
        renderer.method = args.fourier_method
    method = renderer.method
    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    flags = renderer._work(n)[3].cpu().numpy()
    items = renderer._work(n)[0].cpu().numpy().view(_lib.FFT_ITEM)
    assert np.all(flags == 0), 'prep flagged sources: %s' % np.unique(flags)
    pixcomp = float(np.sum(items['sz'].astype(np.float64) ** 2 * items['K']))
    ex2_per_launch = float(np.sum(items['sz'].astype(np.float64) * (items['sz'] // 2 + 1) *
                                  items['K']))

    # ---- device-timed steps (inputs resident in HBM, L2 flushed) ----
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    props = torch.cuda.get_device_properties(dev)
    try:
        gpu_id = '%08X:%02X:%02X.0' % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
    except AttributeError:
        gpu_id = str(torch.cuda.current_device())
    clocks = ClockSampler(gpu_id)
    clocks.start()
    time.sleep(0.3)
    # split: setup + column + row kernels per 256 items and the persistent
    # kernel for the items outside the split path; persistent: one launch
    # after the prep; fused: one launch in all
    launches_per_render = 3 * (-(-n // 256)) + 1 if method == 'split' else 1
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.zero_()
        e0, e1, e2 = ev[k]
        e0.record(stream)
        lib = _lib.load()
        items_t, camp, cvar, flg, misc = renderer._work(n)
        if method == 'fused':
            # preparation and render in one launch: the kernel is the step
            e1.record(stream)
            rc = lib.tb_galaxy_fft_render(d_src.data_ptr(), n,
                                          __import__('ctypes').addressof(renderer.image),
                                          __import__('ctypes').addressof(renderer.tables.struct),
                                          renderer.spec.data_ptr(), out.data_ptr(),
                                          items_t.data_ptr(), flg.data_ptr(), misc.data_ptr(),
                                          misc.data_ptr() + 16, _lib.stream_ptr())
            _lib.check(rc, 'tb_galaxy_fft_render')
        else:
            rc = lib.tb_galaxy_fft_prep(d_src.data_ptr(), n,
                                        __import__('ctypes').addressof(renderer.image),
                                        __import__('ctypes').addressof(renderer.tables.struct),
                                        items_t.data_ptr(), camp.data_ptr(), cvar.data_ptr(),
                                        batch.COMP_STRIDE, flg.data_ptr(), _lib.stream_ptr())
            _lib.check(rc, 'tb_galaxy_fft_prep')
            e1.record(stream)
            R.fourier_render(items_t.data_ptr(), n, camp.data_ptr(), cvar.data_ptr(),
                             renderer.spec.data_ptr(), out.data_ptr(), misc.data_ptr() + 16,
                             method=method)
        e2.record(stream)
    torch.cuda.synchronize()
    gpu_launches = ((0 if method == 'fused' else 1) + launches_per_render) * args.steps
    step_ms = [a.elapsed_time(c) for a, b, c in ev]
    render_ms = [b.elapsed_time(c) for a, b, c in ev]
    t_total = sum(step_ms) / 1e3
    if world > 1:
        t = torch.tensor([t_total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_total = float(t.item())

    # ---- end to end through the host-buffer API (H2D + render + D2H) ----
    # Double-buffered: step k's patches are copied to pinned host memory on a
    # copy stream while step k+1 renders into the other buffer; the timed
    # region runs from the first step's H2D to the last step's D2H.
    copy_stream = torch.cuda.Stream(dev)
    outs = [out, torch.empty_like(out)]
    pins = [out_pinned, torch.empty_like(out_pinned).pin_memory()]
    done = [torch.cuda.Event(), torch.cuda.Event()]
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e_start.record(stream)
    for k in range(args.steps):
        b = k % 2
        flush.zero_()
        d_src.copy_(src_pinned, non_blocking=True)
        if k >= 2:
            stream.wait_event(copied[b])
        renderer.render_device(d_src, n, outs[b])
        done[b].record(stream)
        copy_stream.wait_event(done[b])
        with torch.cuda.stream(copy_stream):
            pins[b].copy_(outs[b], non_blocking=True)
        copied[b].record(copy_stream)
    stream.wait_stream(copy_stream)
    e_end.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    e2e_s = e_start.elapsed_time(e_end) / 1e3
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    R.check_status(renderer.status(n).clone(), 'tb_galaxy_fft_render' if method == 'fused'
                   else 'tb_fourier_render')

    job_pixcomp = pixcomp
    gather_ms = None
    if world > 1:
        t = torch.tensor([pixcomp], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        job_pixcomp = float(t.item())
        # the job's one collective: every rank's patches gathered (fixed-size
        # rows, one per source) after the timed steps
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        full = shard.gather_units(out.view(len(srcs), MASK * MASK), own, len(all_srcs))
        g1.record(stream)
        torch.cuda.synchronize()
        gather_ms = g0.elapsed_time(g1)
        del full
    value = job_pixcomp * args.steps / t_total / 1e6
    e2e = job_pixcomp * args.steps / e2e_s / 1e6
    kern_s = float(np.mean(render_ms)) / 1e3
    sm_mhz = clk['sm_mhz'] if clk else None
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    peak_clk = sm_mhz if sm_mhz else 1965.0
    peak = SFU_EX2_PER_CLK_PER_SM * nsm * peak_clk * 1e6 / 1e9
    achieved = ex2_per_launch / kern_s / 1e9
    line = {
        'metric': METRIC, 'value': value, 'unit': 'Mpix*components/s', 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': t_total / args.steps * 1e3,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
        'data': 'synthetic (seeded)',
        'config': config_keys(),
        'pix_components_per_step': job_pixcomp,
        'parallelism': 'cost-balanced sources per GPU, one all-gather after the timed steps',
        'e2e': {'value': e2e, 'unit': 'Mpix*components/s',
                'h2d_bytes_per_step': int(src_pinned.numel()),
                'd2h_bytes_per_step': int(out_pinned.numel() * 4),
                'overlap': 'D2H of step k on a copy stream during step k+1'},
        'gpu_launches': gpu_launches,
        'fourier_method': {'chosen': method, 'ms': {k: _sig(v) for k, v in tune.items()}},
        'roofline': {'bound': 'sfu', 'kernel': {
                         'split': 'tb_fourier_render_split (setup + column + row kernels)',
                         'persistent': 'tb_fourier_render (persistent)',
                         'fused': 'tb_galaxy_fft_render (preparation + persistent render, '
                                  'one launch)'}[method],
                     'achieved': achieved, 'peak': peak, 'unit': 'Gex2/s',
                     'frac': achieved / peak,
                     'peak_basis': '%d ex2/clk/SM x %d SMs x %s MHz (median under load)'
                                   % (SFU_EX2_PER_CLK_PER_SM, nsm, peak_clk),
                     'algorithmic': '%.0f ex2 (K sz (sz/2+1) per source)' % ex2_per_launch,
                     'kernel_ms': kern_s * 1e3,
                     'traffic': ncu_traffic()},
        'clocks': clk,
    }
    if gather_ms is not None:
        line['gather_ms'] = gather_ms
    if not args.no_secondary:
        cpu_s = None if (args.no_cpu_baseline or world > 1 or rank) else min(args.cpu_seconds, 8.0)
        secondary = run_secondaries(args, dev, flush, clk, cpu_s, rank)
    # the FP64 comparison renderer: the parity check of the batched patches
    # (its rate is one galaxy per Python call, so no speed-up is derived)
    line['plain_fp64'] = fourier_plain_fp64(srcs, out, dev, budget=3.0)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, cores, nsrc, wall = cpu_rate(args.cpu_seconds, use_ref=False)
        line['cpu_baseline'] = {'value': rate, 'unit': 'Mpix*components/s', 'cores': cores,
                                'kind': 'port',
                                'sample': '%d of the 256 sources rendered by the oracle, one '
                                          'process per core, %.0f s budget' % (nsrc, args.cpu_seconds)}
    if not args.no_secondary:
        line['secondary'] = secondary      # last: the part a short tail of the line shows
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
