"""Multi-GPU partitioning (tractor_b200.shard) on the CPU: the cost
balancing, the row bands and, with two gloo ranks, that every partitioned
workload gathers to exactly the single-process result.  The per-rank compute
is the oracle's (the same functions the tests check the kernels against):
Fourier-path galaxies, a scene rendered in row bands, and blob fits.

This mirrors TractorMultiprocMixin._map (tractor/multiproc.py:4-160), the
reference's per-item mapping, with ranks in place of host processes."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as tmp


def test_balance_is_deterministic_and_even():
    from tractor_b200 import shard
    rng = np.random.default_rng(4)
    costs = rng.lognormal(0, 1, 500)
    for world in (1, 2, 3, 8):
        a = shard.balance(costs, world)
        assert np.array_equal(a, shard.balance(costs, world))
        assert a.min() >= 0 and a.max() < world
        load = np.bincount(a, weights=costs, minlength=world)
        # longest-processing-time bound: within one largest unit of the mean
        assert load.max() - costs.sum() / world <= costs.max() + 1e-9
    assert np.all(shard.balance(costs, 1) == 0)
    assert len(shard.balance([], 4)) == 0


def test_row_bands_cover_and_align():
    from tractor_b200 import shard
    for H, world in ((4096, 8), (4096, 3), (100, 4), (64, 2), (1000, 1)):
        b = shard.row_bands(H, world)
        assert len(b) == world and b[0][0] == 0 and b[-1][1] == H
        for (a0, a1), (c0, _) in zip(b[:-1], b[1:]):
            assert a1 == c0 and a1 % 64 == 0 and a0 <= a1


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _scene_rows(rng, n, H, W):
    rows = []
    for _ in range(n):
        kind = int(rng.integers(0, 4))
        px, py = rng.uniform(0, W), rng.uniform(0, H)
        hw = int(rng.integers(5, 20))
        cx, cy = int(round(px)), int(round(py))
        mx0, mx1 = max(0, cx - hw), min(W, cx + hw + 1)
        my0, my1 = max(0, cy - hw), min(H, cy + hw + 1)
        rows.append([kind, px, py, rng.uniform(10, 1000), mx0, my0, mx1 - mx0, my1 - my0,
                     rng.uniform(0, 1), rng.uniform(0.8, 3), 0.1, -0.2, rng.uniform(0.8, 3),
                     -0.05, 0.15])
    return np.array(rows)


def _small_blobs(n_blobs):
    from tractor_b200 import fit
    from oracle import oracle as O
    rng = np.random.default_rng(21)
    w = fit.blob_workload(n_blobs, rng, side_range=(32, 40), mean_src=1, max_src=2,
                          flux_range=(500., 2000.))
    ns = np.array([0.8, 1.2, 2.2, 4.5])
    w['truth'][:, 8] = ns[rng.integers(0, len(ns), len(w['truth']))]
    w['start'][:, 8] = w['truth'][:, 8] + 0.03
    data = []
    for b in range(n_blobs):
        s0, s1 = w['blob_src'][b], w['blob_src'][b + 1]
        W, H = (int(v) for v in w['sides'][b])
        rects = [tuple(int(v) for v in (r['x0'], r['y0'], r['w'], r['h']))
                 for r in w['sources'][s0:s1]]
        mod = O.blob_model(w['truth'][s0:s1], rects, W, H, w['psf'][b], 3)
        data.append((rects, W, H, mod + w['noise'][b][:, None, None] * rng.normal(size=mod.shape)))
    return w, data


def _fit_blob(w, data, b):
    from oracle import oracle as O
    s0, s1 = w['blob_src'][b], w['blob_src'][b + 1]
    rects, W, H, d = data[b]
    inv = np.broadcast_to(1. / w['noise'][b][:, None, None], d.shape)
    p, _, _ = O.blob_fit(w['start'][s0:s1], rects, W, H, w['psf'][b], 3, d, inv, tol=1e-6,
                         max_iter=8)
    out = np.zeros(2 * 9)          # fixed-size row: up to 2 sources x 9 parameters
    out[:p.size] = p.ravel()
    return out


def _workloads():
    from tractor_b200 import batch
    rng = np.random.default_rng(12)
    masks = rng.integers(16, 40, 10)
    srcs = batch.sersic_sources(10, rng, mask=masks)
    H, W = 200, 96
    rows = _scene_rows(np.random.default_rng(13), 40, H, W)
    return srcs, (rows, H, W)


def _render_fourier(srcs, i):
    from oracle import oracle as O
    from tractor_b200 import batch
    s = srcs[i]
    amp, var = O.sersic_profile(float(s['sersic_n']))
    T = O.nullwcs_cdinv() @ O.ellipseE_basis(s['s0'], s['s1'], s['s2'])
    a2, v2 = O.sheared(amp, var, T)
    m = int(s['mw'])
    img, _ = O.galaxy_fft_masked(a2, v2, s['px'], s['py'], batch.moffat_psf(), 0, 0, m, m)
    out = np.zeros(40 * 40, np.float32)     # fixed-size row: masks are below 40 px
    out[:m * m] = np.asarray(img, np.float32).ravel()
    return out


PSF_AMP, PSF_SIG = np.array([0.7, 0.2, 0.1]), np.array([1.3, 2.6, 5.2])


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=__import__('datetime').timedelta(seconds=60))
    try:
        from oracle import oracle as O
        from tractor_b200 import shard
        srcs, (rows, H, W) = _workloads()
        res = {}
        # Fourier-path galaxies, cost-balanced
        own = np.flatnonzero(shard.balance(shard.fourier_costs(srcs), world) == rank)
        mine = torch.from_numpy(np.stack([_render_fourier(srcs, i) for i in own]))
        res['fourier'] = shard.gather_units(mine, own, len(srcs)).numpy()
        # the scene in row bands: the band's sources in catalog order, shifted
        y0, y1 = shard.row_bands(H, world)[rank]
        sel = shard.band_members(rows[:, 5], rows[:, 7], rows[:, 6], y0, y1)
        band = rows[sel].copy()
        band[:, 2] -= y0
        band[:, 5] -= y0
        # clip the shifted masks to the band (the renderer clips to its image)
        top = np.maximum(band[:, 5], 0)
        bot = np.minimum(band[:, 5] + band[:, 7], y1 - y0)
        band[:, 7] = bot - top
        band[:, 5] = top
        img = O.scene_model(band, PSF_AMP, PSF_SIG, y1 - y0, W)
        res['scene'] = shard.gather_rows(torch.from_numpy(img)).numpy()
        # blobs, cost-balanced, one fixed-size row of parameters each
        w, data = _small_blobs(4)
        costs = shard.blob_costs(w['blob_src'], w['sides'], w['sources'], w['start'])
        own = np.flatnonzero(shard.balance(costs, world) == rank)
        mine = torch.from_numpy(np.stack([_fit_blob(w, data, b) for b in own])
                                if len(own) else np.zeros((0, 18)))
        res['blobs'] = shard.gather_units(mine, own, 4).numpy()
        if rank == 0:
            np.savez(os.path.join(out_dir, 'sharded.npz'), **res)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_the_single_process_results(tmp_path):
    from oracle import oracle as O
    from tractor_b200 import shard
    tmp.start_processes(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2,
                        join=True, start_method='spawn')
    got = np.load(os.path.join(str(tmp_path), 'sharded.npz'))
    srcs, (rows, H, W) = _workloads()
    ref = np.stack([_render_fourier(srcs, i) for i in range(len(srcs))])
    assert np.array_equal(got['fourier'], ref)
    full = O.scene_model(rows, PSF_AMP, PSF_SIG, H, W)
    assert got['scene'].shape == full.shape
    assert np.array_equal(got['scene'], full)
    w, data = _small_blobs(4)
    ref = np.stack([_fit_blob(w, data, b) for b in range(4)])
    assert np.array_equal(got['blobs'], ref)
    # both ranks had work
    costs = shard.blob_costs(w['blob_src'], w['sides'], w['sources'], w['start'])
    assert set(shard.balance(costs, 2)) == {0, 1}
