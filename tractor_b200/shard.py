"""Multi-GPU partitioning of the batched workloads.

One process per GPU (torch.distributed, NCCL between GPUs, gloo on CPU).
The forward model's units are independent -- galaxies on their own patches,
blobs, and the patches summed into one image -- so each rank takes a share
and works alone: there is no collective inside the render or fit loops, and
one gather of each rank's results at the end.  This replaces the
reference's only parallelism, TractorMultiprocMixin._map
(tractor/multiproc.py:4-160), which maps sources and images over host
processes.

  balance             cost-balanced assignment of units to ranks (longest
                      processing time first, deterministic);
  fourier_costs,      the cost models: pixels x Gaussian components (x
  blob_costs            parameters for fitting) of each unit;
  row_bands,          a scene image split into row bands whose edges are
  band_members,         multiples of the largest render tile, and the sources
  band_records          whose masks reach a band (the records shifted into
                        the band's coordinates);
  gather_rows         one all-gather of every rank's variable-length rows,
                        returned in rank order.

A band renders exactly the pixels of the whole-image render: sources are
shifted by an integer number of rows and the band edges fall on tile edges,
so every tile sees the same relative coordinates.
"""
import numpy as np
import torch

from . import _lib, profiles


def balance(costs, world):
    """Owner rank of each unit: units taken in order of decreasing cost
    (ties by index), each given to the rank with the least total so far
    (ties to the lowest rank).  Deterministic, so every rank computes the
    same assignment without communicating."""
    costs = np.asarray(costs, np.float64)
    world = int(world)
    if world < 1:
        raise ValueError('world size must be >= 1')
    owner = np.zeros(len(costs), np.int32)
    if world == 1 or len(costs) == 0:
        return owner
    load = np.zeros(world)
    for i in np.argsort(-costs, kind='stable'):
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += costs[i]
    return owner


def _sersic_k(n):
    """Gaussian components of the Sersic mixture at index n (core included)."""
    S = profiles.tables()['sersic']
    n = float(n)
    for r in S['ranges']:
        if r['lo'] <= n < r['hi']:
            return r['K'] + (1 if n > 1 else 0)
    return S['ranges'][-1]['K'] + 1


def fourier_costs(srcs):
    """Cost of each GALAXY_SRC record on the Fourier path: the FFT box's
    pixels (the next power of two of the mask's size, at least 32) times
    the profile's component count."""
    m = np.maximum(srcs['mw'], srcs['mh']).astype(np.int64)
    sz = np.maximum(32, 2 ** np.ceil(np.log2(np.maximum(m, 1) + 2)).astype(np.int64))
    k = np.array([_sersic_k(n) if p == _lib.PROFILE_SERSIC else 8
                  for n, p in zip(srcs['sersic_n'], srcs['profile'])], np.float64)
    return sz.astype(np.float64) ** 2 * k


def blob_costs(blob_src, sides, sources, params, n_bands=3, psf_k=3):
    """Cost of each blob of a fit: per source, its mask pixels inside the
    blob times galaxy components times PSF components times bands, times the
    blob's parameter count (the normal-equation blocks grow with it)."""
    blob_src = np.asarray(blob_src, np.int64)
    nb = len(blob_src) - 1
    side = np.repeat(np.asarray(sides)[:, 0], np.diff(blob_src))
    x0 = np.maximum(sources['x0'], 0)
    y0 = np.maximum(sources['y0'], 0)
    x1 = np.minimum(sources['x0'] + sources['w'], side)
    y1 = np.minimum(sources['y0'] + sources['h'], side)
    area = np.maximum(x1 - x0, 0).astype(np.float64) * np.maximum(y1 - y0, 0)
    k = np.array([_sersic_k(n) for n in np.asarray(params)[:, 8]], np.float64)
    per_src = area * k * psf_k * n_bands
    blob_of = np.repeat(np.arange(nb), np.diff(blob_src))
    cost = np.bincount(blob_of, weights=per_src, minlength=nb)
    return cost * (9. * np.diff(blob_src))


def row_bands(H, world, align=64):
    """[(y0, y1)] per rank: [0, H) cut into `world` bands of whole multiples
    of `align` rows (the tallest render tile), as equal as that allows."""
    H, world = int(H), int(world)
    blocks = -(-H // align)
    cuts = [min(H, (blocks * r // world) * align) for r in range(world + 1)]
    cuts[-1] = H
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def band_members(my0, mh, mw, y0, y1):
    """Indices of the sources whose mask rows [my0, my0 + mh) reach the band
    [y0, y1) (empty masks excluded), in catalog order."""
    my0 = np.asarray(my0, np.int64)
    mh = np.asarray(mh, np.int64)
    return np.flatnonzero((my0 + mh > y0) & (my0 < y1) & (np.asarray(mw) > 0) & (mh > 0))


def band_records(recs, y0, y1):
    """The SCENE_SRC records whose mask rectangle reaches rows [y0, y1),
    shifted into the band's coordinates (py and the mask's my0 less y0; the
    renderer clips each mask to the band).  Returns (records, indices)."""
    recs = np.asarray(recs)
    sel = band_members(recs['my0'], recs['mh'], recs['mw'], y0, y1)
    out = recs[sel].copy()
    out['py'] -= y0
    out['my0'] -= y0
    return out, sel


def gather_rows(local, group=None):
    """All-gather of each rank's rows (a tensor whose first dimension may
    differ between ranks), concatenated in rank order on every rank.  Two
    collectives: the row counts, then the rows padded to the largest count.
    The tensor's device must suit the process group's backend."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    if world == 1:
        return local
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=local.device)
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n, group=group)
    counts = [int(c.item()) for c in counts]
    m = max(counts)
    pad = torch.zeros((m,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[:c] for p, c in zip(parts, counts)])


def gather_units(rows, mine, n_units, group=None):
    """Every unit's result row in unit order, on every rank: `rows` holds this
    rank's results (one row per unit of `mine`, this rank's unit indices),
    gathered with their indices in one gather_rows each."""
    idx = torch.as_tensor(np.asarray(mine, np.int64), device=rows.device)
    all_rows = gather_rows(rows, group)
    all_idx = gather_rows(idx, group)
    out = torch.zeros((int(n_units),) + tuple(rows.shape[1:]), dtype=rows.dtype,
                      device=rows.device)
    out[all_idx] = all_rows
    return out
