"""tb_normal_equations on the tensor cores (tcgen05 kind::tf32, three-term
TF32 split, FP32 partial sums over at most 128 rows, FP64 totals) against
FP64 numpy: the stacked one-MMA kernel for P <= 63 (launches whose max_p is
at most 63), the general kernel for P <= 255, and the CUDA-core kernel kept
for P > 255.

Tolerance: every A^T A entry within 2e-6 of sqrt(H_ii H_jj) (the
Cauchy-Schwarz bound of the entry's sum of |products|), every A^T r entry
within 2e-6 of sqrt(H_ii r^T r); AtA exactly symmetric; no tensor-core wait
timed out."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 2e-6


def _problems(Ps, Rs, seed, pad=0, align=False):
    """Column-major problems in flat arrays.  pad: extra rows of the leading
    dimension; align: leading dimensions and right-hand-side segments
    rounded up to 4 floats, so every column starts on a 16-byte boundary."""
    rng = np.random.default_rng(seed)
    A_list, r_list = [], []
    for P, R in zip(Ps, Rs):
        A = rng.normal(size=(R, P)) * rng.uniform(0.1, 100, P)
        A += rng.normal(size=(R, 1)) * 3.   # correlated columns (off-diagonal mass)
        A_list.append(A.astype(np.float32))
        r_list.append((rng.normal(size=R) * 5 + A @ rng.normal(size=P) * 0.01).astype(np.float32))
    up = (lambda n: (n + 3) // 4 * 4) if align else (lambda n: n)   # noqa: E731
    lda = [up(R + pad) for R in Rs]
    A_flat = np.concatenate([np.pad(a.T, ((0, 0), (0, l - len(a)))).ravel()
                             for a, l in zip(A_list, lda)] + [[0.]])
    r_flat = np.concatenate([np.pad(r, (0, up(len(r)) - len(r))) for r in r_list] + [[0.]])
    a_off = np.concatenate([[0], np.cumsum([P * l for P, l in zip(Ps, lda)])[:-1]])
    r_off = np.concatenate([[0], np.cumsum([up(R) for R in Rs])[:-1]])
    return A_list, r_list, A_flat.astype(np.float32), r_flat.astype(np.float32), a_off, r_off, lda


def _run_and_check(Ps, Rs, seed, pad=0, align=False):
    import torch
    from tractor_b200 import render, _lib
    A_list, r_list, A_flat, r_flat, a_off, r_off, lda = _problems(Ps, Rs, seed, pad, align)
    AtA, Atr, ao, ro = render.normal_equations(torch.from_numpy(A_flat).cuda(),
                                               torch.from_numpy(r_flat).cuda(),
                                               a_off, r_off, lda, Ps, Rs)
    AtA, Atr = AtA.cpu().numpy(), Atr.cpu().numpy()
    ao, ro = ao.cpu().numpy(), ro.cpu().numpy()
    worst = 0.
    for i, (P, A, r) in enumerate(zip(Ps, A_list, r_list)):
        M = AtA[ao[i]:ao[i] + P * P].reshape(P, P)
        g = Atr[ro[i]:ro[i] + P]
        A64, r64 = A.astype(np.float64), r.astype(np.float64)
        refM, refg = A64.T @ A64, A64.T @ r64
        assert np.array_equal(M, M.T), i
        if len(r) == 0:
            assert np.all(M == 0) and np.all(g == 0)
            continue
        d = np.sqrt(np.diag(refM))
        eM = np.abs(M - refM) / np.outer(d, d)
        eg = np.abs(g - refg) / (d * np.sqrt(r64 @ r64))
        worst = max(worst, eM.max(), eg.max())
        assert eM.max() < TOL, (i, P, len(r), eM.max())
        assert eg.max() < TOL, (i, P, len(r), eg.max())
    lib = _lib.load()
    n = ctypes.c_uint32(0)
    assert lib.tb_tensor_core_timeouts(ctypes.byref(n)) == 0
    assert n.value == 0
    return worst


def test_stacked_kernel_mixed_sizes(tb):
    """P <= 63 (one MMA per K step on the stacked [Hi; Lo] operand): sizes on
    and off the 8 / 16 / 32 boundaries and the 32-row block edge, rows not a
    multiple of the 64-row stage or of the 128-row chunk, a single stage,
    R = 0."""
    w = _run_and_check([1, 6, 7, 15, 31, 32, 33, 47, 54, 63, 20],
                       [4096, 33, 1, 3000, 2049, 128, 64, 1025, 2500, 700, 0], seed=7)
    w2 = _run_and_check([63, 32, 5], [5003, 130, 9], seed=8, align=True)
    print('worst scaled error (stacked):', w, w2)


def test_stacked_kernel_whole_quads(tb):
    """P <= 63 with 16-byte-aligned columns and R a multiple of 4 (whole
    16-byte copies in every stage): a last stage of 4 .. 28 rows, a single
    short stage, exact stage and chunk multiples, more stages than the raw
    ring holds, the benchmark's 16,384 rows."""
    w = _run_and_check([63, 63, 1, 31, 32, 47, 7, 63],
                       [16384, 1004, 4, 36, 4096, 2052, 128, 96], seed=11, align=True)
    print('worst scaled error (stacked, whole quads):', w)


def test_one_m_tile_mixed_sizes(tb):
    """Q = P + 1 <= 128: sizes on and off the 8 / 16 / 32 boundaries, rows not
    a multiple of the 32-row stage, several 1024-row chunks, R = 0."""
    w = _run_and_check([1, 6, 7, 15, 31, 54, 127, 100], [4096, 33, 1, 3000, 2049, 1025, 2500, 0],
                       seed=1)
    print('worst scaled error (one tile):', w)


def test_two_m_tiles(tb):
    """128 < Q <= 256: the second M tile (rows 128-255 against columns
    128..Q) and the mirrored block; a padded leading dimension."""
    w = _run_and_check([128, 200, 255, 3], [1500, 2049, 777, 100], seed=2, pad=5)
    print('worst scaled error (two tiles):', w)


def test_aligned_columns(tb):
    """Every column on a 16-byte boundary: the 16-byte copy path, with rows
    not a multiple of 4 (partial quads) and of the stage."""
    w = _run_and_check([6, 63, 127, 1, 30], [4096, 1001, 2050, 7, 3333], seed=5, align=True)
    w2 = _run_and_check([200, 129], [1003, 2500], seed=6, align=True)
    print('worst scaled error (aligned):', w, w2)


def test_cuda_core_path_above_255(tb):
    _run_and_check([300, 64], [500, 700], seed=3)


def test_long_rows(tb):
    """A long problem (16 chunks of FP32 accumulation)."""
    w = _run_and_check([63], [16384 + 17], seed=4)
    print('worst scaled error (long):', w)
