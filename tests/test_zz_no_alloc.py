"""tb_solve_update_noalloc: the least-squares solve for callers that cannot
allocate device memory when they call (they run under another allocator
that owns the device memory, or in a latency-bound loop where an allocation,
which can synchronise the device, is not acceptable).  It uses the library's
own file-scope scratch array instead of a caller-provided workspace.

Checked through the C ABI against tb_solve_update (which takes the
workspace from the caller) on two calls in a row, so the second call runs
over the scratch the first one left behind.  Same tolerance as the other
solver tests.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problems(rng, Ps, Rs):
    A, r = [], []
    for P, R in zip(Ps, Rs):
        A.append(rng.normal(size=(R, P)) * rng.uniform(0.1, 10, P))
        r.append(rng.normal(size=R))
    AtA = np.concatenate([(a.T @ a).ravel() for a in A])
    Atr = np.concatenate([a.T @ b for a, b in zip(A, r)])
    return AtA, Atr


def _solve(lib, fn, AtA, Atr, Ps, damp, with_work):
    import torch
    dev = 'cuda'
    Ps = np.asarray(Ps, np.int32)
    n, maxp = len(Ps), int(Ps.max())
    ata_off = np.concatenate([[0], np.cumsum(Ps.astype(np.int64) ** 2)[:-1]]).astype(np.int64)
    atr_off = np.concatenate([[0], np.cumsum(Ps.astype(np.int64))[:-1]]).astype(np.int64)
    t = lambda a: torch.as_tensor(a, device=dev)  # noqa: E731
    dA, dr, dao, dro, dP, dxo = t(AtA), t(Atr), t(ata_off), t(atr_off), t(Ps), t(atr_off)
    X = torch.full((int(Ps.sum()),), np.nan, dtype=torch.float64, device=dev)
    info = torch.full((n,), -7, dtype=torch.int32, device=dev)
    args = [dA.data_ptr(), dr.data_ptr(), dao.data_ptr(), dro.data_ptr(), dP.data_ptr(),
            dxo.data_ptr(), X.data_ptr(), info.data_ptr(), ctypes.c_double(damp), n, maxp]
    if with_work:
        work = torch.empty(n * maxp * maxp, dtype=torch.float64, device=dev)
        args.append(work.data_ptr())
    rc = fn(*args, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return rc, X.cpu().numpy(), info.cpu().numpy()


def test_noalloc_solve_matches_allocating_solve(tb):
    from tractor_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(77)
    for call, (Ps, Rs, damp) in enumerate([([6, 11, 54, 3], [500, 300, 2000, 40], 0.0),
                                            ([30, 7, 120], [900, 60, 4000], 0.25)]):
        AtA, Atr = _problems(rng, Ps, Rs)
        rc0, X0, i0 = _solve(lib, lib.tb_solve_update, AtA, Atr, Ps, damp, True)
        rc1, X1, i1 = _solve(lib, lib.tb_solve_update_noalloc, AtA, Atr, Ps, damp, False)
        assert rc0 == 0 and rc1 == 0, (call, rc0, rc1)
        assert np.all(i0 == 0) and np.array_equal(i0, i1), (call, i0, i1)
        assert np.all(np.isfinite(X1))
        np.testing.assert_allclose(X1, X0, rtol=1e-12, atol=0, err_msg='call %d' % call)


def test_noalloc_rejects_sizes_beyond_its_scratch(tb):
    from tractor_b200 import _lib
    lib = _lib.load()
    # 40 problems of 200 parameters need 1.6M doubles > 1,048,576
    rc = lib.tb_solve_update_noalloc(1, 1, 1, 1, 1, 1, 1, 1, ctypes.c_double(0.), 40, 200, None)
    assert rc == -3


def test_problem_larger_than_max_p_is_refused(tb):
    """P[b] is device data the host cannot check: a problem with P[b] > max_p
    gets info = -1 and writes nothing, so the other problems' factors (in the
    caller's workspace, or in the shared array) are left intact."""
    import torch
    from tractor_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(78)
    Ps, Rs = [8, 12, 8], [200, 300, 200]
    AtA, Atr = _problems(rng, Ps, Rs)
    rc_ok, X_ok, i_ok = _solve(lib, lib.tb_solve_update, AtA, Atr, Ps, 0.0, True)
    assert rc_ok == 0 and np.all(i_ok == 0)
    dev = 'cuda'
    Pa = np.asarray(Ps, np.int32)
    ata_off = np.concatenate([[0], np.cumsum(Pa.astype(np.int64) ** 2)[:-1]]).astype(np.int64)
    atr_off = np.concatenate([[0], np.cumsum(Pa.astype(np.int64))[:-1]]).astype(np.int64)
    t = lambda a: torch.as_tensor(a, device=dev)  # noqa: E731
    max_p = 8           # the middle problem (P = 12) exceeds it
    for fn, with_work in ((lib.tb_solve_update, True), (lib.tb_solve_update_noalloc, False)):
        dA, dr, dao, dro, dP, dxo = t(AtA), t(Atr), t(ata_off), t(atr_off), t(Pa), t(atr_off)
        X = torch.full((int(Pa.sum()),), 123.0, dtype=torch.float64, device=dev)
        info = torch.full((3,), -7, dtype=torch.int32, device=dev)
        args = [dA.data_ptr(), dr.data_ptr(), dao.data_ptr(), dro.data_ptr(), dP.data_ptr(),
                dxo.data_ptr(), X.data_ptr(), info.data_ptr(), ctypes.c_double(0.0), 3, max_p]
        if with_work:
            # the 3 slices of max_p^2 doubles, then a sentinel region
            work = torch.full((3 * max_p * max_p + 256,), -5.0, dtype=torch.float64, device=dev)
            args.append(work.data_ptr())
        rc = fn(*args, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert rc == 0
        inf = info.cpu().numpy()
        assert inf.tolist() == [0, -1, 0], inf
        x = X.cpu().numpy()
        assert np.all(x[8:20] == 123.0)          # the refused problem's X untouched
        np.testing.assert_allclose(x[:8], X_ok[:8], rtol=1e-12, atol=0)
        np.testing.assert_allclose(x[20:], X_ok[20:], rtol=1e-12, atol=0)
        if with_work:
            assert torch.all(work[3 * max_p * max_p:] == -5.0)
            assert torch.all(work[max_p * max_p:2 * max_p * max_p] == -5.0)


def test_noalloc_call_allocates_no_device_memory(tb):
    """The entry point's purpose: a warm call leaves the device's free memory
    unchanged (no cudaMalloc inside, no allocating library routine)."""
    import torch
    from tractor_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(79)
    Ps = np.asarray([20, 35, 9], np.int32)
    AtA, Atr = _problems(rng, Ps, [400, 800, 100])
    dev = 'cuda'
    ata_off = np.concatenate([[0], np.cumsum(Ps.astype(np.int64) ** 2)[:-1]]).astype(np.int64)
    atr_off = np.concatenate([[0], np.cumsum(Ps.astype(np.int64))[:-1]]).astype(np.int64)
    t = lambda a: torch.as_tensor(a, device=dev)  # noqa: E731
    dA, dr, dao, dro, dP, dxo = t(AtA), t(Atr), t(ata_off), t(atr_off), t(Ps), t(atr_off)
    X = torch.zeros(int(Ps.sum()), dtype=torch.float64, device=dev)
    info = torch.zeros(3, dtype=torch.int32, device=dev)
    args = [dA.data_ptr(), dr.data_ptr(), dao.data_ptr(), dro.data_ptr(), dP.data_ptr(),
            dxo.data_ptr(), X.data_ptr(), info.data_ptr(), ctypes.c_double(0.1), 3,
            int(Ps.max()), torch.cuda.current_stream().cuda_stream]
    assert lib.tb_solve_update_noalloc(*args) == 0     # first call: address look-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert lib.tb_solve_update_noalloc(*args) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert np.all(info.cpu().numpy() == 0)
