"""The C-ABI library loads and exports every entry point its header declares
(no kernel is called: this runs without a GPU)."""
import ctypes
import os

import pytest


def test_library_exports_header_symbols():
    from tractor_b200 import _lib, build
    build.build()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    declared = _lib.header_symbols()
    assert len(declared) >= 9
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # every declared entry point has a binding signature, and vice versa
    assert set(declared) == set(_lib.SIGNATURES), set(declared) ^ set(_lib.SIGNATURES)


def test_struct_layouts_match_bindings():
    from tractor_b200 import _lib
    lib = _lib.load()   # raises if the C structs and the numpy dtypes disagree
    assert lib.tb_version().startswith(b'tractor_b200')


def test_invalid_arguments_are_rejected_without_a_device():
    """Host-side validation returns an error code before touching the GPU."""
    from tractor_b200 import _lib
    lib = _lib.load()
    assert lib.tb_mog_render(None, 1, 1, None, None, None, None, None, None, None, None) == -1
    assert lib.tb_lanczos3_shift(None, None, None, -1, 4, 4, None) == -1
    assert lib.tb_psf_spectrum(1, 1, 1, 48, 0, None) == -3
    assert lib.tb_normal_equations(None, None, None, None, None, None, None, None, None, None,
                                   None, 1, 400, None) == -3
    assert lib.tb_em_fit_2d(None, 1, 9, 9, None, None, None, None, 3, 0., 10, None, None) == -1
    assert lib.tb_em_fit_2d(None, 1, 9, 9, None, None, None, None, 9, 0., 10, None, None) == -1


def test_mog_render_host_checks_items_before_any_copy():
    """tb_mog_render_host sizes its staging and refuses items that reach
    outside the given component, mask or output sizes, a wrong tile count
    and a short workspace, all on the host before any CUDA call."""
    import numpy as np
    from tractor_b200 import _lib
    lib = _lib.load()
    K, w, h = 3, 40, 20
    item = np.zeros(1, _lib.MOG_ITEM)
    item[0] = (0, 0, w, h, 0, K, _lib.MOG_STORE, 0, 10., 5., -50., 1., _lib.FLOOR_FIXED,
               0, -1, 0, -1, -1, 0)
    tiles = ((w + 31) // 32) * ((h + 31) // 32)
    amp, mean, var = np.ones(K), np.zeros((K, 2)), np.tile(np.eye(2), (K, 1, 1))
    nbytes = ctypes.c_int64()
    assert lib.tb_mog_render_host_bytes(1, K, 0, w * h, ctypes.byref(nbytes)) == _lib.TB_OK
    assert nbytes.value >= item.nbytes + K * 56 + w * h * 4 + 16
    assert lib.tb_mog_render_host_bytes(-1, K, 0, w * h, ctypes.byref(nbytes)) == _lib.TB_ERR_ARG
    lib.tb_mog_render_host_bytes(1, K, 0, w * h, ctypes.byref(nbytes))
    # host stand-ins for the staging buffers: every call below returns first
    pinned = np.zeros(nbytes.value, np.uint8)
    ws = np.zeros(nbytes.value, np.uint8)
    out = np.full(w * h, -7., np.float32)
    st = np.zeros(1, _lib.STATUS)

    def call(it, n_tiles=tiles, n_comp=K, n_out=w * h, ws_bytes=nbytes.value):
        return lib.tb_mog_render_host(it.ctypes.data, 1, n_tiles, amp.ctypes.data,
                                      mean.ctypes.data, var.ctypes.data, n_comp, None, 0,
                                      out.ctypes.data, n_out, st.ctypes.data,
                                      pinned.ctypes.data, ws.ctypes.data, ws_bytes, None)
    assert call(item, n_out=w * h - 1) == _lib.TB_ERR_ARG          # output too small
    assert call(item, n_comp=K - 1) == _lib.TB_ERR_ARG             # components beyond n_comp
    assert call(item, n_tiles=tiles + 1) == _lib.TB_ERR_ARG        # tile count disagrees
    bad = item.copy()
    bad['mask_off'] = 0                                            # a mask with mask_bytes = 0
    assert call(bad) == _lib.TB_ERR_ARG
    bad = item.copy()
    bad['deriv_off'] = w * h                                       # derivative planes past n_out
    assert call(bad) == _lib.TB_ERR_ARG
    bad = item.copy()
    bad['ldo'] = w - 1                                             # row stride below the width
    assert call(bad) == _lib.TB_ERR_ARG
    assert call(item, ws_bytes=nbytes.value - 1) == _lib.TB_ERR_SIZE
    assert np.all(out == -7.)
