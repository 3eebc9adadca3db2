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
