"""Loads libtractor_b200.so (the sm_100a kernels) through its C ABI
(include/tractor_b200.h).  There is no CPU implementation behind this module:
if the library is missing, or no CUDA device is present when a kernel is
called, it raises."""
import ctypes
import os
import re

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libtractor_b200.so')
HEADER = os.path.join(os.path.dirname(_HERE), 'include', 'tractor_b200.h')

# Layouts of the C structs (must match include/tractor_b200.h; checked
# against tb_abi_sizes() at load time).
MOG_ITEM = np.dtype([('x0', '<i4'), ('y0', '<i4'), ('w', '<i4'), ('h', '<i4'),
                     ('c0', '<i4'), ('K', '<i4'), ('mode', '<i4'), ('ldo', '<i4'),
                     ('fx', '<f8'), ('fy', '<f8'), ('floor', '<f8'),
                     ('scale', '<f4'), ('pad1', '<i4'),
                     ('out_off', '<i8'), ('mask_off', '<i8'), ('tile0', '<i8')])
FFT_ITEM = np.dtype([('c0', '<i4'), ('K', '<i4'), ('sz', '<i4'), ('psf', '<i4'),
                     ('mw', '<i4'), ('mh', '<i4'), ('sx', '<i4'), ('sy', '<i4'),
                     ('mux', '<f8'), ('muy', '<f8'), ('scale', '<f4'), ('mode', '<i4'),
                     ('out_off', '<i8'), ('ldo', '<i4'), ('pad0', '<i4')])
STATUS = np.dtype([('code', '<i4'), ('item', '<i4'), ('detail', '<i4'), ('count', '<i4')])

MOG_STORE, MOG_ACCUM, MOG_ATOMIC = 0, 1, 2
MOG_TILE = 32

TB_OK = 0
_ERRORS = {-1: 'invalid argument', -2: 'CUDA launch error', -3: 'unsupported size'}

_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double

# name -> (restype, argtypes)
SIGNATURES = {
    'tb_mog_render': (_I32, [_P, _I32, _I64, _P, _P, _P, _P, _P, _P, _P, _P]),
    'tb_lanczos3_shift': (_I32, [_P, _P, _P, _I32, _I32, _I32, _P]),
    'tb_fourier_render': (_I32, [_P, _I32, _P, _P, _P, _P, _P, _P, _P]),
    'tb_psf_spectrum': (_I32, [_P, _P, _I32, _I32, _I32, _P]),
    'tb_normal_equations': (_I32, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I32, _I32, _P]),
    'tb_solve_update': (_I32, [_P, _P, _P, _P, _P, _P, _P, _P, _D, _I32, _I32, _P, _P]),
    'tb_chi2': (_I32, [_P, _P, _P, _P, _P, _I32, _P, _P]),
    'tb_version': (ctypes.c_char_p, []),
    'tb_abi_sizes': (_I32, [_P]),
}

_lib = None


def header_symbols():
    """Entry points declared in include/tractor_b200.h."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r'^\s*(?:int|const char\*)\s+(tb_\w+)\s*\(', txt, re.M)))


def load():
    """Returns the loaded library, raising ImportError if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError('libtractor_b200.so is not built; run `python -m tractor_b200.build` '
                          '(or __graft_entry__.build()) first')
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    sizes = np.zeros(3, np.int32)
    lib.tb_abi_sizes(sizes.ctypes.data)
    want = (MOG_ITEM.itemsize, FFT_ITEM.itemsize, STATUS.itemsize)
    if tuple(int(s) for s in sizes) != want:
        raise ImportError('libtractor_b200.so struct layout %s != binding %s' %
                          (tuple(sizes), want))
    _lib = lib
    return lib


def check(rc, what):
    if rc != TB_OK:
        raise RuntimeError('%s failed: %s (%d)' % (what, _ERRORS.get(rc, 'error'), rc))


def ptr(t):
    """Device (or host) address of a torch tensor or numpy array, or None."""
    if t is None:
        return None
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    return t.data_ptr()


def stream_ptr(stream=None):
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError('tractor_b200 kernels need a CUDA device (sm_100a); none is available')
