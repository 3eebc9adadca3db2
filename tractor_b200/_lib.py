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
                     ('scale', '<f4'), ('floor_mode', '<i4'),
                     ('out_off', '<i8'), ('mask_off', '<i8'), ('tile0', '<i8'),
                     ('deriv_off', '<i8'), ('diff_c0', '<i4'), ('pad', '<i4')])
FLOOR_FIXED, FLOOR_MINVAL = 0, 1
FFT_ITEM = np.dtype([('c0', '<i4'), ('K', '<i4'), ('sz', '<i4'), ('mode', '<i4'),
                     ('mw', '<i4'), ('mh', '<i4'), ('sx', '<i4'), ('sy', '<i4'),
                     ('mux', '<f8'), ('muy', '<f8'), ('scale', '<f4'), ('ldo', '<i4'),
                     ('out_off', '<i8'), ('spec_off', '<i8'), ('dmode', '<i4'), ('dc0', '<i4'),
                     ('dot_off', '<i8')])
FFT_VALUE, FFT_DSPEC, FFT_DX, FFT_DY, FFT_DIFF = 0, 1, 2, 3, 4
FFT_DOT = 3
STATUS = np.dtype([('code', '<i4'), ('item', '<i4'), ('detail', '<i4'), ('count', '<i4')])
RING_ITEM = np.dtype([('val_off', '<i8'), ('deriv_off', '<i8'), ('edge_col_off', '<i8'),
                      ('edge_row_off', '<i8'), ('w', '<i4'), ('h', '<i4'), ('xc', '<i4'),
                      ('yc', '<i4'), ('edge_x', '<i4'), ('edge_y', '<i4'), ('dcx', '<i4'),
                      ('dcy', '<i4'), ('minradius', '<i4'), ('start_inside', '<i4'),
                      ('minval', '<f8')])
RING_MAX = 4096
GALAXY_SRC = np.dtype([('px', '<f8'), ('py', '<f8'), ('counts', '<f8'), ('s0', '<f8'),
                       ('s1', '<f8'), ('s2', '<f8'), ('sersic_n', '<f8'), ('out_off', '<i8'),
                       ('profile', '<i4'), ('shape_type', '<i4'), ('mx0', '<i4'), ('my0', '<i4'),
                       ('mw', '<i4'), ('mh', '<i4')])

SCENE_SRC = np.dtype([('px', '<f8'), ('py', '<f8'), ('counts', '<f8'), ('fdev', '<f8'),
                      ('sa0', '<f8'), ('sa1', '<f8'), ('sa2', '<f8'),
                      ('sb0', '<f8'), ('sb1', '<f8'), ('sb2', '<f8'), ('sersic_n', '<f8'),
                      ('profile', '<i4'), ('shape_type', '<i4'), ('image', '<i4'),
                      ('mx0', '<i4'), ('my0', '<i4'), ('mw', '<i4'), ('mh', '<i4'),
                      ('pad', '<i4')])
SCENE_IMAGE = np.dtype([('W', '<i4'), ('H', '<i4'), ('ldo', '<i4'), ('psf_c0', '<i4'),
                        ('psf_K', '<i4'), ('pad', '<i4'), ('out_off', '<i8'), ('tile0', '<i8'),
                        ('cd_inv', '<f8', (4,)), ('pixscale', '<f8')])
SCENE_ITEM = np.dtype([('x0', '<i4'), ('y0', '<i4'), ('w', '<i4'), ('h', '<i4'),
                       ('c0', '<i4'), ('K', '<i4'), ('image', '<i4'), ('flag', '<i4'),
                       ('fx', '<f8'), ('fy', '<f8'), ('scale', '<f4'), ('floor', '<f4')])

FIT_NPAR, FIT_MAX_BANDS, FIT_MAX_SRC, FIT_MAX_PSF = 9, 3, 32, 4
FIT_REFINE, FIT_MODEL, FIT_VJP = 0, 1, 2
EM_MAX_K = 8   # TB_EM_MAX_K
FIT_SOURCE = np.dtype([('profile', '<i4'), ('x0', '<i4'), ('y0', '<i4'), ('w', '<i4'),
                       ('h', '<i4'), ('blob', '<i4'), ('frozen', '<i4'), ('pad', '<i4')])
FIT_BLOB = np.dtype([('n_src', '<i4'), ('src0', '<i4'), ('P', '<i4'), ('unit0', '<i4'),
                     ('h_off', '<i8'), ('g_off', '<i8'), ('tile_off', '<i8'),
                     ('n_active', '<i4'), ('n_tiles', '<i4'), ('n_slices', '<i4'),
                     ('pad', '<i4')])
FIT_UNIT = np.dtype([('blob', '<i4'), ('band', '<i4'), ('W', '<i4'), ('H', '<i4'),
                     ('pix_off', '<i8'), ('psf_K', '<i4'), ('slice', '<i4'),
                     ('t0', '<i4'), ('t1', '<i4'),
                     ('psf_amp', '<f8', (4,)), ('psf_mean', '<f8', (8,)),
                     ('psf_var', '<f8', (16,))])
FIT_STATE = np.dtype([('chi2', '<f8'), ('dlnp', '<f8'), ('lambda', '<f8'), ('pred', '<f8'),
                      ('iters', '<i4'),
                      ('accepted', '<i4'), ('rejected', '<i4'), ('status', '<i4')])

PROFILE_EXP, PROFILE_DEV, PROFILE_SERSIC, PROFILE_GAUSSIAN = 0, 1, 2, 3
PROFILE_POINT, PROFILE_COMPOSITE = 4, 5
SHAPE_ELLIPSE_E, SHAPE_ELLIPSE_ESOFT, SHAPE_RABPHI = 0, 1, 2


class FftImage(ctypes.Structure):
    """tb_fft_image."""
    _fields_ = [('cd_inv', ctypes.c_double * 4), ('pixscale', ctypes.c_double),
                ('psf_w', ctypes.c_int32), ('psf_h', ctypes.c_int32),
                ('psf_cx', ctypes.c_double * 4), ('psf_cy', ctypes.c_double * 4),
                ('spec_off', ctypes.c_int64 * 4)]


class ProfileTables(ctypes.Structure):
    """tb_profile_tables (device pointers)."""
    _fields_ = [('n_ranges', ctypes.c_int32), ('core_spline', ctypes.c_int32),
                ('range_lohi', ctypes.c_void_p), ('range_info', ctypes.c_void_p),
                ('spline_info', ctypes.c_void_p), ('knots', ctypes.c_void_p),
                ('coefs', ctypes.c_void_p), ('exp_amp', ctypes.c_void_p),
                ('exp_var', ctypes.c_void_p), ('dev_amp', ctypes.c_void_p),
                ('dev_var', ctypes.c_void_p), ('exp_K', ctypes.c_int32),
                ('dev_K', ctypes.c_int32), ('n_splines', ctypes.c_int32),
                ('n_knots', ctypes.c_int32), ('n_coefs', ctypes.c_int32),
                ('pad', ctypes.c_int32)]

MOG_STORE, MOG_ACCUM, MOG_ATOMIC = 0, 1, 2
MOG_TILE = 32

TB_OK = 0
TB_ERR_ARG, TB_ERR_LAUNCH, TB_ERR_SIZE = -1, -2, -3
_ERRORS = {-1: 'invalid argument', -2: 'CUDA launch error', -3: 'unsupported size'}

_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double

# name -> (restype, argtypes)
SIGNATURES = {
    'tb_mog_render': (_I32, [_P, _I32, _I64, _P, _P, _P, _P, _P, _P, _P, _P]),
    'tb_mog_render_host_bytes': (_I32, [_I32, _I64, _I64, _I64, _P]),
    'tb_mog_render_host': (_I32, [_P, _I32, _I64, _P, _P, _P, _I64, _P, _I64, _P, _I64, _P, _P,
                                  _P, _I64, _P]),
    'tb_lanczos3_shift': (_I32, [_P, _P, _P, _I32, _I32, _I32, _P]),
    'tb_fourier_render': (_I32, [_P, _I32, _P, _P, _P, _P, _P, _P, _P]),
    'tb_psf_spectrum': (_I32, [_P, _P, _I32, _I32, _I32, _P]),
    'tb_normal_equations': (_I32, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I32, _I32, _P]),
    'tb_tensor_core_timeouts': (_I32, [_P]),
    'tb_em_fit_2d': (_I32, [_P, _I32, _I32, _I32, _P, _P, _P, _P, _I32, _D, _I32, _P, _P]),
    'tb_em_fit_2d_sky': (_I32, [_P, _I32, _I32, _I32, _P, _P, _P, _P, _I32, _D, _I32, _D,
                                 _P, _P, _P]),
    'tb_label_workspace_bytes': (ctypes.c_int64, [_I32, _I32]),
    'tb_label_components': (_I32, [_P, _I32, _I32, _I32, _P, _P, _P, _P, _P]),
    'tb_component_boxes': (_I32, [_P, _I32, _I32, _I32, _P, _P]),
    'tb_solve_update': (_I32, [_P, _P, _P, _P, _P, _P, _P, _P, _D, _I32, _I32, _P, _P]),
    'tb_solve_update_noalloc': (_I32, [_P, _P, _P, _P, _P, _P, _P, _P, _D, _I32, _I32, _P]),
    'tb_chi2': (_I32, [_P, _P, _P, _P, _P, _I32, _P, _P]),
    'tb_galaxy_fft_prep': (_I32, [_P, _I32, _P, _P, _P, _P, _P, _I32, _P, _P]),
    'tb_galaxy_fft_render': (_I32, [_P, _I32, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    'tb_fourier_spectrum_grid': (_I32, [_P, _P, _P, _I32, _P, _I32, _P, _P]),
    'tb_galaxy_fft_jac_prep': (_I32, [_P, _I32, _P, _P, _P, _P, _P, _P, _I32, _I32, _I64, _P,
                                      _P]),
    'tb_fourier_render_deriv': (_I32, [_P, _I32, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    'tb_fourier_workspace': (_I32, [_I32, _P]),
    'tb_fourier_render_split': (_I32, [_P, _I32, _P, _P, _P, _P, _P, _P, _P, _I64, _P, _P]),
    'tb_scene_prep': (_I32, [_P, _I32, _P, _I32, _P, _P, _P, _P, _P, _P, _P, _P, _I32, _P]),
    'tb_scene_workspace': (_I32, [_I64, _I64, _P]),
    'tb_fit_workspace': (_I32, [_I32, _I32, _P]),
    'tb_fit_reset': (_I32, [_P, _I32, _D, _P]),
    'tb_fit_prep': (_I32, [_P, _I32, _P, _I32, _P, _I32, _P, _P, _P, _P, _P]),
    'tb_fit_pass': (_I32, [_P, _P, _I32, _P, _P, _I32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I32,
                           _I32, _P, _P, _P]),
    'tb_fit_step': (_I32, [_P, _I32, _I32, _P, _P, _P, _P, _P, _P, _P, _D, _I32, _P]),
    'tb_fit_refine': (_I32, [_P, _P, _I32, _P, _P, _I32, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                             _I32, _P, _P, _P]),
    'tb_fit_model_vjp': (_I32, [_P, _P, _I32, _P, _P, _I32, _P, _P, _P, _P, _P, _I32, _I32, _P,
                                _P, _P]),
    'tb_scene_render': (_I32, [_P, _I32, _P, _I32, _I64, _I32, _P, _P, _P, _P, _I32, _P, _I64,
                               _I64, _P, _P]),
    'tb_version': (ctypes.c_char_p, []),
    'tb_abi_sizes': (_I32, [_P]),
    'tb_approx3_region': (_I32, [_P, _I32, _P, _P, _P, _P]),
}

_lib = None


def header_symbols():
    """Entry points declared in include/tractor_b200.h."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r'^\s*(?:int64_t|int|const char\*)\s+(tb_\w+)\s*\(', txt,
                                 re.M)))


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
    sizes = np.zeros(13, np.int32)
    lib.tb_abi_sizes(sizes.ctypes.data)
    want = (MOG_ITEM.itemsize, FFT_ITEM.itemsize, STATUS.itemsize, GALAXY_SRC.itemsize,
            ctypes.sizeof(FftImage), SCENE_SRC.itemsize, SCENE_IMAGE.itemsize,
            SCENE_ITEM.itemsize, FIT_SOURCE.itemsize, FIT_BLOB.itemsize, FIT_UNIT.itemsize,
            FIT_STATE.itemsize, RING_ITEM.itemsize)
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
    """cudaStream_t of `stream`, or of the current device's current stream
    (read without building a torch Stream object: this runs on every launch)."""
    import torch
    if stream is None:
        return torch._C._cuda_getCurrentRawStream(torch._C._cuda_getDevice())
    return stream.cuda_stream


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError('tractor_b200 kernels need a CUDA device (sm_100a); none is available')
