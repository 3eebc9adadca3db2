"""Builds libtractor_b200.so (the sm_100a kernels behind include/tractor_b200.h)
in-tree with nvcc.  nvcc cross-compiles, so this works without a GPU."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
LIB = os.path.join(HERE, 'libtractor_b200.so')
INCLUDE = os.path.join(ROOT, 'include')

SOURCES = ['mog_render.cu', 'lanczos.cu', 'fourier_render.cu', 'galaxy_prep.cu', 'lsq.cu',
           'scene_render.cu', 'blob_fit.cu', 'emfit.cu', 'blobs.cu', 'fourier_large.cu']
NVCC_FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-lineinfo', '-O3',
              '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr']


def _nvcc():
    for cand in [os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc']:
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return 'nvcc'


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + \
           [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)] + [__file__]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra_flags=()):
    """Compile every kernel source and link the shared library.  Returns the
    library path.  Raises RuntimeError with nvcc's output on failure."""
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, '_build')
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace('.cu', '.o'))
        cmd = [_nvcc(), *NVCC_FLAGS, *extra_flags, '-I', INCLUDE, '-I', CSRC, '-c',
               os.path.join(CSRC, src), '-o', obj]
        if verbose:
            print(' '.join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError('nvcc failed on %s:\n%s%s' % (src, r.stdout, r.stderr))
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr)
        objs.append(obj)
    tmp = LIB + '.tmp'
    cmd = [_nvcc(), '-shared', '-gencode', 'arch=compute_100a,code=sm_100a', *objs, '-o', tmp,
           '-lcudart']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('link failed:\n%s%s' % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    flags = sys.argv[1:]
    print(build(force=True, verbose=True, extra_flags=flags))
