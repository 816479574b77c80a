"""Build liblc3d.so (the C-ABI CUDA library) in-tree for sm_100a.

    python lcode3d_b200/build.py          # (importing the package needs the library)

The library is written next to this file so that it travels with the source
tree; nothing is installed into site-packages.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
LIB = os.path.join(HERE, 'liblc3d.so')

SOURCES = ['particles.cu', 'fields.cu', 'fields_fft.cu', 'fields_mixed.cu', 'run.cu', 'predictor.cu', 'diagnostics.cu', 'lc3d_api.cu']

NVCC_FLAGS = [
    '-gencode', 'arch=compute_100a,code=sm_100a',
    '-O3', '-lineinfo', '-std=c++17',
    '-shared', '-Xcompiler', '-fPIC',
    '-I', os.path.join(ROOT, 'include'),
]


def nvcc():
    cand = os.environ.get('NVCC') or os.path.join(
        os.environ.get('CUDA_HOME', '/usr/local/cuda'), 'bin', 'nvcc')
    return cand if os.path.exists(cand) else 'nvcc'


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(('.cuh', '.h'))]
    deps.append(os.path.join(ROOT, 'include', 'lc3d.h'))
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + ['-o', LIB + '.tmp'] + sources()
    if verbose:
        print(' '.join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(LIB + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True)
    print(LIB)
