"""Build the oracle's C restatement (test infrastructure) with gcc.

    python -m oracle.build

Output: oracle/liblc3d_oracle.so (git-ignored; built again on demand).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, 'lc3d_oracle.c')
LIB = os.path.join(HERE, 'liblc3d_oracle.so')
FLAGS = ['-O2', '-fPIC', '-shared', '-fopenmp', '-ffp-contract=off', '-fno-fast-math']


def _compilers():
    seen = []
    for c in ('/usr/bin/gcc', os.environ.get('CC'), 'gcc', 'cc'):
        if c and c not in seen:
            seen.append(c)
    return seen


def build(force=False, verbose=False):
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    last = None
    # prefer OpenMP (multi-core baseline); fall back to a serial build
    for flags in (FLAGS, [f for f in FLAGS if f != '-fopenmp']):
        for cc in _compilers():
            cmd = [cc] + flags + ['-o', LIB + '.tmp', SRC, '-lm']
            if verbose:
                print(' '.join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode == 0:
                os.replace(LIB + '.tmp', LIB)
                return LIB
            last = r.stderr
    raise RuntimeError('cannot build the oracle C library:\n' + (last or ''))


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True)
