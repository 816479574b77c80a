"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares; host-only entry points behave. CPU only."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT

HEADERS = sorted(glob.glob(os.path.join(ROOT, 'include', '*.h')))
LIB = os.path.join(ROOT, 'lcode3d_b200', 'liblc3d.so')


def declared_functions():
    names = []
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
        names += re.findall(r'\b(lc3d_\w+)\s*\(', src)
    return sorted(set(names))


@pytest.fixture(scope='module')
def lib():
    if not os.path.exists(LIB):
        from lcode3d_b200 import build
        build.build()
    return ctypes.CDLL(LIB)


def test_headers_declare_entry_points():
    names = declared_functions()
    for must in ('lc3d_create', 'lc3d_destroy', 'lc3d_step', 'lc3d_step_arrays',
                 'lc3d_set_state', 'lc3d_get_state', 'lc3d_strerror', 'lc3d_deposit',
                 'lc3d_move_smart', 'lc3d_move_estimate_wo_fields',
                 'lc3d_calculate_Ez', 'lc3d_calculate_Bz', 'lc3d_calculate_Ex_Ey_Bx_By'):
        assert must in names


def test_every_declared_symbol_is_exported(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from lcode3d_b200 import _lib
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(declared_functions()) <= bound


def _params(N=161, h=0.05, c=3, f=2, rpad=5, ppad=10):
    from lcode3d_b200 import _lib
    p = _lib.Params()
    p.grid_steps, p.grid_step_size, p.xi_step_size = N, h, 0.05
    p.plasma_coarseness, p.plasma_fineness = c, f
    p.reflect_padding_steps, p.plasma_padding_steps = rpad, ppad
    p.field_solver_subtraction_trick, p.field_solver_variant_A, p.precision = 1.0, 1, 0
    p.fp64_transform = 0
    p.mixed_slices = 0
    return p


@pytest.mark.parametrize('N,c,f', [(161, 3, 2), (641, 3, 2), (321, 3, 2), (481, 3, 2),
                                   (41, 3, 2), (61, 2, 3), (81, 4, 1)])
def test_sizes_match_plasma_layout(lib, N, c, f):
    """lc3d_sizes (host-only) against the oracle's plasma layout
    (lcode.py:454-487, 947-949)."""
    from lcode3d_b200 import _lib
    from oracle import lcode_oracle as O
    lib.lc3d_sizes.argtypes = [ctypes.POINTER(_lib.Params), ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
    h = 16 / (N - 1)
    p = _params(N, h, c, f, rpad=c + 2)
    nc, nf, rb = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    assert lib.lc3d_sizes(ctypes.byref(p), ctypes.byref(nc), ctypes.byref(nf), ctypes.byref(rb)) == 0
    steps = N - 20
    assert nc.value == len(O.make_coarse_plasma_grid(steps, h, c))
    assert nf.value == len(O.make_fine_plasma_grid(steps, h, f))
    assert rb.value == h * (N / 2 - (c + 2))


@pytest.mark.parametrize('bad', [dict(N=160), dict(rpad=4), dict(c=0), dict(N=21, ppad=10)])
def test_sizes_reject_bad_config(lib, bad):
    """The reference asserts odd grid_steps and reflect padding >
    coarseness + 1 (lcode.py:941, 944); the C ABI returns LC3D_ERR_PARAM."""
    from lcode3d_b200 import _lib
    kw = dict(N=161, c=3, f=2, rpad=5, ppad=10)
    kw.update(bad)
    p = _params(kw['N'], 0.05, kw['c'], kw['f'], kw['rpad'], kw['ppad'])
    lib.lc3d_sizes.argtypes = [ctypes.POINTER(_lib.Params), ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_void_p]
    assert lib.lc3d_sizes(ctypes.byref(p), None, None, None) == 1


@pytest.mark.parametrize('prec,ok', [(0, True), (1, True), (2, True), (3, True), (4, False), (-1, False)])
def test_sizes_check_precision(lib, prec, ok):
    """lc3d_params.precision: LC3D_PREC_FP64, _MIXED, _FFT32 and _TF32 are
    accepted, anything else is LC3D_ERR_PARAM (host-only check)."""
    from lcode3d_b200 import _lib
    p = _params()
    p.precision = prec
    lib.lc3d_sizes.argtypes = [ctypes.POINTER(_lib.Params), ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_void_p]
    assert lib.lc3d_sizes(ctypes.byref(p), None, None, None) == (0 if ok else 1)
    assert (_lib.PREC_FP64, _lib.PREC_MIXED, _lib.PREC_FFT32, _lib.PREC_TF32) == (0, 1, 2, 3)


def test_strerror(lib):
    lib.lc3d_strerror.restype = ctypes.c_char_p
    for code in range(8):
        assert lib.lc3d_strerror(code)
    assert b'stencil' in lib.lc3d_strerror(3)


def test_create_without_gpu_fails_cleanly(lib):
    """Without a device, lc3d_create returns LC3D_ERR_CUDA (no crash, no
    CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    from lcode3d_b200 import _lib
    p = _params()
    ctx = ctypes.c_void_p()
    lib.lc3d_create.argtypes = [ctypes.POINTER(_lib.Params), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    assert lib.lc3d_create(ctypes.byref(p), 0, ctypes.byref(ctx)) == 2
    assert not ctx.value


def test_python_interface_needs_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    import lcode3d_b200 as L
    from make_golden import make_config
    with pytest.raises(RuntimeError, match='CUDA'):
        L.init(make_config(41, 0.1, 0.05, 10, amplitude=0.3))


def declared_arity():
    """{function: number of parameters} from the prototypes in include/*.h."""
    out = {}
    for h in HEADERS:
        src = re.sub(r'/\*.*?\*/', '', open(h).read(), flags=re.S)
        for m in re.finditer(r'\b(lc3d_\w+)\s*\(([^;{]*?)\)\s*;', src):
            args = m.group(2).strip()
            out[m.group(1)] = 0 if args in ('', 'void') else args.count(',') + 1
    return out


def test_binding_arity_matches_header():
    """Every ctypes binding declares as many arguments as the C prototype."""
    from lcode3d_b200 import _lib
    ar = declared_arity()
    for name, _, argtypes in _lib.SIGNATURES:
        assert ar[name] == len(argtypes), (name, ar[name], len(argtypes))


def test_oracle_binding_arity():
    """The oracle's ctypes declarations match its C prototypes."""
    src = open(os.path.join(ROOT, 'oracle', 'lc3d_oracle.c')).read()
    from oracle import lcode_oracle as O
    O.use_c_kernels(1)
    try:
        for name in ('oracle_move_smart', 'oracle_deposit'):
            m = re.search(r'\bint ' + name + r'\(([^{]*?)\)\s*\{', src, flags=re.S)
            n = m.group(1).count(',') + 1
            assert len(getattr(O._C, name).argtypes) == n, name
    finally:
        O.use_numpy_kernels()
