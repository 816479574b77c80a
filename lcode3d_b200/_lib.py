"""ctypes binding of liblc3d.so (declarations in include/lc3d.h).

The library is the product: if it is missing this module raises at import
time, and nothing in the package falls back to a CPU implementation.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'liblc3d.so')

c_int, c_double, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p

OK, ERR_PARAM, ERR_CUDA, ERR_WINDOW, ERR_NONFINITE, ERR_STATE, ERR_SIZE, ERR_TIMEOUT = range(8)
PREC_FP64, PREC_MIXED, PREC_FFT32, PREC_TF32 = 0, 1, 2, 3
FP64_AUTO, FP64_FFT, FP64_DENSE = 0, 1, 2


class Params(ctypes.Structure):
    _fields_ = [('grid_steps', c_int),
                ('grid_step_size', c_double),
                ('xi_step_size', c_double),
                ('plasma_coarseness', c_int),
                ('plasma_fineness', c_int),
                ('reflect_padding_steps', c_int),
                ('plasma_padding_steps', c_int),
                ('field_solver_subtraction_trick', c_double),
                ('field_solver_variant_A', c_int),
                ('precision', c_int),
                ('fp64_transform', c_int),
                ('mixed_slices', c_int)]


STATE_NAMES = ('x_offt', 'y_offt', 'px', 'py', 'pz', 'Ex', 'Ey', 'Ez',
               'Bx', 'By', 'Bz', 'ro', 'jx', 'jy', 'jz')
CONST_NAMES = ('m', 'q', 'x_init', 'y_init', 'ro_initial')
VIRT_NAMES = ('influence_prev', 'influence_next', 'indices_prev',
              'indices_next', 'fine_grid')


class StatePtrs(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in STATE_NAMES]


class ConstPtrs(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in CONST_NAMES]


class VirtPtrs(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in VIRT_NAMES]


class BeamParams(ctypes.Structure):
    _fields_ = [('amplitude', c_double), ('sigma_r', c_double), ('length_factor', c_double)]


# (name, restype, argtypes) of every exported entry point
P = c_void_p
SIGNATURES = [
    ('lc3d_sizes', c_int, [ctypes.POINTER(Params), ctypes.POINTER(c_int),
                           ctypes.POINTER(c_int), ctypes.POINTER(c_double)]),
    ('lc3d_create', c_int, [ctypes.POINTER(Params), c_int, ctypes.POINTER(c_void_p)]),
    ('lc3d_destroy', c_int, [P]),
    ('lc3d_strerror', ctypes.c_char_p, [c_int]),
    ('lc3d_set_const', c_int, [P, ctypes.POINTER(ConstPtrs), ctypes.POINTER(VirtPtrs), P]),
    ('lc3d_set_state', c_int, [P, ctypes.POINTER(StatePtrs), P]),
    ('lc3d_get_state', c_int, [P, ctypes.POINTER(StatePtrs), P]),
    ('lc3d_step', c_int, [P, P, P]),
    ('lc3d_step_arrays', c_int, [P, ctypes.POINTER(StatePtrs), ctypes.POINTER(StatePtrs), P, P]),
    ('lc3d_step_arrays_host_beam', c_int, [P, ctypes.POINTER(StatePtrs), ctypes.POINTER(StatePtrs), P, P]),
    ('lc3d_move_estimate_wo_fields', c_int, [P] * 12),
    ('lc3d_move_smart', c_int, [P] * 24),
    ('lc3d_deposit', c_int, [P] * 14),
    ('lc3d_calculate_Ex_Ey_Bx_By', c_int, [P] * 17),
    ('lc3d_calculate_Ez', c_int, [P] * 5),
    ('lc3d_calculate_Bz', c_int, [P] * 5),
    ('lc3d_check_error', c_int, [P, P]),
    ('lc3d_test_wait_limit', c_int, [P, ctypes.c_longlong, c_int]),
    ('lc3d_set_tiles', c_int, [P, c_int, c_int]),
    ('lc3d_profile', c_int, [P, c_int]),
    ('lc3d_profile_read', c_int, [P, P, P, P]),
    ('lc3d_deposit_noalloc', c_int, [ctypes.POINTER(Params)] + [P] * 18),
    ('lc3d_set_beam', c_int, [P, ctypes.POINTER(BeamParams)]),
    ('lc3d_run', c_int, [P, c_int, c_int, P, P]),
    ('lc3d_batch_create', c_int, [P, c_int, ctypes.POINTER(c_void_p)]),
    ('lc3d_batch_run', c_int, [P, P, c_int, P, P]),
    ('lc3d_batch_destroy', c_int, [P]),
    ('lc3d_batch_set_mode', c_int, [P, c_int]),
    ('lc3d_beam_eval', c_int, [P, c_int, P, P]),
    ('lc3d_diag_zn', c_int, [P, P, P, P]),
    ('lc3d_init_plasma', c_int, [P, P]),
    ('lc3d_get_const', c_int, [P] * 12),
    ('lc3d_step_arrays_first_pass', c_int, [P, ctypes.POINTER(StatePtrs), ctypes.POINTER(StatePtrs), P, P, P]),
    ('lc3d_step_arrays_predicted', c_int, [P, ctypes.POINTER(StatePtrs), ctypes.POINTER(StatePtrs), P, P, P, P]),
    ('lc3d_fields_rel_diff', c_int, [P, P, P, P, P]),
    ('lc3d_predictor_num_params', ctypes.c_longlong, []),
    ('lc3d_predictor_create', c_int, [c_int, c_int, ctypes.POINTER(c_void_p)]),
    ('lc3d_predictor_destroy', c_int, [P]),
    ('lc3d_predictor_set_params', c_int, [P, P, P]),
    ('lc3d_predictor_get_params', c_int, [P, P, P]),
    ('lc3d_predictor_get_grad', c_int, [P, P, P]),
    ('lc3d_predictor_set_scales', c_int, [P, P, P]),
    ('lc3d_predictor_pack', c_int, [P, P, P, P]),
    ('lc3d_predictor_forward', c_int, [P, P]),
    ('lc3d_predictor_predict', c_int, [P, P, P, P, P]),
    ('lc3d_predictor_set_target', c_int, [P, P, P, P, P]),
    ('lc3d_predictor_backward', c_int, [P, P, P]),
    ('lc3d_predictor_adam', c_int, [P, ctypes.c_float, P]),
    ('lc3d_predictor_tensor', c_int, [P, c_int, ctypes.POINTER(c_void_p), ctypes.POINTER(ctypes.c_longlong)]),
    ('lc3d_predictor_check_error', c_int, [P, P]),
]

PRED_INPUT, PRED_OUTPUT, PRED_TARGET = 0, 1, 2

STAGES = ('move', 'deposit', 'deposit_finalize', 'rhs', 'transform', 'field_finalize', 'slice', 'other')


class LC3DError(RuntimeError):
    """A liblc3d call returned a non-zero status."""

    def __init__(self, code, where):
        self.code = code
        super().__init__(f'{where}: {strerror(code)} (code {code})')


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f'{LIB_PATH} is missing: build it with `python lcode3d_b200/build.py` '
            '(nvcc, sm_100a). There is no CPU fallback.')
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def strerror(code):
    return lib.lc3d_strerror(code).decode()


def check(code, where):
    if code != OK:
        raise LC3DError(code, where)
