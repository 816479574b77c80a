"""Drop-in host interface of the B200 LCODE 3D xi-step solver.

Mirrors the public functions of the reference ``lcode.py`` (same names,
same arguments, same returned attribute names) so that the reference's CLI
loop (lcode.py:1032-1051) or embedding code can switch to it:

    init(config) -> (xs, ys, const, virt_params, state)        lcode.py:936-975
    step(config, const, virt_params, prev, beam_ro) -> state    lcode.py:828-931

plus the stage functions ``step`` is made of (``move_estimate_wo_fields``,
``move_smart``, ``deposit``, ``initial_deposition``, ``calculate_Ex_Ey_Bx_By``,
``calculate_Ez``, ``calculate_Bz``). Device arrays are torch CUDA float64
tensors (cupy arrays in the reference); ``GPUArraysView`` copies to numpy on
attribute access like the reference's. All device work runs in liblc3d.so
(include/lc3d.h) on the current torch stream; there is no CPU fallback.

Extra, optional config attributes (absent in the reference's config):
``lc3d_precision`` = 'fp64' (default), 'mixed' (split-bf16 tensor-core
transforms), 'tf32' (split-tf32 tensor-core transforms) or 'fft32' (float32
FFT transforms; right-hand sides, fields, averaging and particles in
float64);
``lc3d_fp64_transform`` = 'auto' (default: FFT where 2(N-1) factors into
2, 3, 5), 'fft' or 'dense' (DGEMM-form transform matrices);
``lc3d_mixed_slices`` = slices per operand of the tensor-core transforms
(1..6; default 4 for 'mixed', 3 for 'tf32').
"""
import ctypes
import operator
import sys

import numpy as np
import torch

from . import _lib
from ._lib import lib, check

ELECTRON_CHARGE = -1
ELECTRON_MASS = 1
WARP_SIZE = 32

#: read the device error flag after every step()/stage call (one host sync);
#: the reference has no such check and silently corrupts memory instead
check_errors = True


# ---------------------------------------------------------------------------
# Array groups (lcode.py:52-119)
# ---------------------------------------------------------------------------

_cuda_seen = False   # a CUDA device was found once; availability does not go away


def _device():
    global _cuda_seen
    if not _cuda_seen:
        if not torch.cuda.is_available():
            raise RuntimeError('lcode3d_b200 needs a CUDA device (B200, sm_100a); '
                               'there is no CPU fallback')
        _cuda_seen = True
    return torch.device('cuda', torch.cuda.current_device())


def to_device(a, dtype=None):
    """Like ``cp.asarray``: a contiguous device tensor (float64 unless the
    input is an integer array)."""
    dev = _device()
    if isinstance(a, torch.Tensor):
        t = a
    else:
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(a)))
    if dtype is None:
        dtype = t.dtype if not t.dtype.is_floating_point else torch.float64
        if dtype in (torch.int32, torch.int16, torch.int8, torch.uint8, torch.bool):
            dtype = torch.int64
    return t.to(device=dev, dtype=dtype).contiguous()


class GPUArrays:
    """Named group of device arrays (lcode.py:52-69)."""

    def __init__(self, **kwargs):
        for name, array in kwargs.items():
            setattr(self, name, to_device(array))


class GPUArraysView:
    """Attribute access copies device -> host numpy; assignment copies
    host -> device (lcode.py:73-119)."""

    def __init__(self, gpu_arrays):
        super().__setattr__('_arrs', gpu_arrays)

    def __dir__(self):
        return list(set(super().__dir__() + dir(self._arrs)))

    def __getattr__(self, attrname):
        return getattr(self._arrs, attrname).cpu().numpy()

    def __setattr__(self, attrname, value):
        t = getattr(self._arrs, attrname)
        t.copy_(torch.as_tensor(np.asarray(value), dtype=t.dtype))


# ---------------------------------------------------------------------------
# Per-config solver context (replaces the cp.memoize caches of the
# reference, lcode.py:144, 215, 316)
# ---------------------------------------------------------------------------

def _precision(config):
    p = getattr(config, 'lc3d_precision', 'fp64')
    if p in ('fp64', _lib.PREC_FP64):
        return _lib.PREC_FP64
    if p in ('mixed', _lib.PREC_MIXED):
        return _lib.PREC_MIXED
    if p in ('fft32', _lib.PREC_FFT32):
        return _lib.PREC_FFT32
    if p in ('tf32', _lib.PREC_TF32):
        return _lib.PREC_TF32
    raise ValueError(f'lc3d_precision must be "fp64", "mixed", "fft32" or "tf32", not {p!r}')


def _fp64_transform(config):
    t = getattr(config, 'lc3d_fp64_transform', 'auto')
    table = {'auto': _lib.FP64_AUTO, 'fft': _lib.FP64_FFT, 'dense': _lib.FP64_DENSE}
    if t not in table:
        raise ValueError(f'lc3d_fp64_transform must be one of {sorted(table)}, not {t!r}')
    return table[t]


def params_of(config):
    p = _lib.Params()
    p.grid_steps = int(config.grid_steps)
    p.grid_step_size = float(config.grid_step_size)
    p.xi_step_size = float(config.xi_step_size)
    p.plasma_coarseness = int(config.plasma_coarseness)
    p.plasma_fineness = int(config.plasma_fineness)
    p.reflect_padding_steps = int(config.reflect_padding_steps)
    p.plasma_padding_steps = int(config.plasma_padding_steps)
    p.field_solver_subtraction_trick = float(config.field_solver_subtraction_trick)
    p.field_solver_variant_A = int(bool(config.field_solver_variant_A))
    p.precision = _precision(config)
    p.fp64_transform = _fp64_transform(config)
    p.mixed_slices = int(getattr(config, 'lc3d_mixed_slices', 0))
    return p


def _key(p, device):
    return tuple(getattr(p, f) for f, _ in p._fields_) + (device,)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class Solver:
    """One liblc3d context: owns the device workspaces and copies of const
    and virt_params for one configuration on one device."""

    def __init__(self, params, device):
        self.params = params
        self.device = device
        self.ctx = ctypes.c_void_p()
        check(lib.lc3d_create(ctypes.byref(params), device, ctypes.byref(self.ctx)),
              'lc3d_create')
        nc, nf, rb = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check(lib.lc3d_sizes(ctypes.byref(params), ctypes.byref(nc), ctypes.byref(nf),
                             ctypes.byref(rb)), 'lc3d_sizes')
        self.N, self.Nc, self.Nf, self.reflect_boundary = params.grid_steps, nc.value, nf.value, rb.value
        self.out_pool = _StatePool()
        self._const_arrays = None
        self._virt_arrays = None
        self._keep = ()

    def __del__(self):
        ctx = getattr(self, 'ctx', None)
        if ctx and ctx.value and lib is not None:
            lib.lc3d_destroy(ctx)
            self.ctx = None

    # -- constants ----------------------------------------------------------
    @staticmethod
    def _unchanged(arrays, seen):
        """The same array objects as last time, none written since (torch
        counts every in-place write of a tensor or of a view of it in
        ``_version``): nothing to copy. The solver holds the arrays, so their
        storage cannot have been freed and reused meanwhile. (map / attrgetter
        keep the per-step check in C: it runs on every step() call.)"""
        return (seen is not None and all(map(operator.is_, arrays, seen[0]))
                and list(map(_VERSION, arrays)) == seen[1])

    @staticmethod
    def _seen(arrays):
        return arrays, list(map(_VERSION, arrays))

    def set_virt(self, virt):
        arrays = _GET_VIRT(virt)
        if self._unchanged(arrays, self._virt_arrays):
            return
        ip = getattr(virt, 'indices_prev').to(torch.int32).contiguous()
        inn = getattr(virt, 'indices_next').to(torch.int32).contiguous()
        v = _lib.VirtPtrs(virt.influence_prev.data_ptr(), virt.influence_next.data_ptr(),
                          ip.data_ptr(), inn.data_ptr(), virt.fine_grid.data_ptr())
        check(lib.lc3d_set_const(self.ctx, None, ctypes.byref(v), _stream()), 'lc3d_set_const')
        self._keep = (ip, inn)   # alive until the stream-ordered copy ran
        torch.cuda.current_stream().synchronize()
        self._virt_arrays = self._seen(arrays)

    def set_const(self, const):
        arrays = _GET_CONST(const)
        if self._unchanged(arrays, self._const_arrays):
            return
        c = _lib.ConstPtrs(*[getattr(const, n).data_ptr() for n in _lib.CONST_NAMES])
        check(lib.lc3d_set_const(self.ctx, ctypes.byref(c), None, _stream()), 'lc3d_set_const')
        self._const_arrays = self._seen(arrays)

    def check_device_flag(self, where):
        if check_errors:
            check(lib.lc3d_check_error(self.ctx, _stream()), where)


_GET_VIRT = operator.attrgetter(*_lib.VIRT_NAMES)
_GET_CONST = operator.attrgetter(*_lib.CONST_NAMES)
_GET_STATE = operator.attrgetter(*_lib.STATE_NAMES)
_VERSION = operator.attrgetter('_version')   # const / virt_params arrays are torch tensors

_solvers = {}
_solvers_raw = {}   # (raw config attribute values, device) -> Solver: skips params_of per call
_CFG_ATTRS = ('grid_steps', 'grid_step_size', 'xi_step_size', 'plasma_coarseness', 'plasma_fineness',
              'reflect_padding_steps', 'plasma_padding_steps', 'field_solver_subtraction_trick',
              'field_solver_variant_A')
_CFG_OPTIONAL = (('lc3d_precision', 'fp64'), ('lc3d_fp64_transform', 'auto'), ('lc3d_mixed_slices', 0))


def solver_for(config):
    """The cached Solver of this configuration on the current device."""
    raw = None
    if _cuda_seen or torch.cuda.is_available():
        raw = (tuple(getattr(config, n, None) for n in _CFG_ATTRS) +
               tuple(getattr(config, n, d) for n, d in _CFG_OPTIONAL) + (torch.cuda.current_device(),))
        try:
            s = _solvers_raw.get(raw)
        except TypeError:   # an unhashable attribute value: take the full path
            raw, s = None, None
        if s is not None:
            return s
    p = params_of(config)
    dev = _device().index
    k = _key(p, dev)
    s = _solvers.get(k)
    if s is None:
        s = _solvers[k] = Solver(p, dev)
    if raw is not None:
        _solvers_raw[raw] = s
    return s


def _grid(config):
    N = config.grid_steps
    return (N, N)


def _zeros(shape):
    return torch.zeros(shape, dtype=torch.float64, device=_device())


def _empty(shape):
    return torch.empty(shape, dtype=torch.float64, device=_device())


def _f64(a, shape=None):
    t = to_device(a, torch.float64)
    if shape is not None and tuple(t.shape) != tuple(shape):
        t = t.expand(shape).contiguous()
    return t


def _state_arrays(state, shape_p, g, dev):
    """The 15 state arrays of ``state`` as contiguous float64 tensors on
    ``dev``; arrays that already are (the usual case: the previous step's
    output) are used as they are, without a conversion call."""
    out = []
    for k, n in enumerate(_lib.STATE_NAMES):
        t = getattr(state, n)
        shape = shape_p if k < 5 else g
        if not (isinstance(t, torch.Tensor) and t.dtype == torch.float64 and t.device == dev and
                t.is_contiguous() and tuple(t.shape) == shape):
            t = _f64(t, shape)
        out.append(t)
    return out


_use_count = getattr(torch._C, '_storage_Use_Count', None)


class _StatePool:
    """Output states of ``step`` kept for reuse (per Solver). An entry (a
    GPUArrays, its 15 arrays and their StatePtrs) is handed out again only
    when nothing outside the pool refers to it:

    * the CPython reference counts of the object and of its 15 arrays are
      back at the values taken when the entry was made, and
    * the use count of the entry's one device allocation (every tensor that
      shares the memory: slices and views such as ``state.Ez[i, j]``, a
      DLPack export) is back at its value then.

    That is the state before last in the reference's loop
    (``state = step(..., state, ...)``), which the caller has dropped. A
    reused state is the same Python object, with the new step's values;
    states the caller keeps, or keeps any view of, are never touched. Saves
    the allocation and the 15 array objects of a step. Without a storage use
    count in this torch build nothing is reused."""

    SIZE = 3

    def __init__(self):
        self.entries = []

    @staticmethod
    def _counts(e):
        return sys.getrefcount(e[0]), list(map(sys.getrefcount, e[1])), _use_count(e[5])

    @staticmethod
    def _free(e):
        """The counts of entry e are back at their baseline e[3], taken the
        same way as _counts, the object's own count first (an entry in use
        usually fails there)."""
        base = e[3]
        return (sys.getrefcount(e[0]) == base[0] and list(map(sys.getrefcount, e[1])) == base[1]
                and _use_count(e[5]) == base[2])

    def ptrs_of(self, state):
        """The StatePtrs of `state` if it is one of the pool's states with
        all 15 arrays still its own (else None)."""
        for e in self.entries:
            if e[0] is state:
                return e[2] if all(map(operator.is_, _GET_STATE(state), e[1])) else None
        return None

    def take(self, shape_p, g, dev):
        for e in self.entries:
            if e[4] == (shape_p, g, dev) and self._free(e):
                return e
        arrays = tuple(_new_state_arrays(shape_p, g, dev))
        obj = GPUArrays.__new__(GPUArrays)
        for n, t in zip(_lib.STATE_NAMES, arrays):
            setattr(obj, n, t)
        # the storage object only lends its handle: the pool's arrays keep the allocation alive
        e = [obj, arrays, _lib.StatePtrs(*[t.data_ptr() for t in arrays]), None, (shape_p, g, dev),
             arrays[0].untyped_storage()._cdata]
        del obj, arrays, n, t
        if len(self.entries) < self.SIZE and _use_count is not None:
            self.entries.append(e)
            e[3] = self._counts(e)
        return e


def _new_state_arrays(shape_p, g, dev):
    """Uninitialised output arrays of one step: views of ONE allocation (one
    allocator call instead of 15), each starting on a 256-byte boundary.
    The allocation lives while any of its arrays does."""
    n_p, n_g = shape_p[0] * shape_p[1], g[0] * g[1]
    pad = lambda n: (n + 31) // 32 * 32   # float64 words to a 256-byte multiple
    sizes = [pad(n_p)] * 5 + [pad(n_g)] * 10
    parts = torch.empty(sum(sizes), dtype=torch.float64, device=dev).split(sizes)
    return [p[:n_p].view(shape_p) if k < 5 else p[:n_g].view(g) for k, p in enumerate(parts)]


# ---------------------------------------------------------------------------
# Field solvers (lcode.py:160-184, 246-290, 333-364)
# ---------------------------------------------------------------------------

def calculate_Ez(config, jx, jy):
    """Ez from the Dirichlet Poisson problem (lcode.py:160-184)."""
    s = solver_for(config)
    jx, jy = _f64(jx), _f64(jy)
    Ez = _empty(_grid(config))
    check(lib.lc3d_calculate_Ez(s.ctx, _ptr(jx), _ptr(jy), _ptr(Ez), _stream()), 'calculate_Ez')
    s.check_device_flag('calculate_Ez')
    return Ez


def calculate_Ex_Ey_Bx_By(config, Ex_avg, Ey_avg, Bx_avg, By_avg,
                          beam_ro, ro, jx, jy, jz, jx_prev, jy_prev):
    """Transverse fields from the Helmholtz (subtraction trick) or Laplace
    problems with mixed boundary conditions (lcode.py:246-290)."""
    s = solver_for(config)
    g = _grid(config)
    args = [_f64(a, g) for a in (Ex_avg, Ey_avg, Bx_avg, By_avg, beam_ro, ro, jx, jy, jz,
                                 jx_prev, jy_prev)]
    out = [_empty(g) for _ in range(4)]
    check(lib.lc3d_calculate_Ex_Ey_Bx_By(s.ctx, *[_ptr(a) for a in args],
                                         *[_ptr(o) for o in out], _stream()),
          'calculate_Ex_Ey_Bx_By')
    s.check_device_flag('calculate_Ex_Ey_Bx_By')
    return tuple(out)


def calculate_Bz(config, jx, jy):
    """Bz from the Neumann Poisson problem, mean removed (lcode.py:333-364)."""
    s = solver_for(config)
    jx, jy = _f64(jx), _f64(jy)
    Bz = _empty(_grid(config))
    check(lib.lc3d_calculate_Bz(s.ctx, _ptr(jx), _ptr(jy), _ptr(Bz), _stream()), 'calculate_Bz')
    s.check_device_flag('calculate_Bz')
    return Bz


# ---------------------------------------------------------------------------
# Particles (lcode.py:369-391, 576-689, 692-699, 704-823)
# ---------------------------------------------------------------------------

def move_estimate_wo_fields(config, m, x_init, y_init, prev_x_offt, prev_y_offt, px, py, pz):
    """Field-free drift with coordinate reflection (lcode.py:369-391)."""
    s = solver_for(config)
    shape = tuple(to_device(prev_x_offt).shape)
    a = [_f64(v, shape) for v in (m, x_init, y_init, prev_x_offt, prev_y_offt, px, py, pz)]
    ox, oy = _empty(shape), _empty(shape)
    check(lib.lc3d_move_estimate_wo_fields(s.ctx, *[_ptr(v) for v in a], _ptr(ox), _ptr(oy),
                                           _stream()), 'move_estimate_wo_fields')
    return ox, oy


def move_smart(config, m, q, x_init, y_init, x_prev_offt, y_prev_offt,
               estimated_x_offt, estimated_y_offt, px_prev, py_prev, pz_prev,
               Ex_avg, Ey_avg, Ez_avg, Bx_avg, By_avg, Bz_avg):
    """Pusher with half-step TSC field interpolation (lcode.py:704-823)."""
    s = solver_for(config)
    shape = tuple(to_device(x_prev_offt).shape)
    part = [_f64(v, shape) for v in (m, q, x_init, y_init, x_prev_offt, y_prev_offt,
                                     estimated_x_offt, estimated_y_offt, px_prev, py_prev, pz_prev)]
    g = _grid(config)
    fields = [_f64(v, g) for v in (Ex_avg, Ey_avg, Ez_avg, Bx_avg, By_avg, Bz_avg)]
    out = [_empty(shape) for _ in range(5)]
    check(lib.lc3d_move_smart(s.ctx, *[_ptr(v) for v in part + fields],
                              *[_ptr(o) for o in out], _stream()), 'move_smart')
    s.check_device_flag('move_smart')
    return tuple(out)


def deposit(config, ro_initial, x_offt, y_offt, m, q, px, py, pz, virt_params):
    """Coarse->fine interpolation and deterministic TSC deposition of rho,
    jx, jy, jz, plus ro_initial (lcode.py:666-689)."""
    s = solver_for(config)
    s.set_virt(virt_params)
    shape = tuple(to_device(x_offt).shape)
    part = [_f64(v, shape) for v in (x_offt, y_offt, m, q, px, py, pz)]
    g = _grid(config)
    roi = None
    if not (np.isscalar(ro_initial) and ro_initial == 0):
        roi = _f64(ro_initial, g)
    out = [_empty(g) for _ in range(4)]
    check(lib.lc3d_deposit(s.ctx, _ptr(roi), *[_ptr(v) for v in part],
                           *[_ptr(o) for o in out], _stream()), 'deposit')
    s.check_device_flag('deposit')
    return tuple(out)


def initial_deposition(config, x_offt, y_offt, px, py, pz, m, q, virt_params):
    """Ion background = minus the initial electron density (lcode.py:692-699)."""
    ro_electrons_initial, _, _, _ = deposit(config, 0, x_offt, y_offt, m, q, px, py, pz,
                                            virt_params)
    return -ro_electrons_initial


# ---------------------------------------------------------------------------
# Plasma layout (lcode.py:454-573), host side: runs once per simulation
# ---------------------------------------------------------------------------

def make_coarse_plasma_grid(steps, step_size, coarseness=3):
    """Coarse lattice, symmetric about 0 (lcode.py:454-465)."""
    assert coarseness == int(coarseness)
    half = np.arange(steps // (coarseness * 2)) * (step_size * coarseness)
    grid = np.concatenate([-half[:0:-1], half])
    assert np.array_equal(grid, -grid[::-1])
    return grid


def make_fine_plasma_grid(steps, step_size, fineness=2):
    """Fine lattice avoiding cell edges (lcode.py:468-487)."""
    assert fineness == int(fineness)
    d = step_size / fineness
    if fineness % 2:
        half = np.arange(steps // 2 * fineness) * d
        grid = np.concatenate([-half[:0:-1], half])
    else:
        half = (.5 + np.arange(steps // 2 * fineness)) * d
        grid = np.concatenate([-half[::-1], half])
    assert np.array_equal(grid, -grid[::-1])
    return grid


def make_plasma(steps, cell_size, coarseness=3, fineness=2):
    """Coarse particles and the coarse->fine interpolation parameters
    (lcode.py:490-573)."""
    coarse = make_coarse_plasma_grid(steps, cell_size, coarseness)
    fine = make_fine_plasma_grid(steps, cell_size, fineness)
    Nc = len(coarse)
    zeros = np.zeros((Nc, Nc))
    x_init = np.broadcast_to(coarse[:, None], (Nc, Nc))
    y_init = np.broadcast_to(coarse[None, :], (Nc, Nc))
    m = np.full((Nc, Nc), float(ELECTRON_MASS * coarseness ** 2))
    q = np.full((Nc, Nc), float(ELECTRON_CHARGE * coarseness ** 2))
    pos = np.searchsorted(coarse, fine)
    nxt = np.clip(pos, 0, Nc - 1)
    prv = np.clip(pos - 1, 0, Nc - 1)
    inf_prev = (coarse[nxt] - fine) / (cell_size * coarseness)
    inf_next = (fine - coarse[prv]) / (cell_size * coarseness)
    inf_prev[nxt == 0] = 0
    inf_next[nxt == 0] = 1
    inf_next[prv == Nc - 1] = 0
    inf_prev[prv == Nc - 1] = 1
    virt = GPUArrays(influence_prev=inf_prev, influence_next=inf_next,
                     indices_prev=prv, indices_next=nxt, fine_grid=fine)
    dev = [to_device(a) for a in (x_init, y_init, zeros, zeros, zeros, zeros, zeros, m, q)]
    return (*dev, virt)


# ---------------------------------------------------------------------------
# The xi step and init (lcode.py:828-975)
# ---------------------------------------------------------------------------

def _beam(config, beam_ro):
    if isinstance(beam_ro, (int, float)) and beam_ro == 0:
        return None
    return _f64(beam_ro, _grid(config))


def _host_beam(config, beam_ro):
    """The beam as a contiguous float64 host array of N x N (None for a
    device array or the scalar 0)."""
    if isinstance(beam_ro, (int, float)) and beam_ro == 0:
        return None
    if isinstance(beam_ro, torch.Tensor):
        if beam_ro.is_cuda:
            return None
        if (beam_ro.dtype == torch.float64 and beam_ro.dim() == 2 and beam_ro.shape[0] == config.grid_steps
                and beam_ro.shape[1] == config.grid_steps and beam_ro.is_contiguous()):
            return beam_ro   # already what the C call takes (e.g. a pinned beam buffer)
        t = beam_ro.to(torch.float64)
    else:
        t = torch.from_numpy(np.asarray(beam_ro, dtype=np.float64))
    g = _grid(config)
    if tuple(t.shape) != g:
        t = t.expand(g)
    return t.contiguous()


def step(config, const, virt_params, prev, beam_ro):
    """One xi step: estimate, predictor, corrector, final move and deposit
    (lcode.py:828-931). Returns a new GPUArrays; ``prev`` is not modified.
    A beam given in host memory (the reference's loop evaluates it with
    numpy) is copied to the device during the step's first deposition
    (lc3d_step_arrays_host_beam)."""
    s = solver_for(config)
    s.set_virt(virt_params)
    s.set_const(const)
    hb = _host_beam(config, beam_ro)
    beam = None if hb is not None else _beam(config, beam_ro)
    shape_p = tuple(prev.x_offt.shape)
    g = _grid(config)
    dev = _device()
    sp = s.out_pool.ptrs_of(prev)   # the previous step's output: its arrays are known
    if sp is None:
        prev_t = _state_arrays(prev, shape_p, g, dev)
        sp = _lib.StatePtrs(*[t.data_ptr() for t in prev_t])
    e = s.out_pool.take(shape_p, g, dev)
    so = e[2]
    if hb is not None:
        check(lib.lc3d_step_arrays_host_beam(s.ctx, ctypes.byref(sp), ctypes.byref(so),
                                             ctypes.c_void_p(hb.data_ptr()), _stream()), 'step')
        s._host_beam_keep = hb   # read by the copy until the next call on this context
    else:
        check(lib.lc3d_step_arrays(s.ctx, ctypes.byref(sp), ctypes.byref(so), _ptr(beam), _stream()),
              'step')
    s.check_device_flag('step')
    return e[0]


def run(config, const, virt_params, state, xi0, nsteps, beam=None):
    """Advance ``state`` by ``nsteps`` xi steps starting at xi index ``xi0``
    with the beam evaluated on the device, each step a CUDA-graph replay
    (lc3d_run). ``beam`` = (amplitude, sigma_r, length_factor) of the
    axisymmetric driver rho_b = A exp(-r^2 / (2 sigma_r^2)) 0.5
    (1 - cos(sqrt(pi/2) xi / L)) on 0 <= xi <= 2 sqrt(2 pi) L, or None for no
    beam. Returns (new state, Ez(N/2, N/2) after every step as a device
    tensor). Replaces the reference's host loop (lcode.py:1039-1046) for
    this beam shape; ``prev`` is not modified."""
    s = solver_for(config)
    s.set_virt(virt_params)
    s.set_const(const)
    g = _grid(config)
    shape_p = tuple(state.x_offt.shape)
    src = [_f64(getattr(state, n), shape_p if k < 5 else g) for k, n in enumerate(_lib.STATE_NAMES)]
    check(lib.lc3d_set_state(s.ctx, ctypes.byref(_lib.StatePtrs(*[t.data_ptr() for t in src])), _stream()),
          'lc3d_set_state')
    bp = None
    if beam is not None:
        bp = _lib.BeamParams(*[float(v) for v in beam])
    check(lib.lc3d_set_beam(s.ctx, ctypes.byref(bp) if bp is not None else None), 'lc3d_set_beam')
    ez = _empty((max(int(nsteps), 1),))
    check(lib.lc3d_run(s.ctx, int(xi0), int(nsteps), _ptr(ez), _stream()), 'lc3d_run')
    out = {n: _empty(shape_p if k < 5 else g) for k, n in enumerate(_lib.STATE_NAMES)}
    check(lib.lc3d_get_state(s.ctx, ctypes.byref(_lib.StatePtrs(*[out[n].data_ptr() for n in _lib.STATE_NAMES])),
                             _stream()), 'lc3d_get_state')
    s.check_device_flag('run')
    new = GPUArrays.__new__(GPUArrays)
    for n in _lib.STATE_NAMES:
        setattr(new, n, out[n])
    return new, ez[:nsteps]


# ---------------------------------------------------------------------------
# Checkpoint / resume: the arrays of const, virt_params and state under the
# reference's attribute names (lcode.py:926-929, 964-965, 566-570)
# ---------------------------------------------------------------------------

def save_checkpoint(path, xi_i, const, virt_params, state):
    """Write ``xi_i`` (the next xi index) and all arrays to an .npz file."""
    arrs = {'xi_i': np.array(int(xi_i))}
    for prefix, group, names in (('const_', const, _lib.CONST_NAMES),
                                 ('virt_', virt_params, _lib.VIRT_NAMES),
                                 ('state_', state, _lib.STATE_NAMES)):
        for n in names:
            arrs[prefix + n] = getattr(group, n).detach().cpu().numpy()
    np.savez(path, **arrs)


def load_checkpoint(path):
    """Read a file written by ``save_checkpoint``: (xi_i, const, virt_params,
    state) with device arrays, ready for ``step``."""
    with np.load(path) as f:
        const = GPUArrays(**{n: f['const_' + n] for n in _lib.CONST_NAMES})
        virt = GPUArrays(**{n: f['virt_' + n] for n in _lib.VIRT_NAMES})
        state = GPUArrays(**{n: f['state_' + n] for n in _lib.STATE_NAMES})
        return int(f['xi_i']), const, virt, state


def init(config):
    """Check the config, set config.reflect_boundary, lay out the plasma and
    deposit the ion background (lcode.py:936-975)."""
    assert config.grid_steps % 2 == 1
    assert config.reflect_padding_steps > config.plasma_coarseness + 1
    config.reflect_boundary = config.grid_step_size * (
        config.grid_steps / 2 - config.reflect_padding_steps)
    N = config.grid_steps
    grid = (np.arange(N) - N // 2) * config.grid_step_size
    xs, ys = grid[:, None], grid[None, :]
    x_init, y_init, x_offt, y_offt, px, py, pz, m, q, virt_params = make_plasma(
        N - config.plasma_padding_steps * 2, config.grid_step_size,
        coarseness=config.plasma_coarseness, fineness=config.plasma_fineness)
    ro_initial = initial_deposition(config, x_offt, y_offt, px, py, pz, m, q, virt_params)
    const = GPUArrays(m=m, q=q, x_init=x_init, y_init=y_init, ro_initial=ro_initial)
    z = lambda: _zeros((N, N))
    state = GPUArrays(x_offt=x_offt, y_offt=y_offt, px=px, py=py, pz=pz,
                      Ex=z(), Ey=z(), Ez=z(), Bx=z(), By=z(), Bz=z(),
                      ro=z(), jx=z(), jy=z(), jz=z())
    return xs, ys, const, virt_params, state


def init_config_checks(config):
    """The configuration checks of init() and config.reflect_boundary
    (lcode.py:941-949)."""
    assert config.grid_steps % 2 == 1
    assert config.reflect_padding_steps > config.plasma_coarseness + 1
    config.reflect_boundary = config.grid_step_size * (
        config.grid_steps / 2 - config.reflect_padding_steps)


def init_device(config):
    """init(config) with the plasma layout, the ion background and the
    initial state built on the device (lc3d_init_plasma); returns the same
    (xs, ys, const, virt_params, state), bit-identical to init()."""
    init_config_checks(config)
    N = config.grid_steps
    grid = (np.arange(N) - N // 2) * config.grid_step_size
    xs, ys = grid[:, None], grid[None, :]
    s = solver_for(config)
    check(lib.lc3d_init_plasma(s.ctx, _stream()), 'lc3d_init_plasma')
    Nc, Nf = s.Nc, s.Nf
    const = GPUArrays(m=_empty((Nc, Nc)), q=_empty((Nc, Nc)), x_init=_empty((Nc, Nc)), y_init=_empty((Nc, Nc)),
                      ro_initial=_empty((N, N)))
    ip = torch.empty(Nf, dtype=torch.int32, device=_device())
    inn = torch.empty(Nf, dtype=torch.int32, device=_device())
    virt = GPUArrays(influence_prev=_empty((Nf,)), influence_next=_empty((Nf,)), fine_grid=_empty((Nf,)))
    check(lib.lc3d_get_const(s.ctx, *[_ptr(t) for t in (const.m, const.q, const.x_init, const.y_init,
                                                         const.ro_initial, virt.influence_prev,
                                                         virt.influence_next, ip, inn, virt.fine_grid)],
                             _stream()), 'lc3d_get_const')
    virt.indices_prev = ip.to(torch.int64)
    virt.indices_next = inn.to(torch.int64)
    out = {n: _empty((Nc, Nc) if k < 5 else (N, N)) for k, n in enumerate(_lib.STATE_NAMES)}
    check(lib.lc3d_get_state(s.ctx, ctypes.byref(_lib.StatePtrs(*[out[n].data_ptr() for n in _lib.STATE_NAMES])),
                             _stream()), 'lc3d_get_state')
    state = GPUArrays.__new__(GPUArrays)
    for n in _lib.STATE_NAMES:
        setattr(state, n, out[n])
    return xs, ys, const, virt, state


# ---------------------------------------------------------------------------
# CLI loop (lcode.py:1032-1051) with the diagnostics line of
# lcode.py:979-1026: on-axis Ez, its peak drift and the zn noise figure (the
# PNG slices of lcode.py:1005-1013 are omitted: no plotting stack)
# ---------------------------------------------------------------------------

max_zn = 0.0


def diags_ro_zn(config, ro):
    """The running maximum of the density-noise figure (lcode.py:979-987):
    mean |ro - gaussian_filter(ro, sigma = 0.25 / h)| / 4.23045376e-04,
    computed on the device (lc3d_diag_zn); one scalar is read back."""
    global max_zn
    s = solver_for(config)
    g = _grid(config)
    r = _f64(ro, g)
    out = _empty((1,))
    check(lib.lc3d_diag_zn(s.ctx, _ptr(r), _ptr(out), _stream()), 'lc3d_diag_zn')
    max_zn = max(max_zn, float(out.item()))
    return max_zn


def diags_peak_msg(Ez_00_history):
    """Last on-axis Ez peak and its drift from the first peak
    (lcode.py:992-1002)."""
    a = np.asarray(Ez_00_history)
    if a.size < 3:
        return '...'
    inner = a[1:-1]
    peaks = np.nonzero((inner > a[:-2]) & (inner > a[2:]))[0] + 1
    if not peaks.size:
        return '...'
    v = a[peaks]
    dev = 100 * (v / v[0] - 1)
    return f'{v[-1]:0.4e} {dev[-1]:+0.2f}%'


def main():
    import config
    with torch.cuda.device(getattr(config, 'gpu_index', 0)):
        xs, ys, const, virt_params, state = init(config)
        Ez_00_history = []
        N = config.grid_steps
        for xi_i in range(config.xi_steps):
            beam_ro = config.beam(xi_i, xs, ys)
            state = step(config, const, virt_params, state, beam_ro)
            ez = float(state.Ez[N // 2, N // 2])
            Ez_00_history.append(ez)
            if xi_i % config.diagnostics_each_N_steps == 0 or xi_i == config.xi_steps - 1:
                xi = -xi_i * config.xi_step_size
                zn = diags_ro_zn(config, state.ro)
                print(f'xi={xi:+.4f} {ez:+.4e}|{diags_peak_msg(Ez_00_history)}|zn={zn:.3f}')
                sys.stdout.flush()


if __name__ == '__main__':
    main()
