"""Batched parameter scans: many independent LCODE 3D simulations advanced
together on one GPU, and partitioned across GPUs.

The reference runs one simulation per process (lcode.py:1032-1051). A scan
here is a set of simulations of possibly different grid sizes; every one
gets its own liblc3d context, and ``lc3d_batch_run`` advances all of them
with one CUDA-graph launch per xi step (each simulation's whole step on its
own branch of the graph, beam evaluated on the device, Ez(0,0) recorded on
the device). Across GPUs the simulations are partitioned by cost with no
exchange during the run; only the Ez(0,0) histories are gathered at the end.
"""
import ctypes
import types

import numpy as np
import torch

from . import _lib
from . import lcode as L
from ._lib import check, lib

GRIDS = (161, 321, 481, 641)


def scan_specs(count, seed, grids=GRIDS, window=16.0, xi_step=0.01):
    """Seeded draws of a scan: grid N uniform over ``grids`` with h chosen so
    the window stays ``window`` wide, beam amplitude log-uniform on
    [0.01, 1], sigma_r uniform on [0.5, 2], length factor uniform on
    [0.5, 1.5]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        N = int(rng.choice(grids))
        out.append(dict(grid_steps=N, grid_step_size=window / (N - 1), xi_step_size=xi_step,
                        amplitude=float(np.exp(rng.uniform(np.log(0.01), np.log(1.0)))),
                        sigma_r=float(rng.uniform(0.5, 2.0)),
                        length_factor=float(rng.uniform(0.5, 1.5))))
    return out


def cost(spec):
    """Relative cost of one xi step: the fine-particle and cell counts both
    grow with N^2."""
    return spec['grid_steps'] ** 2


def partition(specs, world):
    """Split simulation indices over ``world`` ranks, balancing the summed
    cost (longest-processing-time greedy; deterministic)."""
    order = sorted(range(len(specs)), key=lambda i: (-cost(specs[i]), i))
    loads = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += cost(specs[i])
    return [sorted(p) for p in parts]


def make_config(spec, precision='fp64', transform='auto', slices=0):
    """A config object with the reference's attributes for one scan member."""
    c = types.SimpleNamespace(
        grid_steps=spec['grid_steps'], grid_step_size=spec['grid_step_size'],
        xi_step_size=spec['xi_step_size'], xi_steps=10 ** 9, diagnostics_each_N_steps=10 ** 9,
        field_solver_subtraction_trick=1, field_solver_variant_A=True,
        reflect_padding_steps=5, plasma_padding_steps=10, plasma_coarseness=3, plasma_fineness=2,
        gpu_index=0, lc3d_precision=precision, lc3d_fp64_transform=transform,
        lc3d_mixed_slices=slices)
    A, sr, lf = spec['amplitude'], spec['sigma_r'], spec['length_factor']

    def beam(xi_i, x, y):
        xi = xi_i * c.xi_step_size
        if xi < 0 or xi > 2 * np.sqrt(2 * np.pi) * lf:
            return 0
        return A * np.exp(-(x ** 2 + y ** 2) / (2 * sr ** 2)) * 0.5 * (1 - np.cos(np.sqrt(np.pi / 2) * xi / lf))
    c.beam = beam
    return c


class Sim:
    """One scan member: its own context (not shared through the per-config
    cache of ``lcode``) with its plasma, ion background and initial state
    built on the device (lc3d_init_plasma)."""

    def __init__(self, spec, precision='fp64', transform='auto', slices=0, tiles=None):
        self.spec = spec
        self.config = make_config(spec, precision, transform, slices)
        L.init_config_checks(self.config)
        self.solver = L.Solver(L.params_of(self.config), L._device().index)
        if tiles:
            check(lib.lc3d_set_tiles(self.solver.ctx, int(tiles[0]), int(tiles[1])), 'lc3d_set_tiles')
        check(lib.lc3d_init_plasma(self.solver.ctx, L._stream()), 'lc3d_init_plasma')
        bp = _lib.BeamParams(spec['amplitude'], spec['sigma_r'], spec['length_factor'])
        check(lib.lc3d_set_beam(self.solver.ctx, ctypes.byref(bp)), 'lc3d_set_beam')
        self.xi = 0

    def state(self):
        """The current state as device arrays (a copy)."""
        N = self.spec['grid_steps']
        shape_p = (self.solver.Nc, self.solver.Nc)
        out = {n: L._empty(shape_p if k < 5 else (N, N)) for k, n in enumerate(_lib.STATE_NAMES)}
        check(lib.lc3d_get_state(self.solver.ctx,
                                 ctypes.byref(_lib.StatePtrs(*[out[n].data_ptr() for n in _lib.STATE_NAMES])),
                                 L._stream()), 'lc3d_get_state')
        st = L.GPUArrays.__new__(L.GPUArrays)
        for n in _lib.STATE_NAMES:
            setattr(st, n, out[n])
        return st


class Batch:
    """Simulations advanced together by ``lc3d_batch_run``."""

    def __init__(self, specs, precision='fp64', transform=None, slices=0, tiles=None, multi_deposit=False):
        """``transform``: one form or {N: form}; ``tiles``: {N: (deposit
        rows, FFT CTAs per SM)} as lc3d_set_tiles takes them (both as
        ``autotune`` returns them); ``multi_deposit``: every deposition point
        of a step is one launch over all simulations (lc3d_batch_set_mode)."""
        transform = transform or {}
        tiles = tiles or {}
        self.sims = [Sim(s, precision, transform.get(s['grid_steps'], 'auto') if isinstance(transform, dict)
                         else transform, slices, tiles.get(s['grid_steps'])) for s in specs]
        self._ctxs = (ctypes.c_void_p * len(self.sims))(*[s.solver.ctx.value for s in self.sims])
        self.handle = ctypes.c_void_p()
        check(lib.lc3d_batch_create(self._ctxs, len(self.sims), ctypes.byref(self.handle)), 'lc3d_batch_create')
        if multi_deposit:
            check(lib.lc3d_batch_set_mode(self.handle, 1), 'lc3d_batch_set_mode')

    def __del__(self):
        h = getattr(self, 'handle', None)
        if h is not None and h.value and lib is not None:
            lib.lc3d_batch_destroy(h)
            self.handle = None

    def run(self, nsteps):
        """Advance every simulation by ``nsteps`` steps; returns the list of
        Ez(0,0) histories (device tensors of nsteps values)."""
        n = len(self.sims)
        hist = [L._empty((max(nsteps, 1),)) for _ in range(n)]
        xi0 = (ctypes.c_int * n)(*[s.xi for s in self.sims])
        ptrs = (ctypes.c_void_p * n)(*[h.data_ptr() for h in hist])
        check(lib.lc3d_batch_run(self.handle, xi0, int(nsteps), ptrs, L._stream()), 'lc3d_batch_run')
        for s in self.sims:
            s.xi += nsteps
        return [h[:nsteps] for h in hist]

    def check_errors(self):
        for s in self.sims:
            check(lib.lc3d_check_error(s.solver.ctx, L._stream()), 'batch simulation')


def _time_sim(spec, precision, form, tiles, steps):
    """ms per graph-replayed step of one simulation, or None if the form is
    not available for this grid."""
    try:
        sim = Sim(spec, precision, form, tiles=tiles)
    except _lib.LC3DError:
        return None
    ez = L._empty((steps,))
    check(lib.lc3d_run(sim.solver.ctx, 0, 2, ctypes.c_void_p(ez.data_ptr()), L._stream()), 'warm')
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    check(lib.lc3d_run(sim.solver.ctx, 2, steps, ctypes.c_void_p(ez.data_ptr()), L._stream()), 'tune')
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


TILE_CHOICES = {'deposit_rows': (4, 8, 16), 'fft_ctas_per_sm': (0, 2)}


def autotune(grids, steps=6, precision='fp64'):
    """Pick, per grid size, the float64 transform form (FFT or dense) and
    the tile shapes (deposition fine rows per CTA; resident FFT CTAs per SM,
    0 = as many as fit) by timing a few graph-replayed steps of every
    combination on this GPU. Returns ({N: {'transform', 'deposit_rows',
    'fft_ctas_per_sm'}}, {N: {label: ms per step}})."""
    choice, timings = {}, {}
    for N in sorted(set(grids)):
        spec = dict(grid_steps=N, grid_step_size=16.0 / (N - 1), xi_step_size=0.01, amplitude=0.5,
                    sigma_r=1.0, length_factor=1.0)
        timings[N] = {}
        best = None
        for form in ('fft', 'dense'):
            for rows in TILE_CHOICES['deposit_rows']:
                for per_sm in (TILE_CHOICES['fft_ctas_per_sm'] if form == 'fft' else (0,)):
                    ms = _time_sim(spec, precision, form, (rows, per_sm), steps)
                    if ms is None:
                        continue
                    timings[N][f'{form} rows={rows} fft_per_sm={per_sm}'] = ms
                    if best is None or ms < best[0]:
                        best = (ms, {'transform': form, 'deposit_rows': rows, 'fft_ctas_per_sm': per_sm})
        choice[N] = best[1]
    return choice, timings


def autotune_transform(grids, steps=6, precision='fp64'):
    """The transform form part of ``autotune``: ({N: 'fft' | 'dense'},
    {N: {form: ms per step}}) at the default tile shapes."""
    choice, timings = {}, {}
    for N in sorted(set(grids)):
        spec = dict(grid_steps=N, grid_step_size=16.0 / (N - 1), xi_step_size=0.01, amplitude=0.5,
                    sigma_r=1.0, length_factor=1.0)
        timings[N] = {}
        for form in ('fft', 'dense'):
            ms = _time_sim(spec, precision, form, None, steps)
            if ms is not None:
                timings[N][form] = ms
        choice[N] = min(timings[N], key=timings[N].get)
    return choice, timings


# ---------------------------------------------------------------------------
# Several GPUs: one process per GPU, simulations partitioned by `partition`,
# no exchange during the run.
# ---------------------------------------------------------------------------

def max_over_ranks(value, dist=None):
    """The maximum of a per-rank float over all ranks (the elapsed time of a
    job is the slowest rank's)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    dev = 'cuda' if dist.get_backend() == 'nccl' else 'cpu'
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_histories(local, dist=None):
    """Merge every rank's {simulation index: Ez(0,0) history (numpy)} into
    one dict on every rank (one collective at the end of a run)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, {int(k): np.asarray(v) for k, v in local.items()})
    out = {}
    for p in parts:
        out.update(p)
    return out
